"""Malformed input files and out-of-range queries of the model layer (host code,
CPU only).  The reference's InputGroup prints and exits on a missing file, a
missing key or an unterminated group (src/util/input.cc); the library returns
DMRG_E_ARG with the reason instead, and never crashes on such input."""
import ctypes as C
import os

import numpy as np
import pytest

from dmrgcc_b200 import capi

INPUTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "dmrgcc_b200", "inputs")
CHAIN = os.path.join(INPUTS, "chain6_spinless.in")


def _create(path, model="real_spinless_bose_square"):
    h = C.c_void_p()
    rc = capi.lib().dmrg_model_create(path.encode(), model.encode(), C.byref(h))
    return rc, h, capi.lib().dmrg_last_error().decode()


def _variant(tmp_path, old, new, name="bad.in"):
    with open(CHAIN) as f:
        text = f.read()
    assert old in text
    p = tmp_path / name
    p.write_text(text.replace(old, new, 1))
    return str(p)


def test_missing_file(tmp_path):
    rc, h, msg = _create(str(tmp_path / "nope.in"))
    assert rc == capi.E_ARG and not h.value
    assert "can't open input file" in msg


def test_missing_key(tmp_path):
    rc, _, msg = _create(_variant(tmp_path, "num_boson", "num_bosons_typo"))
    assert rc == capi.E_ARG
    assert "num_boson" in msg


def test_group_name_without_bracket(tmp_path):
    rc, _, msg = _create(_variant(tmp_path, "input\n{", "input\n("))
    assert rc == capi.E_ARG
    assert "bracket does not follow group name" in msg


def test_unknown_model():
    rc, _, msg = _create(CHAIN, "no_such_model")
    assert rc == capi.E_ARG and msg


def test_empty_file(tmp_path):
    p = tmp_path / "empty.in"
    p.write_text("")
    rc, _, msg = _create(str(p))
    assert rc == capi.E_ARG and msg


def test_model_queries_out_of_range():
    m = capi.Model(CHAIN)
    lib = capi.lib()
    lb, rb = C.c_int(), C.c_int()
    for site in (-1, m.num_site):
        assert lib.dmrg_model_mpo(m.h, site, C.byref(lb), C.byref(rb), 0, None) == capi.E_ARG
    # a buffer smaller than the tensor receives `cap` values and nothing beyond
    assert lib.dmrg_model_mpo(m.h, 0, C.byref(lb), C.byref(rb), 0, None) == 0
    need = lb.value * rb.value * m.physics_dim ** 2
    buf = np.full(need, 12345.0)
    assert lib.dmrg_model_mpo(m.h, 0, C.byref(lb), C.byref(rb), need - 1,
                              buf.ctypes.data_as(C.POINTER(C.c_double))) == 0
    assert buf[need - 1] == 12345.0
    assert np.array_equal(buf[:need - 1], m.mpo(0).ravel()[:need - 1])
    rows = C.c_int()
    for which, bond in ((0, -1), (0, m.num_site + 1), (2, 0)):
        assert lib.dmrg_model_quantum_table(m.h, which, bond, 0, None, C.byref(rows)) == capi.E_ARG
    m.close()


@pytest.mark.parametrize("bad", ["physics_dim = 0", "physics_dim = 1", "num_site_x = 0", "num_boson = -1",
                                 "num_boson = 1000"])
def test_nonphysical_sizes_are_rejected(tmp_path, bad):
    key = bad.split("=")[0].strip()
    with open(CHAIN) as f:
        lines = f.read().split("\n")
    out = [f"    {bad}" if ln.strip().startswith(key + " ") or ln.strip().startswith(key + "=") else ln
           for ln in lines]
    p = tmp_path / "nonphysical.in"
    p.write_text("\n".join(out))
    rc, _, msg = _create(str(p))
    assert rc == capi.E_ARG and msg


def test_every_shipped_input_builds_its_model():
    """Every input file under dmrgcc_b200/inputs passes the model layer's size
    checks: spinless files as the real and the complex spinless model, spinful
    ones as the complex spinful model, and as the real one where the flux is 0."""
    for name in sorted(os.listdir(INPUTS)):
        path = os.path.join(INPUTS, name)
        with open(path) as f:
            text = f.read()
        if "Nup" in text:
            models = ["complex_spinful_bose_square"]
            flux = [ln for ln in text.splitlines() if ln.strip().startswith("flux")][0]
            if float(flux.split("=")[1]) == 0.0:
                models.append("real_spinful_bose_square")
        else:
            models = ["real_spinless_bose_square", "complex_spinless_bose_square"]
        for model in models:
            rc, h, msg = _create(path, model)
            assert rc == 0, (name, model, msg)
            capi.lib().dmrg_model_destroy(h)
