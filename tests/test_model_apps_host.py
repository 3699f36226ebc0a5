"""The reference's model executables rebuilt on the library
(dmrgcc_b200/csrc/apps/model_main.cc: real_spinless_bose_square_model,
complex_spinless_bose_square_model, complex_spinful_bose_square_model,
real_spinful_bose_square_model) and the
optional input keys that choose the run options (dmrg_run_options_from_input),
host side: usage and error behaviour as the reference's main()
(model/real_spinless_bose_square_model.cc:3-9), the keys' defaults and values,
and, without a GPU, a clean CUDA error instead of a crash."""
import ctypes as C
import os
import subprocess

import pytest

from dmrgcc_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INPUTS = os.path.join(ROOT, "dmrgcc_b200", "inputs")
CHAIN = os.path.join(INPUTS, "chain6_spinless.in")


@pytest.fixture(scope="module")
def apps():
    build.build()
    paths = {name: os.path.join(build.LIBDIR, name) for name in build.APPS}
    for p in paths.values():
        assert os.access(p, os.X_OK), p
    return paths


def _with_keys(tmp_path, lines, name="opts.in"):
    with open(CHAIN) as f:
        text = f.read()
    head, rest = text.split("{", 1)
    p = tmp_path / name
    p.write_text(head + "{\n" + "".join(f"    {ln}\n" for ln in lines) + rest)
    return str(p)


def test_usage_as_the_reference(apps):
    for exe in apps.values():
        r = subprocess.run([exe], capture_output=True, text=True, timeout=60)
        assert r.returncode == 0
        assert r.stdout == f"Usage: {exe} inputfile"


def test_missing_input_file(apps, tmp_path):
    r = subprocess.run([apps["real_spinless_bose_square_model"], str(tmp_path / "missing.in")],
                       capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
    assert "can't open input file" in r.stderr


def test_without_a_gpu_the_run_reports_a_cuda_error(apps):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    r = subprocess.run([apps["real_spinless_bose_square_model"], CHAIN], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1
    assert r.stderr.startswith("dmrg_ctx_create:")


def test_reference_input_gives_the_reference_options():
    o = capi.run_options_from_input(CHAIN)
    assert (o.precision, o.verbose, o.seed, o.stop_after_half_sweeps, o.lanczos_precision, o.two_site,
            o.lanczos_graph) == (capi.DMRG_PREC_FP64, 1, 1, -1, 0.0, 0, 0)


def test_optional_keys(tmp_path):
    p = _with_keys(tmp_path, ["precision = tf32x3", "mode = twosite", "seed = 7", "lanczos_tol = 1e-12",
                              "lanczos_graph = -1"])
    o = capi.run_options_from_input(p)
    assert (o.precision, o.two_site, o.seed, o.lanczos_precision, o.lanczos_graph) == (
        capi.DMRG_PREC_TF32X3, 1, 7, 1e-12, -1)
    o = capi.run_options_from_input(_with_keys(tmp_path, ["precision = bf16x3", "mode = onesite"], "b.in"))
    assert (o.precision, o.two_site) == (capi.DMRG_PREC_BF16X3, 0)
    # the model layer reads the same file unchanged
    m = capi.Model(p)
    assert m.num_site == 6
    m.close()


@pytest.mark.parametrize("bad", ["precision = fp16", "mode = threesite", "seed = -3", "lanczos_tol = -1",
                                 "lanczos_graph = 2"])
def test_invalid_option_values(tmp_path, bad):
    with pytest.raises(capi.DmrgError) as err:
        capi.run_options_from_input(_with_keys(tmp_path, [bad]))
    assert err.value.code == capi.E_ARG
    assert bad.split("=")[0].strip() in str(err.value)


def test_null_arguments():
    lib = capi.lib()
    o = capi.RunOptions()
    assert lib.dmrg_run_options_from_input(None, C.byref(o)) == capi.E_ARG
    assert lib.dmrg_run_options_from_input(CHAIN.encode(), None) == capi.E_ARG
