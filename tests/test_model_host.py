"""Model layer of the product library (host only): the MPO built by the
deparallelising term-by-term construction and the quantum-number tables are
bit-identical to the reference's (dumped by oracle/_ref/probe_dump)."""
import os

import numpy as np
import pytest

from dmrgcc_b200 import build, capi
from oracle.nac import read_nac

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
CASES = [("chain16_spinless.in", "model_chain16.nac"), ("cylinder8x4_spinless.in", "model_cyl8x4.nac")]


@pytest.fixture(scope="module", autouse=True)
def _lib():
    try:
        build.nvcc()
        build.build()
    except RuntimeError:
        pass
    capi._lib = None
    capi.lib()


@pytest.mark.parametrize("inp,gold", CASES)
def test_mpo_and_quantum_tables_bit_exact(inp, gold):
    ref = read_nac(os.path.join(GOLD, gold))
    m = capi.Model(os.path.join(ROOT, "dmrgcc_b200", "inputs", inp))
    n = int(ref["num_site"][0])
    assert m.num_site == n
    for i in range(n):
        W = m.mpo(i)
        d, lb, rb = (int(x) for x in ref[f"op{i}.dims"])
        assert W.shape == (lb, rb, d, d)
        assert np.array_equal(W.ravel(), ref[f"op{i}.W"])  # bit-exact doubles
    for b in range(n + 1):
        assert np.array_equal(m.quantum_table(0, b).ravel(), ref[f"sq{b}"])
        assert np.array_equal(m.quantum_table(1, b).ravel(), ref[f"hq{b}"])


@pytest.mark.parametrize("name", ["spinful4x4", "spinful3x3_periodic_y"])
def test_spinful_mpo_and_quantum_tables_bit_exact(name):
    """The spinful U(1) x U(1) model (species on alternating MPS sites): MPO and
    quantum tables bit-identical to the reference's ComplexSpinfulBoseSquare
    classes at zero flux (oracle/_ref/probe_model); the 4x4 open lattice is
    the spinful benchmark geometry, 3x3 periodic in y exercises the wrap-around terms."""
    ref = read_nac(os.path.join(GOLD, f"model_{name}.nac"))
    m = capi.Model(os.path.join(ROOT, "dmrgcc_b200", "inputs", f"{name}.in"), "real_spinful_bose_square")
    n = int(ref["num_site"][0])
    assert m.num_site == n and m.num_quantum == 2
    for i in range(n):
        W = m.mpo(i)
        d, lb, rb = (int(x) for x in ref[f"op{i}.dims"])
        assert W.shape == (lb, rb, d, d)
        assert np.array_equal(W.ravel(), ref[f"op{i}.W"])
    for b in range(n + 1):
        assert np.array_equal(m.quantum_table(0, b).ravel(), ref[f"sq{b}"])
        assert np.array_equal(m.quantum_table(1, b).ravel(), ref[f"hq{b}"])


def test_spinful_model_rejects_flux(tmp_path):
    """The Peierls phases of a nonzero flux need complex tensors."""
    src = open(os.path.join(ROOT, "dmrgcc_b200", "inputs", "spinful3x2.in")).read()
    p = tmp_path / "flux.in"
    p.write_text(src.replace("flux = 0.0", "flux = 0.1666666666666667"))
    with pytest.raises(capi.DmrgError):
        capi.Model(str(p), "real_spinful_bose_square")


def test_spinful_exact_diagonalisation_matches_reference():
    """oracle/ed.py's spinful ground energy equals the reference's converged run
    of the same 3x2 input (D = 729 covers the whole space): pins the ED."""
    from oracle.ed import ground_energy_spinful

    with open(os.path.join(GOLD, "spinful_reference.txt")) as f:
        e_ref = float([ln.split()[1] for ln in f if ln.startswith("spinful3x2")][0])
    e = ground_energy_spinful(3, 2, 3, 3, 3, -1.0, -1.0, 6.0, 6.0, 3.0, 0.0)
    assert abs(e - e_ref) / 12 <= 1e-12


def test_complex_spinful_mpo_with_flux_bit_exact():
    """The complex spinful model with the Peierls phases exp(i 2 pi (x+1) flux)
    on the y-bonds (hofstadter4x3.in: flux 1/6, periodic in y, one species
    filled): every complex MPO entry and both quantum tables bit-identical to
    the reference's ComplexSpinfulBoseSquare classes (oracle/_ref/probe_model)."""
    ref = read_nac(os.path.join(GOLD, "model_hofstadter4x3.nac"))
    m = capi.Model(os.path.join(ROOT, "dmrgcc_b200", "inputs", "hofstadter4x3.in"), "complex_spinful_bose_square")
    assert m.is_complex
    n = int(ref["num_site"][0])
    assert m.num_site == n and m.num_quantum == 2
    assert any(np.any(ref[f"op{i}.Wi"]) for i in range(n))
    for i in range(n):
        W = m.mpo(i)
        d, lb, rb = (int(x) for x in ref[f"op{i}.dims"])
        assert W.shape == (lb, rb, d, d)
        assert np.array_equal(W.real.ravel(), ref[f"op{i}.W"])
        assert np.array_equal(W.imag.ravel(), ref[f"op{i}.Wi"])
    for b in range(n + 1):
        assert np.array_equal(m.quantum_table(0, b).ravel(), ref[f"sq{b}"])
        assert np.array_equal(m.quantum_table(1, b).ravel(), ref[f"hq{b}"])


def test_hofstadter_exact_diagonalisation_matches_reference():
    """oracle/ed.py with the Peierls phase equals the reference's converged complex
    run of hofstadter4x3.in (its last Lanczos energy, tests/golden/
    steps_hofstadter4x3.txt; D = 64 spans the 3-boson space): pins the complex ED."""
    from oracle.ed import ground_energy_spinful

    with open(os.path.join(GOLD, "steps_hofstadter4x3.txt")) as f:
        e_ref = float([ln.split() for ln in f if ln.strip() and not ln.startswith("#")][-1][4])
    e = ground_energy_spinful(4, 3, 3, 0, 3, -1.0, -1.0, 10.0, 0.0, 0.0, 0.0, False, True, flux=0.16666666666666666)
    assert abs(e - e_ref) / 12 <= 1e-12
    e0 = ground_energy_spinful(4, 3, 3, 0, 3, -1.0, -1.0, 10.0, 0.0, 0.0, 0.0, False, True)
    assert e0 < e - 1.0  # the flux matters


@pytest.mark.parametrize("name", ["chain16_spinless", "cylinder3x3_spinless"])
def test_complex_spinless_mpo_bit_exact(name):
    """The complex spinless model (model/complex_spinless_bose_square_model.cc:
    the real spinless terms on complex operators, run by the complex engine):
    every complex MPO entry and both quantum tables bit-identical to the
    reference's ComplexSpinlessBoseSquare classes (oracle/_ref/probe_model ...
    spinless), and its real parts equal to the real spinless model's MPO."""
    ref = read_nac(os.path.join(GOLD, f"model_complex_{name}.nac"))
    inp = os.path.join(ROOT, "dmrgcc_b200", "inputs", f"{name}.in")
    m = capi.Model(inp, "complex_spinless_bose_square")
    real = capi.Model(inp)
    assert m.is_complex and not real.is_complex
    n = int(ref["num_site"][0])
    assert m.num_site == n and m.num_quantum == 1
    for i in range(n):
        W = m.mpo(i)
        d, lb, rb = (int(x) for x in ref[f"op{i}.dims"])
        assert W.shape == (lb, rb, d, d)
        assert np.array_equal(W.real.ravel(), ref[f"op{i}.W"])
        assert np.array_equal(W.imag.ravel(), ref[f"op{i}.Wi"])
        Wr = real.mpo(i)
        assert Wr.shape == W.shape and np.array_equal(Wr, W.real)
    for b in range(n + 1):
        assert np.array_equal(m.quantum_table(0, b).ravel(), ref[f"sq{b}"])
        assert np.array_equal(m.quantum_table(1, b).ravel(), ref[f"hq{b}"])
    m.close()
    real.close()
