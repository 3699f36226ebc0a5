"""The C++ classes of include/dmrg_b200.hpp (reference class and member names
over the C ABI), compiled with g++ into a test program and run on the host.

Its host-only members must give what the C ABI gives, and the C ABI is pinned
to the reference elsewhere: QuickSort's order on the reference's golden cases,
ComputeTruncateDim's dimensions and re-sorted values on seeded cases, and the
model layer's MPO and quantum tables of a real and a complex input.  Without a
GPU, constructing a Context throws an Error carrying DMRG_E_CUDA.  The
device-side classes (RealTensorContraction, RealTensorLanczos,
RealTensorLattice's canonicalisations, RealTensorRundmrg) are compiled and
linked into the same program here; this test does not run them."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from dmrgcc_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden")
INPUTS = os.path.join(ROOT, "dmrgcc_b200", "inputs")
LIBDIR = os.path.join(ROOT, "dmrgcc_b200", "lib")


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    if not os.path.exists(os.path.join(LIBDIR, "libdmrg_b200.so")):
        build.build()
    exe = str(tmp_path_factory.mktemp("cxx") / "layer_host")
    subprocess.run(["g++", "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cxx", "layer_host.cc"), "-L", LIBDIR, "-ldmrg_b200",
                    f"-Wl,-rpath,{LIBDIR}", "-o", exe], check=True)
    return exe


def _truncate_cases(path):
    cases = []
    with open(path, "w") as f:
        for seed in range(20):
            rng = np.random.default_rng(seed)
            nsec = int(rng.integers(1, 12))
            pool = np.array([1e-14, 1e-13, 1e-6, 0.01, 0.1, 0.25, 0.5])
            sv = [np.sort(rng.choice(pool, size=int(rng.integers(1, 9))))[::-1].copy() for _ in range(nsec)]
            max_dim = int(rng.integers(-1, 20))
            canpre = float(rng.choice([1e-12, 0.0, 2.0, 1e-7]))
            toks = [str(nsec), str(max_dim), repr(canpre)]
            for s in sv:
                toks += [str(len(s))] + [repr(float(x)) for x in s]
            f.write(" ".join(toks) + "\n")
            cases.append((sv, max_dim, canpre))
    return cases


def _run(program, tmp_path, inp, model):
    trunc = str(tmp_path / "truncate_cases.txt")
    cases = _truncate_cases(trunc)
    r = subprocess.run([program, os.path.join(GOLD, "quicksort_cases.txt"), trunc, os.path.join(INPUTS, inp), model],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().split("\n")
    return cases, lines


def _by_tag(lines, tag):
    return [ln.split()[1:] for ln in lines if ln.split()[0] == tag]


def test_quicksort_and_truncation_through_the_cxx_classes(program, tmp_path):
    cases, lines = _run(program, tmp_path, "chain16_spinless.in", "real_spinless_bose_square")
    with open(os.path.join(GOLD, "quicksort_cases.txt")) as f:
        gold = f.read().strip().split("\n")[1::2]
    got = _by_tag(lines, "quicksort")
    assert len(got) == len(gold) == 40
    for g, want in zip(got, gold):
        assert [int(x) for x in g] == [int(x) for x in want.split()]
    # flag 2, empty and one-element ranges change nothing; v[1..3] sorted ascending
    edges = _by_tag(lines, "quicksort_edges")[0]
    assert edges == ["0:0.29999999999999999", "2:0.10000000000000001", "1:0.90000000000000002",
                     "3:0.90000000000000002", "4:0.5"]
    got = [" ".join(t).split("|") for t in _by_tag(lines, "truncate")]
    assert len(got) == len(cases)
    for (dims, vals), (sv, max_dim, canpre) in zip(got, cases):
        t_lib, s_lib = capi.truncate_dims([s.copy() for s in sv], max_dim, canpre)
        assert [int(x) for x in dims.split()] == list(t_lib)
        assert np.array_equal(np.array([float(x) for x in vals.split()]), np.concatenate(s_lib))


@pytest.mark.parametrize("inp,model", [("chain16_spinless.in", "real_spinless_bose_square"),
                                       ("hofstadter4x3.in", "complex_spinful_bose_square")])
def test_model_layer_through_the_cxx_classes(program, tmp_path, inp, model):
    _, lines = _run(program, tmp_path, inp, model)
    ref = capi.Model(os.path.join(INPUTS, inp), model)
    ns, d, nq, cplx = (int(x) for x in _by_tag(lines, "model")[0])
    assert (ns, d, nq, bool(cplx)) == (ref.num_site, ref.physics_dim, ref.num_quantum, ref.is_complex)
    mpos = _by_tag(lines, "mpo")
    assert len(mpos) == ns
    for rec in mpos:
        site, lb, rb = (int(x) for x in rec[:3])
        w = np.array([float(x) for x in rec[3:]])
        want = ref.mpo(site)
        assert want.shape[:2] == (lb, rb)
        want = want.view(np.float64).ravel() if ref.is_complex else want.ravel()
        assert np.array_equal(w, want)
    qts = _by_tag(lines, "quantum")
    assert len(qts) == 2 * (ns + 1)
    for rec in qts:
        which, bond, rows = (int(x) for x in rec[:3])
        want = ref.quantum_table(which, bond)
        assert want.shape[0] == rows
        assert [int(x) for x in rec[3:]] == list(want.ravel())
    ref.close()


def test_context_without_a_gpu_throws_cuda_error(program, tmp_path):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    _, lines = _run(program, tmp_path, "chain16_spinless.in", "real_spinless_bose_square")
    assert lines[-1] == f"context error {capi.E_CUDA}"
