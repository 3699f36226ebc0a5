"""The C-ABI library loads and exports every entry point that include/*.h
declares (no compute calls: CPU only)."""
import ctypes
import glob
import os
import re

import pytest

from dmrgcc_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_]*\s*\**\s+\**(dmrg_[A-Za-z0-9_]+)\s*\(", src,
                             flags=re.M):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def libpath():
    # Incremental: recompiles only units older than their sources (nvcc
    # cross-compiles for sm_100a without a GPU).
    try:
        build.nvcc()
        build.build()
    except RuntimeError:
        if not os.path.exists(capi.LIB_PATH):
            raise
    return capi.LIB_PATH


def test_header_parsed():
    names = header_functions()
    assert "dmrg_heff_apply" in names and "dmrg_env_apply" in names and len(names) >= 20


def test_library_exports_all_declared_symbols(libpath):
    capi._lib = None
    lib = ctypes.CDLL(libpath)
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header(libpath):
    assert set(header_functions()) <= set(capi.declared_symbols())


def test_version_and_error_string(libpath):
    L = capi.lib()
    assert b"sm_100a" in L.dmrg_version()
    assert L.dmrg_last_error() is not None


def test_null_arguments_are_rejected_without_gpu(libpath):
    L = capi.lib()
    assert L.dmrg_ctx_create(0, None) == -1
    assert L.dmrg_heff_flops(None, None, None) == -1
    assert b"null" in L.dmrg_last_error()
