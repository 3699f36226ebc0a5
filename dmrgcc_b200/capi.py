"""ctypes binding of the libdmrg_b200 C ABI (include/dmrg_b200.h).

The library is the product: every numeric call here goes to the sm_100a
kernels.  There is no CPU fallback; loading fails loudly when the shared
library has not been built (python -m dmrgcc_b200.build).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "lib", "libdmrg_b200.so")

DMRG_PREC_FP64 = 0
DMRG_PREC_BF16X3 = 1
DMRG_PREC_TF32X3 = 2

# status codes (DMRG_OK, DMRG_E_*)
OK, E_ARG, E_CUDA, E_NOMEM, E_NUMERIC, E_STATE, E_IO = 0, -1, -2, -3, -4, -5, -6

_lib: C.CDLL | None = None


class DmrgError(RuntimeError):
    def __init__(self, code: int, where: str):
        msg = lib().dmrg_last_error().decode()
        super().__init__(f"{where} failed ({code}): {msg}")
        self.code = code


class Blocks(C.Structure):
    """dmrg_blocks_t."""

    _fields_ = [("nblocks", C.c_int), ("left", C.POINTER(C.c_int)), ("right", C.POINTER(C.c_int)),
                ("rows", C.POINTER(C.c_int)), ("cols", C.POINTER(C.c_int))]


_I = C.POINTER(C.c_int)
_D = C.POINTER(C.c_double)
_I64 = C.POINTER(C.c_int64)
_VP = C.c_void_p

_SIGS = {
    "dmrg_version": (C.c_char_p, []),
    "dmrg_last_error": (C.c_char_p, []),
    "dmrg_ctx_create": (C.c_int, [C.c_int, C.POINTER(_VP)]),
    "dmrg_ctx_destroy": (C.c_int, [_VP]),
    "dmrg_ctx_set_stream": (C.c_int, [_VP, _VP]),
    "dmrg_ctx_stream": (_VP, [_VP]),
    "dmrg_ctx_sync": (C.c_int, [_VP]),
    "dmrg_malloc": (C.c_int, [_VP, C.c_size_t, C.POINTER(_VP)]),
    "dmrg_free": (C.c_int, [_VP, _VP]),
    "dmrg_memcpy_h2d": (C.c_int, [_VP, _VP, _VP, C.c_size_t]),
    "dmrg_memcpy_d2h": (C.c_int, [_VP, _VP, _VP, C.c_size_t]),
    "dmrg_memset": (C.c_int, [_VP, _VP, C.c_int, C.c_size_t]),
    "dmrg_fill_uniform": (C.c_int, [_VP, _VP, C.c_int64, C.c_uint64, C.c_int64]),
    "dmrg_fp64_peak": (C.c_int, [_VP, C.c_int, C.c_int, _D]),
    "dmrg_launch_count": (C.c_int, [_I64]),
    "dmrg_heff_create": (C.c_int, [_VP, C.c_int, C.c_int, _I, C.POINTER(Blocks), C.c_int, C.c_int, C.c_int, _D,
                                   C.POINTER(Blocks), C.POINTER(Blocks), C.c_int, C.POINTER(_VP)]),
    "dmrg_heff_create_blocks": (C.c_int, [_VP, C.c_int, C.c_int, _I, C.POINTER(Blocks), C.c_int, C.c_int, C.c_int,
                                          _D, C.POINTER(Blocks), C.POINTER(Blocks), C.c_int, C.POINTER(_VP)]),
    "dmrg_heff_destroy": (C.c_int, [_VP]),
    "dmrg_heff_set_split_threshold": (C.c_int, [_VP, C.c_int64]),
    "dmrg_heff_split_iters": (C.c_int, [_VP, _I]),
    "dmrg_lanczos_set_polish": (C.c_int, [C.c_int]),
    "dmrg_heff_set_graph": (C.c_int, [_VP, C.c_int]),
    "dmrg_heff_sizes": (C.c_int, [_VP, _I64, _I64, _I64]),
    "dmrg_heff_flops": (C.c_int, [_VP, _D, _D]),
    "dmrg_heff_set_env": (C.c_int, [_VP, _VP, _VP]),
    "dmrg_heff_apply": (C.c_int, [_VP, _VP, _VP, C.c_int]),
    "dmrg_heff_apply_host": (C.c_int, [_VP, _VP, _VP, C.c_int]),
    "dmrg_heff_profile": (C.c_int, [_VP, _VP, _VP, _D, _D]),
    "dmrg_heff_apply_noalloc": (C.c_int, [C.c_int, C.c_int, _I, C.POINTER(Blocks), C.c_int, C.c_int, C.c_int, _D,
                                          C.POINTER(Blocks), C.POINTER(Blocks), _VP, _VP, _VP, _VP, C.c_int, _VP]),
    "dmrg_lanczos": (C.c_int, [_VP, _VP, C.c_int, C.c_double, C.c_double, _D, _I]),
    "dmrg_zheff_create": (C.c_int, [_VP, C.c_int, C.c_int, _I, C.POINTER(Blocks), C.c_int, C.c_int, C.c_int, _D,
                                    C.POINTER(Blocks), C.POINTER(Blocks), C.POINTER(_VP)]),
    "dmrg_zheff_destroy": (C.c_int, [_VP]),
    "dmrg_zheff_sizes": (C.c_int, [_VP, _I64, _I64, _I64, _D]),
    "dmrg_zheff_set_env": (C.c_int, [_VP, _VP, _VP]),
    "dmrg_zheff_apply": (C.c_int, [_VP, _VP, _VP, C.c_int]),
    "dmrg_zlanczos": (C.c_int, [_VP, _VP, C.c_int, C.c_double, C.c_double, _D, _I]),
    "dmrg_zenv_create": (C.c_int, [_VP, C.c_int, C.c_int, C.c_int, _I, C.POINTER(Blocks), C.c_int, C.c_int, C.c_int,
                                   _D, C.POINTER(Blocks), C.POINTER(_VP)]),
    "dmrg_zenv_apply": (C.c_int, [_VP, _VP, _VP, _VP]),
    "dmrg_canon_create": (C.c_int, [_VP, C.c_int, C.c_int, C.c_int, _I, _I, C.POINTER(Blocks), C.POINTER(_VP)]),
    "dmrg_canon_destroy": (C.c_int, [_VP]),
    "dmrg_canon_run": (C.c_int, [_VP, _VP, C.c_int, C.c_double, _I, _D]),
    "dmrg_canon_out_info": (C.c_int, [_VP, _I64, _I64, _I]),
    "dmrg_canon_out_blocks": (C.c_int, [_VP, _I, _I, _I, _I, _I]),
    "dmrg_canon_singular_values": (C.c_int, [_VP, C.c_int, C.c_int, _D, _I]),
    "dmrg_canon_write": (C.c_int, [_VP, _VP, _VP, _VP]),
    "dmrg_zcanon_create": (C.c_int, [_VP, C.c_int, C.c_int, C.c_int, _I, _I, C.POINTER(Blocks), C.POINTER(_VP)]),
    "dmrg_zcanon_destroy": (C.c_int, [_VP]),
    "dmrg_zcanon_run": (C.c_int, [_VP, _VP, C.c_int, C.c_double, _I, _D]),
    "dmrg_zcanon_out_info": (C.c_int, [_VP, _I64, _I64, _I]),
    "dmrg_zcanon_out_blocks": (C.c_int, [_VP, _I, _I, _I, _I, _I]),
    "dmrg_zcanon_singular_values": (C.c_int, [_VP, C.c_int, C.c_int, _D, _I]),
    "dmrg_zcanon_write": (C.c_int, [_VP, _VP, _VP, _VP]),
    "dmrg_svd_pair_schedule": (C.c_int, [C.POINTER(C.c_uint)]),
    "dmrg_svd_plan_rounds": (C.c_int, [C.c_int, C.POINTER(C.c_double), C.c_double, C.c_int, C.POINTER(C.c_int),
                                       C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "dmrg_svd_set_max_sweeps": (C.c_int, [C.c_int]),
    "dmrg_quicksort_index": (C.c_int, [_D, _I, C.c_int, C.c_int]),
    "dmrg_truncate_dims": (C.c_int, [C.c_int, _I, _D, C.c_int, C.c_double, _I]),
    "dmrg_rand_stream": (C.c_int, [C.c_uint, C.c_int, _I]),
    "dmrg_run_create": (C.c_int, [_VP, C.c_char_p, C.c_char_p, _VP, C.POINTER(_VP)]),
    "dmrg_run_options_from_input": (C.c_int, [C.c_char_p, _VP]),
    "dmrg_run_execute": (C.c_int, [_VP]),
    "dmrg_run_execute_many": (C.c_int, [C.POINTER(_VP), C.c_int, C.c_int, _I]),
    "dmrg_run_destroy": (C.c_int, [_VP]),
    "dmrg_run_half_sweeps": (C.c_int, [_VP, C.c_int, _D, _D, _I]),
    "dmrg_run_steps": (C.c_int, [_VP, C.c_int, _I, _I, _D, _I, _D, _I64, _D, _I]),
    "dmrg_run_phases": (C.c_int, [_VP, C.c_int, _D, _I, _I]),
    "dmrg_model_create": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(_VP)]),
    "dmrg_model_destroy": (C.c_int, [_VP]),
    "dmrg_model_info": (C.c_int, [_VP, _I, _I, _I]),
    "dmrg_model_mpo": (C.c_int, [_VP, C.c_int, _I, _I, C.c_int, _D]),
    "dmrg_model_is_complex": (C.c_int, [_VP, _I]),
    "dmrg_model_quantum_table": (C.c_int, [_VP, C.c_int, C.c_int, C.c_int, _I, _I]),
    "dmrg_env_create": (C.c_int, [_VP, C.c_int, C.c_int, C.c_int, _I, C.POINTER(Blocks), C.c_int, C.c_int, C.c_int,
                                  _D, C.POINTER(Blocks), C.c_int, C.POINTER(_VP)]),
    "dmrg_env_destroy": (C.c_int, [_VP]),
    "dmrg_env_out_info": (C.c_int, [_VP, _I, _I64]),
    "dmrg_env_out_blocks": (C.c_int, [_VP, C.c_int, C.c_int, _I, _I, _I, _I, _I]),
    "dmrg_env_flops": (C.c_int, [_VP, _D, _D]),
    "dmrg_env_apply": (C.c_int, [_VP, _VP, _VP, _VP]),
}


def declared_symbols() -> list[str]:
    """Every entry point bound here (all of include/dmrg_b200.h)."""
    return sorted(_SIGS)


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `python -m dmrgcc_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int, where: str) -> None:
    if rc != 0:
        raise DmrgError(rc, where)


def launch_count() -> int:
    """Kernels the library has launched in this process (dmrg_launch_count)."""
    n = C.c_int64(0)
    check(lib().dmrg_launch_count(C.byref(n)), "dmrg_launch_count")
    return int(n.value)


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(_I)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(_D)


class BlockSpec:
    """Shape of one block list (the sector indices and sizes of a RealMatrixBlock)."""

    def __init__(self, left: Sequence[int], right: Sequence[int], rows: Sequence[int], cols: Sequence[int]):
        self.left = np.ascontiguousarray(left, dtype=np.int32)
        self.right = np.ascontiguousarray(right, dtype=np.int32)
        self.rows = np.ascontiguousarray(rows, dtype=np.int32)
        self.cols = np.ascontiguousarray(cols, dtype=np.int32)

    @property
    def size(self) -> int:
        return int(np.sum(self.rows.astype(np.int64) * self.cols.astype(np.int64)))

    def c(self) -> Blocks:
        return Blocks(len(self.left), _iptr(self.left), _iptr(self.right), _iptr(self.rows), _iptr(self.cols))


def _blocks_array(specs: Sequence[BlockSpec]):
    arr = (Blocks * max(len(specs), 1))()
    for i, s in enumerate(specs):
        arr[i] = s.c()
    return arr


class Context:
    def __init__(self, device: int = 0):
        h = _VP()
        check(lib().dmrg_ctx_create(device, C.byref(h)), "dmrg_ctx_create")
        self.h = h

    def close(self) -> None:
        if self.h:
            lib().dmrg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_stream(self, stream_ptr: int | None) -> None:
        check(lib().dmrg_ctx_set_stream(self.h, stream_ptr), "dmrg_ctx_set_stream")

    @property
    def stream(self) -> int:
        return lib().dmrg_ctx_stream(self.h) or 0

    def sync(self) -> None:
        check(lib().dmrg_ctx_sync(self.h), "dmrg_ctx_sync")

    def fp64_peak(self, mode: int = 0, iters: int = 20000) -> float:
        """Measured FP64 TFLOP/s (mode 0: DMMA, 1: DFMA)."""
        t = C.c_double()
        check(lib().dmrg_fp64_peak(self.h, mode, iters, C.byref(t)), "dmrg_fp64_peak")
        return t.value


class DeviceArray:
    """A float64 device buffer allocated through the C ABI."""

    def __init__(self, ctx: Context, n: int):
        self.ctx, self.n = ctx, int(n)
        p = _VP()
        check(lib().dmrg_malloc(ctx.h, max(self.n, 1) * 8, C.byref(p)), "dmrg_malloc")
        self.ptr = p.value

    @classmethod
    def from_host(cls, ctx: Context, a: np.ndarray) -> "DeviceArray":
        a = np.ascontiguousarray(a, dtype=np.float64).ravel()
        d = cls(ctx, a.size)
        d.upload(a)
        return d

    def upload(self, a: np.ndarray) -> None:
        a = np.ascontiguousarray(a, dtype=np.float64).ravel()
        assert a.size == self.n
        check(lib().dmrg_memcpy_h2d(self.ctx.h, self.ptr, a.ctypes.data, a.nbytes), "dmrg_memcpy_h2d")

    def download(self) -> np.ndarray:
        out = np.empty(self.n, dtype=np.float64)
        check(lib().dmrg_memcpy_d2h(self.ctx.h, out.ctypes.data, self.ptr, out.nbytes), "dmrg_memcpy_d2h")
        return out

    def fill_uniform(self, seed: int, start: int = 0) -> None:
        check(lib().dmrg_fill_uniform(self.ctx.h, self.ptr, self.n, seed, start), "dmrg_fill_uniform")

    def zero(self) -> None:
        check(lib().dmrg_memset(self.ctx.h, self.ptr, 0, self.n * 8), "dmrg_memset")

    def free(self) -> None:
        if self.ptr:
            lib().dmrg_free(self.ctx.h, self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class SiteProblem:
    """Block structure of one site: sectors, ket blocks, MPO tensor."""

    def __init__(self, nl: int, nr: int, phys: np.ndarray | None, ket: BlockSpec, W: np.ndarray,
                 block_phys: np.ndarray | None = None):
        """`phys`: physics index per sector pair (nl x nr, -1 = no block), or None
        with `block_phys`: one physics index per ket block (two-site tensors)."""
        self.nl, self.nr = int(nl), int(nr)
        self.block_phys = None if block_phys is None else np.ascontiguousarray(block_phys, dtype=np.int32)
        if phys is None:
            assert self.block_phys is not None and self.block_phys.size == len(ket.left)
            self.phys = None
        else:
            self.phys = np.ascontiguousarray(phys, dtype=np.int32).reshape(-1)
            assert self.phys.size == self.nl * self.nr
        self.ket = ket
        self.W = np.ascontiguousarray(W, dtype=np.float64)
        self.lb, self.rb, self.d = self.W.shape[0], self.W.shape[1], self.W.shape[2]


class Heff:
    """H_eff*psi operator (MultiplyEffectHamilton)."""

    def __init__(self, ctx: Context, site: SiteProblem, L: Sequence[BlockSpec], R: Sequence[BlockSpec],
                 precision: int = DMRG_PREC_FP64):
        self.ctx, self.site = ctx, site
        self._L, self._R = _blocks_array(L), _blocks_array(R)
        kb = site.ket.c()
        h = _VP()
        if site.block_phys is not None:
            check(lib().dmrg_heff_create_blocks(ctx.h, site.nl, site.nr, _iptr(site.block_phys), C.byref(kb), site.d,
                                                site.lb, site.rb, _dptr(site.W), self._L, self._R, precision,
                                                C.byref(h)), "dmrg_heff_create_blocks")
        else:
            check(lib().dmrg_heff_create(ctx.h, site.nl, site.nr, _iptr(site.phys), C.byref(kb), site.d, site.lb,
                                         site.rb, _dptr(site.W), self._L, self._R, precision, C.byref(h)),
                  "dmrg_heff_create")
        self.h = h
        a, b, c = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().dmrg_heff_sizes(h, C.byref(a), C.byref(b), C.byref(c)), "dmrg_heff_sizes")
        self.psi_dim, self.l_size, self.r_size = a.value, b.value, c.value

    def flops(self) -> tuple[float, float]:
        a, e = C.c_double(), C.c_double()
        check(lib().dmrg_heff_flops(self.h, C.byref(a), C.byref(e)), "dmrg_heff_flops")
        return a.value, e.value

    def set_env(self, L_dev: DeviceArray, R_dev: DeviceArray) -> None:
        self._env_refs = (L_dev, R_dev)
        check(lib().dmrg_heff_set_env(self.h, L_dev.ptr, R_dev.ptr), "dmrg_heff_set_env")

    def apply(self, psi: DeviceArray, out: DeviceArray, accumulate: bool = False) -> None:
        check(lib().dmrg_heff_apply(self.h, psi.ptr, out.ptr, int(accumulate)), "dmrg_heff_apply")

    def apply_ptr(self, psi_ptr: int, out_ptr: int, accumulate: bool = False) -> None:
        check(lib().dmrg_heff_apply(self.h, psi_ptr, out_ptr, int(accumulate)), "dmrg_heff_apply")

    def profile(self, psi: DeviceArray, out: DeviceArray) -> tuple[float, float]:
        """Durations (ms) of the two grouped launches of one accumulating apply."""
        a, b = C.c_double(), C.c_double()
        check(lib().dmrg_heff_profile(self.h, psi.ptr, out.ptr, C.byref(a), C.byref(b)), "dmrg_heff_profile")
        return a.value, b.value

    def apply_host(self, psi: np.ndarray, out: np.ndarray, accumulate: bool = False) -> None:
        check(lib().dmrg_heff_apply_host(self.h, psi.ctypes.data, out.ctypes.data, int(accumulate)),
              "dmrg_heff_apply_host")

    def set_split_threshold(self, min_psi_dim: int) -> None:
        check(lib().dmrg_heff_set_split_threshold(self.h, int(min_psi_dim)), "dmrg_heff_set_split_threshold")

    def split_iters(self) -> int:
        it = C.c_int(0)
        check(lib().dmrg_heff_split_iters(self.h, C.byref(it)), "dmrg_heff_split_iters")
        return it.value

    def set_graph(self, enable: bool) -> None:
        """Lanczos loop as one captured CUDA graph (default) or launch by launch."""
        check(lib().dmrg_heff_set_graph(self.h, int(bool(enable))), "dmrg_heff_set_graph")

    def lanczos(self, psi: DeviceArray, niter: int, precision: float = 1e-15,
                zero_tol: float = 1e-15) -> tuple[float, int]:
        """Ground state in place (psi: start vector -> ground vector). Returns (E, dim)."""
        e, it = C.c_double(), C.c_int()
        check(lib().dmrg_lanczos(self.h, psi.ptr, niter, precision, zero_tol, C.byref(e), C.byref(it)),
              "dmrg_lanczos")
        return e.value, it.value

    def close(self) -> None:
        if self.h:
            lib().dmrg_heff_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ZHeff:
    """Complex H_eff*psi operator (ComplexTensorContraction::MultiplyEffectHamilton)
    and its Lanczos ground state.  Device arrays hold interleaved (re, im) doubles:
    twice as many doubles as complex elements."""

    def __init__(self, ctx: Context, site: SiteProblem, L: Sequence[BlockSpec], R: Sequence[BlockSpec],
                 Wc: np.ndarray):
        self.ctx, self.site = ctx, site
        self._L, self._R = _blocks_array(L), _blocks_array(R)
        self._W = np.ascontiguousarray(np.asarray(Wc, dtype=np.complex128)).view(np.float64)
        kb = site.ket.c()
        h = _VP()
        check(lib().dmrg_zheff_create(ctx.h, site.nl, site.nr, _iptr(site.phys), C.byref(kb), site.d, site.lb,
                                      site.rb, _dptr(self._W), self._L, self._R, C.byref(h)), "dmrg_zheff_create")
        self.h = h
        a, b, c, f = C.c_int64(), C.c_int64(), C.c_int64(), C.c_double()
        check(lib().dmrg_zheff_sizes(h, C.byref(a), C.byref(b), C.byref(c), C.byref(f)), "dmrg_zheff_sizes")
        self.psi_dim, self.l_size, self.r_size, self.flops = a.value, b.value, c.value, f.value

    def set_env(self, L_dev: "DeviceArray", R_dev: "DeviceArray") -> None:
        self._env_refs = (L_dev, R_dev)
        check(lib().dmrg_zheff_set_env(self.h, L_dev.ptr, R_dev.ptr), "dmrg_zheff_set_env")

    def apply(self, psi: "DeviceArray", out: "DeviceArray", accumulate: bool = False) -> None:
        check(lib().dmrg_zheff_apply(self.h, psi.ptr, out.ptr, int(accumulate)), "dmrg_zheff_apply")

    def lanczos(self, psi: "DeviceArray", niter: int, precision: float = 1e-15, zero_tol: float = 1e-15):
        e, it = C.c_double(), C.c_int()
        check(lib().dmrg_zlanczos(self.h, psi.ptr, niter, precision, zero_tol, C.byref(e), C.byref(it)),
              "dmrg_zlanczos")
        return e.value, it.value

    def close(self) -> None:
        if self.h:
            lib().dmrg_zheff_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Env:
    """Environment update (Left/RightComputeTensorContraction)."""

    def __init__(self, ctx: Context, side: int, site: SiteProblem, env_in: Sequence[BlockSpec],
                 precision: int = DMRG_PREC_FP64, Wc: np.ndarray | None = None):
        """Wc: a complex MPO ([lb][rb][d][d] complex128) for the complex update
        (dmrg_zenv_create; ket and environments then hold interleaved complex)."""
        self.ctx, self.site, self.side = ctx, site, side
        self._in = _blocks_array(env_in)
        self.complex = Wc is not None
        kb = site.ket.c()
        h = _VP()
        if self.complex:
            self._W = np.ascontiguousarray(np.asarray(Wc, dtype=np.complex128)).view(np.float64)
            check(lib().dmrg_zenv_create(ctx.h, side, site.nl, site.nr, _iptr(site.phys), C.byref(kb), site.d,
                                         site.lb, site.rb, _dptr(self._W), self._in, C.byref(h)), "dmrg_zenv_create")
        else:
            check(lib().dmrg_env_create(ctx.h, side, site.nl, site.nr, _iptr(site.phys), C.byref(kb), site.d,
                                        site.lb, site.rb, _dptr(site.W), self._in, precision, C.byref(h)),
                  "dmrg_env_create")
        self.h = h
        bond, size = C.c_int(), C.c_int64()
        check(lib().dmrg_env_out_info(h, C.byref(bond), C.byref(size)), "dmrg_env_out_info")
        self.out_bond, self.out_size = bond.value, size.value

    def out_blocks(self) -> list[BlockSpec]:
        res = []
        for o in range(self.out_bond):
            n = C.c_int()
            check(lib().dmrg_env_out_blocks(self.h, o, 0, C.byref(n), None, None, None, None), "env_out_blocks")
            arrs = [np.zeros(max(n.value, 1), dtype=np.int32) for _ in range(4)]
            check(lib().dmrg_env_out_blocks(self.h, o, max(n.value, 1), C.byref(n), *[_iptr(a) for a in arrs]),
                  "env_out_blocks")
            res.append(BlockSpec(*[a[:n.value] for a in arrs]))
        return res

    def flops(self) -> tuple[float, float]:
        a, e = C.c_double(), C.c_double()
        check(lib().dmrg_env_flops(self.h, C.byref(a), C.byref(e)), "dmrg_env_flops")
        return a.value, e.value

    def apply(self, ket: DeviceArray, env_in: DeviceArray, env_out: DeviceArray) -> None:
        if self.complex:
            check(lib().dmrg_zenv_apply(self.h, ket.ptr, env_in.ptr, env_out.ptr), "dmrg_zenv_apply")
        else:
            check(lib().dmrg_env_apply(self.h, ket.ptr, env_in.ptr, env_out.ptr), "dmrg_env_apply")

    def close(self) -> None:
        if self.h:
            lib().dmrg_env_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Canonical:
    """Per-sector SVD canonicalisation (Left/RightCanonicalTensorLattice); with
    complex=True the complex twin (dmrg_zcanon_*: interleaved complex ket)."""

    def __init__(self, ctx: Context, side: int, left_dim, right_dim, ket: BlockSpec, complex: bool = False):
        self.ctx, self.side, self.ket = ctx, side, ket
        self._p = "dmrg_zcanon_" if complex else "dmrg_canon_"
        self.left_dim = np.ascontiguousarray(left_dim, dtype=np.int32)
        self.right_dim = np.ascontiguousarray(right_dim, dtype=np.int32)
        kb = ket.c()
        h = _VP()
        check(self._f("create")(ctx.h, side, len(self.left_dim), len(self.right_dim), _iptr(self.left_dim),
                                _iptr(self.right_dim), C.byref(kb), C.byref(h)), self._p + "create")
        self.h = h
        self.nsec = len(self.right_dim) if side == 0 else len(self.left_dim)

    def _f(self, name: str):
        return getattr(lib(), self._p + name)

    def run(self, ket_dev: DeviceArray, max_dim: int, canpre: float):
        t = np.zeros(self.nsec, dtype=np.int32)
        d = C.c_double()
        check(self._f("run")(self.h, ket_dev.ptr, max_dim, canpre, _iptr(t), C.byref(d)), self._p + "run")
        ks, cs, sw = C.c_int64(), C.c_int64(), C.c_int()
        check(self._f("out_info")(self.h, C.byref(ks), C.byref(cs), C.byref(sw)), self._p + "out_info")
        n = len(self.ket.left)
        kr, kc = np.zeros(max(n, 1), np.int32), np.zeros(max(n, 1), np.int32)
        cr, cc, md = (np.zeros(self.nsec, np.int32) for _ in range(3))
        check(self._f("out_blocks")(self.h, _iptr(kr), _iptr(kc), _iptr(cr), _iptr(cc), _iptr(md)),
              self._p + "out_blocks")
        return {"tdim": t, "discarded": d.value, "ket_size": ks.value, "canonical_size": cs.value,
                "sweeps": sw.value, "ket_rows": kr[:n], "ket_cols": kc[:n], "canon_rows": cr, "canon_cols": cc,
                "match_dim": md}

    def singular_values(self, sector: int) -> np.ndarray:
        n = C.c_int()
        check(self._f("singular_values")(self.h, sector, 0, None, C.byref(n)), "singular_values")
        out = np.zeros(max(n.value, 1))
        check(self._f("singular_values")(self.h, sector, n.value, _dptr(out), C.byref(n)), "singular_values")
        return out[:n.value]

    def write(self, ket_dev: DeviceArray, new_ket: DeviceArray, canonical: DeviceArray) -> None:
        check(self._f("write")(self.h, ket_dev.ptr, new_ket.ptr, canonical.ptr), self._p + "write")

    def close(self) -> None:
        if self.h:
            self._f("destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def quicksort_index(values, descending: bool = True):
    """The reference's QuickSort with index, run by the library's host code."""
    v = np.ascontiguousarray(values, dtype=np.float64).copy()
    idx = np.arange(len(v), dtype=np.int32)
    check(lib().dmrg_quicksort_index(_dptr(v), _iptr(idx), len(v), int(descending)), "dmrg_quicksort_index")
    return v, idx


def truncate_dims(svals, max_dim: int, canpre: float):
    """ComputeTruncateDim through the library (host bookkeeping)."""
    counts = np.array([len(s) for s in svals], dtype=np.int32)
    flat = np.ascontiguousarray(np.concatenate([np.asarray(s, dtype=np.float64) for s in svals])
                                if len(svals) else np.zeros(0))
    t = np.zeros(max(len(svals), 1), dtype=np.int32)
    check(lib().dmrg_truncate_dims(len(svals), _iptr(counts), _dptr(flat), max_dim, canpre, _iptr(t)),
          "dmrg_truncate_dims")
    out, pos = [], 0
    for c in counts:
        out.append(flat[pos:pos + c].copy())
        pos += c
    return t[:len(svals)], out


def svd_plan_rounds(cols: int, bm, tol: float):
    """The Jacobi sweep's rounds for one sector (host data; no GPU needed):
    a list of rounds, each a list of (bi, bj) block pairs."""
    bm = np.ascontiguousarray(bm, dtype=np.float64)
    cap = 4096
    out = np.zeros(cap, dtype=np.int32)
    n_pairs, n_rounds = C.c_int(), C.c_int()
    check(lib().dmrg_svd_plan_rounds(cols, _dptr(bm), tol, cap, _iptr(out), C.byref(n_pairs), C.byref(n_rounds)),
          "dmrg_svd_plan_rounds")
    rounds = [[] for _ in range(n_rounds.value)]
    for v in out[:n_pairs.value]:
        rounds[int(v) >> 16].append(((int(v) >> 8) & 255, int(v) & 255))
    return rounds


def svd_pair_schedule() -> np.ndarray:
    """The Jacobi pair solve's rotation schedule, [63 steps, 32 lanes] of
    a | b << 6 | flip << 12 | seat lane << 13 | seat flip << 18 (host data; no
    GPU needed)."""
    out = np.zeros(63 * 32, dtype=np.uint32)
    check(lib().dmrg_svd_pair_schedule(out.ctypes.data_as(C.POINTER(C.c_uint))), "dmrg_svd_pair_schedule")
    return out.reshape(63, 32)


class RunOptions(C.Structure):
    """dmrg_run_options_t."""

    _fields_ = [("precision", C.c_int), ("verbose", C.c_int), ("seed", C.c_uint),
                ("stop_after_half_sweeps", C.c_int), ("lanczos_precision", C.c_double), ("two_site", C.c_int),
                ("lanczos_graph", C.c_int)]


def run_options_from_input(input_path: str) -> RunOptions:
    """The options an input file's optional keys ask for (precision, mode, seed,
    lanczos_tol, lanczos_graph); host only."""
    o = RunOptions()
    check(lib().dmrg_run_options_from_input(input_path.encode(), C.byref(o)), "dmrg_run_options_from_input")
    return o


class Run:
    """A whole DMRG run of a reference input file on the device (RealTensorRundmrg)."""

    def __init__(self, ctx: Context, input_path: str, model: str = "real_spinless_bose_square", verbose: int = 0,
                 seed: int = 1, stop_after_half_sweeps: int = -1, precision: int = DMRG_PREC_FP64,
                 two_site: bool = False, lanczos_graph: int = 0):
        self.ctx = ctx
        self._opt = RunOptions(precision, verbose, seed, stop_after_half_sweeps, 0.0, int(bool(two_site)),
                               int(lanczos_graph))
        h = _VP()
        check(lib().dmrg_run_create(ctx.h, input_path.encode(), model.encode(), C.byref(self._opt), C.byref(h)),
              "dmrg_run_create")
        self.h = h

    def execute(self) -> None:
        check(lib().dmrg_run_execute(self.h), "dmrg_run_execute")

    def half_sweeps(self):
        n = C.c_int()
        check(lib().dmrg_run_half_sweeps(self.h, 0, None, None, C.byref(n)), "dmrg_run_half_sweeps")
        e, s = np.zeros(max(n.value, 1)), np.zeros(max(n.value, 1))
        check(lib().dmrg_run_half_sweeps(self.h, n.value, _dptr(e), _dptr(s), C.byref(n)), "dmrg_run_half_sweeps")
        return e[:n.value], s[:n.value]

    @staticmethod
    def execute_many(runs: Sequence["Run"], threads: int = 0) -> np.ndarray:
        """Executes independent runs side by side (each on its own context's
        stream, `threads` host threads); returns the per-run status codes."""
        arr = (_VP * max(len(runs), 1))(*[r.h for r in runs])
        status = np.zeros(max(len(runs), 1), np.int32)
        check(lib().dmrg_run_execute_many(arr, len(runs), threads, _iptr(status)), "dmrg_run_execute_many")
        return status[:len(runs)]

    PHASES = ("lanczos", "expansion", "canonicalisation", "environment", "match_merge")

    def phases(self):
        """(seconds[half_sweep, phase] in PHASES order, Jacobi SVD sweeps per half-sweep)."""
        n = C.c_int()
        check(lib().dmrg_run_phases(self.h, 0, None, None, C.byref(n)), "dmrg_run_phases")
        k = max(n.value, 1)
        sec = np.zeros((k, len(self.PHASES)))
        sw = np.zeros(k, np.int32)
        check(lib().dmrg_run_phases(self.h, n.value, _dptr(sec), _iptr(sw), C.byref(n)), "dmrg_run_phases")
        return sec[:n.value], sw[:n.value]

    def steps(self) -> dict:
        n = C.c_int()
        check(lib().dmrg_run_steps(self.h, 0, None, None, None, None, None, None, None, C.byref(n)), "dmrg_run_steps")
        k = max(n.value, 1)
        hs, st, dims = (np.zeros(k, np.int32) for _ in range(3))
        en, dis, sec = (np.zeros(k) for _ in range(3))
        psi = np.zeros(k, np.int64)
        check(lib().dmrg_run_steps(self.h, n.value, _iptr(hs), _iptr(st), _dptr(en), _iptr(dims), _dptr(dis),
                                   psi.ctypes.data_as(_I64), _dptr(sec), C.byref(n)), "dmrg_run_steps")
        m = n.value
        return {"half_sweep": hs[:m], "site": st[:m], "energy": en[:m], "lanczos_dim": dims[:m],
                "discarded": dis[:m], "psi_dim": psi[:m], "seconds": sec[:m]}

    def log_records(self) -> list[dict]:
        """The run as log records: one per site step ("step": half-sweep, site,
        Lanczos energy and Krylov dimension, discarded weight of the truncation,
        psi_dim, seconds), then one per half-sweep ("half_sweep": its energy,
        the reference's "right/left energy =", seconds, per-phase seconds,
        Jacobi SVD sweeps).  The reference prints only the energies."""
        return run_log_records(self.steps(), *self.half_sweeps(), *self.phases())

    def write_log(self, path: str) -> None:
        """The records of log_records() as JSON lines."""
        import json

        with open(path, "w") as f:
            for r in self.log_records():
                f.write(json.dumps(r) + "\n")

    def close(self) -> None:
        if self.h:
            lib().dmrg_run_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def run_log_records(steps: dict, energies, seconds, phase_seconds, svd_sweeps) -> list[dict]:
    """Log records of a run from its step records (Run.steps()), half-sweep
    energies and times (Run.half_sweeps()) and phases (Run.phases())."""
    out = []
    for k in range(len(steps["site"])):
        out.append({"record": "step", "half_sweep": int(steps["half_sweep"][k]), "site": int(steps["site"][k]),
                    "energy": float(steps["energy"][k]), "lanczos_dim": int(steps["lanczos_dim"][k]),
                    "discarded": float(steps["discarded"][k]), "psi_dim": int(steps["psi_dim"][k]),
                    "seconds": float(steps["seconds"][k])})
    for h in range(len(energies)):
        rec = {"record": "half_sweep", "half_sweep": h, "direction": "right" if h % 2 == 0 else "left",
               "energy": float(energies[h]), "seconds": float(seconds[h])}
        if h < len(phase_seconds):
            rec["phase_seconds"] = {name: float(v) for name, v in zip(Run.PHASES, phase_seconds[h])}
            rec["svd_sweeps"] = int(svd_sweeps[h])
        out.append(rec)
    return out


class Model:
    """The model layer (MPO and quantum tables) of an input file; host only."""

    def __init__(self, input_path: str, model: str = "real_spinless_bose_square"):
        h = _VP()
        check(lib().dmrg_model_create(input_path.encode(), model.encode(), C.byref(h)), "dmrg_model_create")
        self.h = h
        a, b, c = C.c_int(), C.c_int(), C.c_int()
        check(lib().dmrg_model_info(h, C.byref(a), C.byref(b), C.byref(c)), "dmrg_model_info")
        self.num_site, self.physics_dim, self.num_quantum = a.value, b.value, c.value
        z = C.c_int()
        check(lib().dmrg_model_is_complex(h, C.byref(z)), "dmrg_model_is_complex")
        self.is_complex = bool(z.value)

    def mpo(self, site: int) -> np.ndarray:
        """W[l][r][p1][p2] (complex128 for a complex model)."""
        lb, rb = C.c_int(), C.c_int()
        check(lib().dmrg_model_mpo(self.h, site, C.byref(lb), C.byref(rb), 0, None), "dmrg_model_mpo")
        d = self.physics_dim
        w = np.zeros(lb.value * rb.value * d * d * (2 if self.is_complex else 1))
        check(lib().dmrg_model_mpo(self.h, site, C.byref(lb), C.byref(rb), w.size, _dptr(w)), "dmrg_model_mpo")
        if self.is_complex:
            w = w.view(np.complex128)
        return w.reshape(lb.value, rb.value, d, d)

    def quantum_table(self, which: int, bond: int) -> np.ndarray:
        rows = C.c_int()
        check(lib().dmrg_model_quantum_table(self.h, which, bond, 0, None, C.byref(rows)), "quantum_table")
        v = np.zeros(max(rows.value * self.num_quantum, 1), np.int32)
        check(lib().dmrg_model_quantum_table(self.h, which, bond, v.size, _iptr(v), C.byref(rows)), "quantum_table")
        return v[:rows.value * self.num_quantum].reshape(rows.value, self.num_quantum)

    def close(self) -> None:
        if self.h:
            lib().dmrg_model_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
