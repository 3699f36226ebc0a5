"""Site problems: the block structure (and optionally the values) of one DMRG
site step, read from a .nac container, ready for the C ABI.

A .nac file is a sequence of named arrays:
    int32 name_len; bytes name; char dtype ('i' int32 | 'd' f64);
    int32 ndim; int32 shape[ndim]; little-endian data.
The arrays describe the site tensor ("lattice.*": sector dims, physics index
table, ket block list), the MPO tensor ("op.W", "op.dims") and the left/right
environments ("L.<o>.*", "R.<o>.*"), each block list as .left/.right/.rows/.cols
(+ .data when values are stored).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass

import numpy as np

from . import capi


def read_nac(path: str) -> dict[str, np.ndarray]:
    with open(path, "rb") as f:
        buf = f.read()
    out: dict[str, np.ndarray] = {}
    pos = 0
    while pos + 4 <= len(buf):
        (n,) = struct.unpack_from("<i", buf, pos)
        name = buf[pos + 4:pos + 4 + n].decode()
        pos += 4 + n
        dt = chr(buf[pos])
        (nd,) = struct.unpack_from("<i", buf, pos + 1)
        shape = struct.unpack_from("<%di" % nd, buf, pos + 5)
        pos += 5 + 4 * nd
        dtype = np.int32 if dt == "i" else np.float64
        count = int(np.prod(shape)) if nd else 1
        out[name] = np.frombuffer(buf, dtype=dtype, count=count, offset=pos).reshape(shape)
        pos += count * np.dtype(dtype).itemsize
    return out


def _spec(d: dict, p: str) -> capi.BlockSpec:
    return capi.BlockSpec(d[p + ".left"], d[p + ".right"], d[p + ".rows"], d[p + ".cols"])


@dataclass
class SiteStep:
    """One H_eff problem: site structure, MPO tensor and environment structure."""

    site: capi.SiteProblem
    L: list
    R: list
    ket_data: np.ndarray | None = None
    L_data: np.ndarray | None = None
    R_data: np.ndarray | None = None

    @classmethod
    def from_nac(cls, path: str) -> "SiteStep":
        d = read_nac(path)
        nl = len(d["lattice.left_dim"])
        nr = len(d["lattice.right_dim"])
        dd, lb, rb = (int(x) for x in d["op.dims"])
        W = np.asarray(d["op.W"]).reshape(lb, rb, dd, dd)
        if "lattice.block_phys" in d:  # a two-site tensor: one physics index per block
            site = capi.SiteProblem(nl, nr, None, _spec(d, "lattice.ket"), W, block_phys=d["lattice.block_phys"])
        else:
            site = capi.SiteProblem(nl, nr, d["lattice.physics_index"], _spec(d, "lattice.ket"), W)
        L = [_spec(d, f"L.{o}") for o in range(lb)]
        R = [_spec(d, f"R.{o}") for o in range(rb)]
        step = cls(site, L, R)
        if "lattice.ket.data" in d:
            step.ket_data = np.asarray(d["lattice.ket.data"], dtype=np.float64)
            step.L_data = np.concatenate([np.asarray(d[f"L.{o}.data"]) for o in range(lb)] or [np.zeros(0)])
            step.R_data = np.concatenate([np.asarray(d[f"R.{o}.data"]) for o in range(rb)] or [np.zeros(0)])
        return step

    @property
    def psi_dim(self) -> int:
        return self.site.ket.size

    @property
    def l_size(self) -> int:
        return sum(s.size for s in self.L)

    @property
    def r_size(self) -> int:
        return sum(s.size for s in self.R)

    def synthetic_device(self, ctx: capi.Context, seed: int):
        """Device arrays (psi, L, R) filled from the seeded splitmix64 stream: psi takes
        elements [0, psi_dim), L the next l_size, R the next r_size."""
        psi = capi.DeviceArray(ctx, self.psi_dim)
        L = capi.DeviceArray(ctx, self.l_size)
        R = capi.DeviceArray(ctx, self.r_size)
        psi.fill_uniform(seed, 0)
        L.fill_uniform(seed, self.psi_dim)
        R.fill_uniform(seed, self.psi_dim + self.l_size)
        return psi, L, R
