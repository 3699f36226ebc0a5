"""Reader for the reference's checkpoint file (cache_record / cache_resume).

TEST INFRASTRUCTURE ONLY: tests read checkpoint files with it to compare the
library's with the reference's.  It restates the reference's writers, field by
field, in their order:
  RealTensorSpace::WriteTensorSpace     src/dmrg/realdmrg/real_tensor_space.cc:182-208
  RealTensorLattice::WriteTensorLattice src/dmrg/realdmrg/real_tensor_lattice.cc:218-239
  RealMatrixBlock::WriteMatrixBlock     src/tensor/real_matrix_block.cc:227-240
  RealMatrix::WriteMatrix               src/tensor/real_matrix.cc:139-150
Native-endian int32 / float64, no padding.  Matrix elements are row-major
(real_matrix.cc:97, element (i, j) at i * column + j).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class Lattice:
    physics_dim: int
    left_block: list[int]
    left_dim: list[int]
    right_block: list[int]
    right_dim: list[int]
    physics_index: np.ndarray          # [num_left, num_right]
    blocks: list[tuple[int, int, np.ndarray]] = field(default_factory=list)  # (left, right, rows x cols)


@dataclass
class Space:
    num_site: int
    num_quantum: int
    quantum_table: list[np.ndarray]    # per bond 0..num_site: [num_table, num_quantum]
    lattices: list[Lattice]
    max_block: int
    max_dim: int
    canonical_precision: float
    noise_factor: float


class _Reader:
    def __init__(self, buf: bytes):
        self.buf, self.pos = buf, 0

    def ints(self, n: int) -> np.ndarray:
        a = np.frombuffer(self.buf, dtype=np.int32, count=n, offset=self.pos)
        self.pos += 4 * n
        return a.copy()

    def int(self) -> int:
        return int(self.ints(1)[0])

    def doubles(self, n: int) -> np.ndarray:
        a = np.frombuffer(self.buf, dtype=np.float64, count=n, offset=self.pos)
        self.pos += 8 * n
        return a.copy()


def read_space(path: str) -> Space:
    with open(path, "rb") as f:
        r = _Reader(f.read())
    num_site, num_site_pp, num_site_mm, num_quantum = r.ints(4)
    assert num_site_pp == num_site + 1 and num_site_mm == num_site - 1, "bad header"
    num_table = r.ints(num_site_pp)
    tables = [r.ints(int(t) * num_quantum).reshape(int(t), num_quantum) for t in num_table]
    lattices = []
    for _ in range(num_site):
        pd = r.int()
        nl = r.int()
        lb = r.ints(2 * nl).reshape(nl, 2) if nl else np.zeros((0, 2), np.int32)
        nr = r.int()
        rb = r.ints(2 * nr).reshape(nr, 2) if nr else np.zeros((0, 2), np.int32)
        phys = r.ints(nl * nr).reshape(nl, nr)
        lat = Lattice(pd, lb[:, 0].tolist(), lb[:, 1].tolist(), rb[:, 0].tolist(), rb[:, 1].tolist(), phys)
        for _ in range(r.int()):
            left, right, rows, cols, total = r.ints(5)
            assert rows * cols == total, "bad matrix header"
            lat.blocks.append((int(left), int(right), r.doubles(int(total)).reshape(int(rows), int(cols))))
        lattices.append(lat)
    max_block, max_dim = r.ints(2)
    canpre, noise = r.doubles(2)
    assert r.pos == len(r.buf), "trailing bytes"
    return Space(int(num_site), int(num_quantum), tables, lattices, int(max_block), int(max_dim), float(canpre),
                 float(noise))
