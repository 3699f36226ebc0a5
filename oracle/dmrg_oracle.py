"""CPU oracle: a numpy restatement of the reference's DMRG hot path.

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the CPU
baseline legs of bench.py may import this module, and only as the checker.
The product path (dmrgcc_b200) never calls into oracle/.

Each function follows one reference routine (jiandong94/dmrgcc, real FP64 twin)
loop for loop, so that the order of block visits, the zero tests on the MPO and
the block-list orders it produces are the reference's.  Dense GEMMs go through
numpy (BLAS); floating-point results therefore agree with the reference to
rounding, while every integer/bookkeeping output (block lists, truncation
dimensions, sort order) is exact.

The restatement is pinned against outputs of the reference itself, built from
its own sources by oracle/Makefile and dumped by oracle/probe/probe_dump.cc
(fixtures under tests/golden/, test_oracle_pins.py).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

ZERO_TOL = 1e-15  # RealTensorOperator::*CheckZero threshold, real_tensor_operator.cc:363-409


# ----------------------------------------------------------------------------------
# Block lists (RealMatrixBlock, src/tensor/real_matrix_block.{h,cc})
# ----------------------------------------------------------------------------------
@dataclass
class BlockList:
    """Ordered list of (left_index, right_index, dense matrix)."""

    left: list = field(default_factory=list)
    right: list = field(default_factory=list)
    mats: list = field(default_factory=list)

    def __len__(self) -> int:
        return len(self.left)

    def find(self, l: int, r: int) -> int:
        """FindMatrixBlock(left, right): first match by linear scan (real_matrix_block.cc:314)."""
        for i in range(len(self.left)):
            if self.left[i] == l and self.right[i] == r:
                return i
        return -1

    def same_index(self, leigh: int, target: int) -> list:
        """FindMatrixBlock(num, pos, leigh, target): positions in list order (:332)."""
        idx = self.left if leigh == 0 else self.right
        return [i for i in range(len(idx)) if idx[i] == target]

    def offsets(self) -> list:
        """ComputePartMatrixBlockDim for every position (:154)."""
        off, acc = [], 0
        for m in self.mats:
            off.append(acc)
            acc += m.size
        return off

    def vectorize(self) -> np.ndarray:
        """VectorizeMatrixBlock(true, state) (:173)."""
        if not self.mats:
            return np.zeros(0)
        return np.concatenate([m.ravel() for m in self.mats])

    def unvectorize(self, v: np.ndarray) -> None:
        """VectorizeMatrixBlock(false, state)."""
        pos = 0
        for i, m in enumerate(self.mats):
            n = m.size
            self.mats[i] = v[pos:pos + n].reshape(m.shape).copy()
            pos += n

    def copy(self) -> "BlockList":
        return BlockList(list(self.left), list(self.right), [m.copy() for m in self.mats])


@dataclass
class Lattice:
    """RealTensorLattice (real_tensor_lattice.h:10-42)."""

    physics_dim: int
    left_block: list
    left_dim: list
    right_block: list
    right_dim: list
    physics_index: np.ndarray  # [num_left_block, num_right_block], -1 where no block
    ket: BlockList
    canonical: BlockList | None = None
    match_dim: list | None = None

    def psi_dim(self) -> int:
        return int(sum(m.size for m in self.ket.mats))


def _blocklist_from_nac(d: dict, p: str) -> BlockList:
    left = [int(x) for x in d[p + ".left"]]
    right = [int(x) for x in d[p + ".right"]]
    rows = [int(x) for x in d[p + ".rows"]]
    cols = [int(x) for x in d[p + ".cols"]]
    data = d.get(p + ".data")
    mats, pos = [], 0
    for r, c in zip(rows, cols):
        if data is None:
            mats.append(np.zeros((r, c)))
        else:
            mats.append(np.asarray(data[pos:pos + r * c], dtype=np.float64).reshape(r, c).copy())
        pos += r * c
    return BlockList(left, right, mats)


def lattice_from_nac(d: dict, p: str) -> Lattice:
    nl = len(d[p + ".left_dim"])
    nr = len(d[p + ".right_dim"])
    lat = Lattice(
        physics_dim=int(d[p + ".physics_dim"][0]) if (p + ".physics_dim") in d else 0,
        left_block=[int(x) for x in d.get(p + ".left_block", np.arange(nl))],
        left_dim=[int(x) for x in d[p + ".left_dim"]],
        right_block=[int(x) for x in d.get(p + ".right_block", np.arange(nr))],
        right_dim=[int(x) for x in d[p + ".right_dim"]],
        physics_index=np.asarray(d[p + ".physics_index"], dtype=np.int64).reshape(nl, nr),
        ket=_blocklist_from_nac(d, p + ".ket"),
    )
    if (p + ".canonical.left") in d:
        lat.canonical = _blocklist_from_nac(d, p + ".canonical")
        lat.match_dim = [int(x) for x in d[p + ".match_dim"]]
    return lat


def operator_from_nac(d: dict, p: str) -> np.ndarray:
    dd, lb, rb = (int(x) for x in d[p + ".dims"])
    return np.asarray(d[p + ".W"], dtype=np.float64).reshape(lb, rb, dd, dd).copy()


def env_from_nac(d: dict, p: str) -> list:
    bond = int(d[p + ".bond"][0])
    return [_blocklist_from_nac(d, f"{p}.{o}") for o in range(bond)]


# ----------------------------------------------------------------------------------
# MPO zero tests (RealTensorOperator, real_tensor_operator.cc:363-409)
# ----------------------------------------------------------------------------------
def left_check_zero(W: np.ndarray, l: int, p1: int) -> bool:
    """True when row (l, p1) of W holds an element above 1e-15 (LeftCheckZero)."""
    return bool(np.any(np.abs(W[l, :, p1, :]) > ZERO_TOL))


def right_check_zero(W: np.ndarray, r: int, p2: int) -> bool:
    """RightCheckZero(r, p2)."""
    return bool(np.any(np.abs(W[:, r, :, p2]) > ZERO_TOL))


def mixed_check_zero(W: np.ndarray, l: int, p2: int) -> bool:
    """MixedCheckZero(l, p2)."""
    return bool(np.any(np.abs(W[l, :, :, p2]) > ZERO_TOL))


# ----------------------------------------------------------------------------------
# a1: H_eff * psi  (RealTensorContraction::MultiplyEffectHamilton,
#                   src/dmrg/realdmrg/real_tensor_contraction.cc:1223-1291)
# ----------------------------------------------------------------------------------
def multiply_effect_hamilton(lat: Lattice, W: np.ndarray, L: list, R: list, state: np.ndarray) -> None:
    """Adds H_eff * ket into `state` (flat, ket block order), like the reference."""
    ket = lat.ket
    lb, rb = W.shape[0], W.shape[1]
    nr = len(lat.right_dim)
    same = [ket.same_index(1, r) for r in range(nr)]
    off = ket.offsets()
    for o2 in range(rb):
        Ro = R[o2]
        for i in range(len(Ro)):
            ldx, jdx = Ro.left[i], Ro.right[i]
            Rm = Ro.mats[i]
            if Rm.shape[0] == 0:
                continue
            for pos in same[ldx]:
                kdx = ket.left[pos]
                p2 = int(lat.physics_index[kdx, ldx])
                if not right_check_zero(W, o2, p2):
                    continue
                first = ket.mats[pos] @ Rm
                for pos2 in same[jdx]:
                    idx = ket.left[pos2]
                    p1 = int(lat.physics_index[idx, jdx])
                    for o1 in range(lb):
                        w = W[o1, o2, p1, p2]
                        if w != 0.0:
                            q = L[o1].find(idx, kdx)
                            if q != -1:
                                second = (L[o1].mats[q] @ first) * w
                                state[off[pos2]:off[pos2] + second.size] += second.ravel()


def heff_flops(lat: Lattice, W: np.ndarray, L: list, R: list) -> tuple[int, int]:
    """Algorithmic FLOPs of one H_eff*psi, counted over the reference loop above.

    Returns (flops of the K*R products, flops of the L*(KR) products)."""
    ket = lat.ket
    lb, rb = W.shape[0], W.shape[1]
    nr = len(lat.right_dim)
    same = [ket.same_index(1, r) for r in range(nr)]
    fa = fb = 0
    for o2 in range(rb):
        Ro = R[o2]
        for i in range(len(Ro)):
            ldx, jdx = Ro.left[i], Ro.right[i]
            Rm = Ro.mats[i]
            if Rm.shape[0] == 0:
                continue
            for pos in same[ldx]:
                kdx = ket.left[pos]
                p2 = int(lat.physics_index[kdx, ldx])
                if not right_check_zero(W, o2, p2):
                    continue
                a_k, b_l = ket.mats[pos].shape
                b_j = Rm.shape[1]
                fa += 2 * a_k * b_l * b_j
                for pos2 in same[jdx]:
                    idx = ket.left[pos2]
                    p1 = int(lat.physics_index[idx, jdx])
                    for o1 in range(lb):
                        if W[o1, o2, p1, p2] != 0.0:
                            q = L[o1].find(idx, kdx)
                            if q != -1:
                                a_i = L[o1].mats[q].shape[0]
                                fb += 2 * a_i * a_k * b_j
    return fa, fb


# ----------------------------------------------------------------------------------
# a5: dense H_eff (ComputeEffectHamilton, real_tensor_contraction.cc:1136-1205)
# ----------------------------------------------------------------------------------
def compute_effect_hamilton(lat: Lattice, W: np.ndarray, L: list, R: list) -> np.ndarray:
    ket = lat.ket
    n = lat.psi_dim()
    H = np.zeros((n, n))
    off = ket.offsets()
    lb, rb = W.shape[0], W.shape[1]
    for o1 in range(lb):
        Lo = L[o1]
        for i in range(len(Lo)):
            idx, kdx = Lo.left[i], Lo.right[i]
            Lm = Lo.mats[i]
            if Lm.shape[0] == 0:
                continue
            for o2 in range(rb):
                Ro = R[o2]
                for j in range(len(Ro)):
                    ldx, jdx = Ro.left[j], Ro.right[j]
                    Rm = Ro.mats[j]
                    if Rm.shape[0] == 0:
                        continue
                    p0 = ket.find(idx, jdx)
                    p1_ = ket.find(kdx, ldx)
                    if p0 != -1 and p1_ != -1:
                        p1 = int(lat.physics_index[idx, jdx])
                        p2 = int(lat.physics_index[kdx, ldx])
                        w = W[o1, o2, p1, p2]
                        if w != 0:
                            kr = np.kron(Lm, Rm.T) * w
                            if kr.size == 0:
                                continue
                            a, b = off[p0], off[p1_]
                            H[a:a + kr.shape[0], b:b + kr.shape[1]] += kr
    return H


# ----------------------------------------------------------------------------------
# a2/a3: environment updates (real_tensor_contraction.cc:782-940, 959-1119)
# ----------------------------------------------------------------------------------
def _add_to(mats: list, pos: int, w: float, M: np.ndarray) -> None:
    """RealMatrix::AddToMatrix(factor, m) (real_matrix.cc:252-281)."""
    if M.size == 0:
        return
    if mats[pos].size == 0:
        mats[pos] = w * M
    else:
        mats[pos] = mats[pos] + w * M


def left_compute_env(lat: Lattice, W: np.ndarray, Lin: list) -> list:
    """Returns the next left environment: one BlockList per right MPO bond index."""
    ket = lat.ket
    lb, rb = W.shape[0], W.shape[1]
    nl, nr = len(lat.left_dim), len(lat.right_dim)
    same = [ket.same_index(0, l) for l in range(nl)]
    flag = np.zeros((rb, nr, nr), dtype=bool)
    for o1 in range(lb):
        Lo = Lin[o1]
        for i in range(len(Lo)):
            kdx, ldx = Lo.left[i], Lo.right[i]
            if Lo.mats[i].shape[0] == 0:
                continue
            for pk in same[kdx]:
                idx = ket.right[pk]
                p1 = int(lat.physics_index[kdx, idx])
                if not left_check_zero(W, o1, p1):
                    continue
                for pl in same[ldx]:
                    jdx = ket.right[pl]
                    p2 = int(lat.physics_index[ldx, jdx])
                    for o2 in range(rb):
                        if W[o1, o2, p1, p2] != 0.0:
                            flag[o2, idx, jdx] = True
    out = []
    for o2 in range(rb):
        li, ri = np.nonzero(flag[o2])  # row-major order == the reference's i-then-j loop
        out.append(BlockList([int(x) for x in li], [int(x) for x in ri], [np.zeros((0, 0)) for _ in li]))
    for o1 in range(lb):
        Lo = Lin[o1]
        for i in range(len(Lo)):
            kdx, ldx = Lo.left[i], Lo.right[i]
            Lm = Lo.mats[i]
            if Lm.shape[0] == 0:
                continue
            for pk in same[kdx]:
                idx = ket.right[pk]
                p1 = int(lat.physics_index[kdx, idx])
                if not left_check_zero(W, o1, p1):
                    continue
                first = ket.mats[pk].T @ Lm
                for pl in same[ldx]:
                    jdx = ket.right[pl]
                    p2 = int(lat.physics_index[ldx, jdx])
                    second = first @ ket.mats[pl]
                    for o2 in range(rb):
                        w = W[o1, o2, p1, p2]
                        if w != 0.0:
                            q = out[o2].find(idx, jdx)
                            _add_to(out[o2].mats, q, w, second)
    return out


def right_compute_env(lat: Lattice, W: np.ndarray, Rin: list) -> list:
    """Returns the next right environment: one BlockList per left MPO bond index."""
    ket = lat.ket
    lb, rb = W.shape[0], W.shape[1]
    nl, nr = len(lat.left_dim), len(lat.right_dim)
    same = [ket.same_index(1, r) for r in range(nr)]
    flag = np.zeros((lb, nl, nl), dtype=bool)
    for o2 in range(rb):
        Ro = Rin[o2]
        for i in range(len(Ro)):
            ldx, kdx = Ro.left[i], Ro.right[i]
            if Ro.mats[i].shape[0] == 0:
                continue
            for pl in same[ldx]:
                jdx = ket.left[pl]
                p2 = int(lat.physics_index[jdx, ldx])
                if not right_check_zero(W, o2, p2):
                    continue
                for pk in same[kdx]:
                    idx = ket.left[pk]
                    p1 = int(lat.physics_index[idx, kdx])
                    for o1 in range(lb):
                        if W[o1, o2, p1, p2] != 0.0:
                            flag[o1, jdx, idx] = True
    out = []
    for o1 in range(lb):
        ji, ii = np.nonzero(flag[o1])
        out.append(BlockList([int(x) for x in ji], [int(x) for x in ii], [np.zeros((0, 0)) for _ in ji]))
    for o2 in range(rb):
        Ro = Rin[o2]
        for i in range(len(Ro)):
            ldx, kdx = Ro.left[i], Ro.right[i]
            Rm = Ro.mats[i]
            if Rm.shape[0] == 0:
                continue
            for pl in same[ldx]:
                jdx = ket.left[pl]
                p2 = int(lat.physics_index[jdx, ldx])
                if not right_check_zero(W, o2, p2):
                    continue
                first = ket.mats[pl] @ Rm
                for pk in same[kdx]:
                    idx = ket.left[pk]
                    p1 = int(lat.physics_index[idx, kdx])
                    second = first @ ket.mats[pk].T
                    for o1 in range(lb):
                        w = W[o1, o2, p1, p2]
                        if w != 0.0:
                            q = out[o1].find(jdx, idx)
                            _add_to(out[o1].mats, q, w, second)
    return out


# ----------------------------------------------------------------------------------
# a7: truncation (ComputeTruncateDim real_tensor_lattice.cc:501-555,
#     QuickSort with index src/util/general.ih:7-65)
# ----------------------------------------------------------------------------------
def quicksort_with_index(a: list, index: list, descending: bool = True) -> None:
    """In-place port of the reference's non-stable quicksort (first element as pivot).

    The recursion is replaced by an explicit stack; the two sub-ranges are disjoint,
    so the order in which they are processed does not change the result."""
    stack = [(0, len(a) - 1)]
    while stack:
        left, right = stack.pop()
        if left >= right:
            continue
        i, j = left, right
        pv, pi = a[i], index[i]
        if descending:
            while i < j:
                while i < j and a[j] <= pv:
                    j -= 1
                if i < j:
                    a[i], index[i] = a[j], index[j]
                    i += 1
                while i < j and a[i] >= pv:
                    i += 1
                if i < j:
                    a[j], index[j] = a[i], index[i]
                    j -= 1
        else:
            while i < j:
                while i < j and a[j] >= pv:
                    j -= 1
                if i < j:
                    a[i], index[i] = a[j], index[j]
                    i += 1
                while i < j and a[i] <= pv:
                    i += 1
                if i < j:
                    a[j], index[j] = a[i], index[i]
                    j -= 1
        a[i], index[i] = pv, pi
        stack.append((left, i - 1))
        stack.append((i + 1, right))


def compute_truncate_dim(max_dim: int, canpre: float, svals: list) -> list:
    """svals: per-sector singular values (descending).  Mutates svals like the reference
    (a sector left with nothing keeps one value, forced to 0)."""
    if canpre > 1:
        canpre = 0.0
    tdim = [int(np.sum(np.asarray(s) > canpre)) for s in svals]
    total = sum(tdim)
    if total > 0 and max_dim > 0 and max_dim < total:
        vals, blk = [], []
        for i, s in enumerate(svals):
            for j in range(tdim[i]):
                vals.append(float(s[j]))
                blk.append(i)
        quicksort_with_index(vals, blk, descending=True)
        tdim = [0] * len(svals)
        for i in range(max_dim):
            tdim[blk[i]] += 1
    for i in range(len(svals)):
        if tdim[i] == 0:
            tdim[i] = 1
            svals[i][0] = 0.0
    return tdim


# ----------------------------------------------------------------------------------
# a6: canonicalisation by per-sector SVD (real_tensor_lattice.cc:558-676, 794-911)
# ----------------------------------------------------------------------------------
def left_canonical(lat: Lattice, max_dim: int, canpre: float) -> dict:
    """Left-canonicalises `lat` in place.  Returns per-sector singular values, the
    truncation dimensions and the discarded weight (sum of dropped sigma^2)."""
    ket = lat.ket
    nr = len(lat.right_dim)
    U, V, S = [None] * nr, [None] * nr, [None] * nr
    for r in range(nr):
        pos = ket.same_index(1, r)
        n = lat.right_dim[r]
        m = sum(ket.mats[p].shape[0] for p in pos)
        if m == 0:
            U[r] = None
            V[r] = np.zeros((n, n))
            S[r] = np.zeros(1)  # singular_dim = 1 with sigma_0 = 0 (real_tensor_lattice.cc:583-590)
        else:
            A = np.zeros((m, n))
            row = 0
            for p in pos:
                B = ket.mats[p]
                A[row:row + B.shape[0], :B.shape[1]] = B
                row += B.shape[0]
            u, s, vt = np.linalg.svd(A, full_matrices=False)
            U[r], S[r] = u, s.copy()
            V[r] = np.zeros((n, n))
            V[r][:vt.shape[0], :] = vt
    svals_full = [s.copy() for s in S]
    tdim = compute_truncate_dim(max_dim, canpre, S)
    lat.canonical = BlockList(list(range(nr)), list(range(nr)), [None] * nr)
    lat.match_dim = [0] * nr
    for r in range(nr):
        if U[r] is not None:
            row = 0
            for p in ket.same_index(1, r):
                rows = ket.mats[p].shape[0]
                ket.mats[p] = U[r][row:row + rows, :tdim[r]].copy()
                row += rows
        lat.right_dim[r] = tdim[r]
        n = V[r].shape[1]
        lat.match_dim[r] = n
        lat.canonical.mats[r] = S[r][:tdim[r], None] * V[r][:tdim[r], :]
    return {"svals": svals_full, "tdim": tdim, "discarded": _discarded(svals_full, tdim)}


def right_canonical(lat: Lattice, max_dim: int, canpre: float) -> dict:
    ket = lat.ket
    nl = len(lat.left_dim)
    U, V, S = [None] * nl, [None] * nl, [None] * nl
    for l in range(nl):
        pos = ket.same_index(0, l)
        m = lat.left_dim[l]
        n = sum(ket.mats[p].shape[1] for p in pos)
        if n == 0:
            U[l] = np.zeros((m, m))
            V[l] = None
            S[l] = np.zeros(1)  # singular_dim = 1 with sigma_0 = 0 (real_tensor_lattice.cc:818-825)
        else:
            A = np.zeros((m, n))
            col = 0
            for p in pos:
                B = ket.mats[p]
                A[:B.shape[0], col:col + B.shape[1]] = B
                col += B.shape[1]
            u, s, vt = np.linalg.svd(A, full_matrices=False)
            U[l] = np.zeros((m, u.shape[1]))
            U[l][:, :] = u
            V[l], S[l] = vt, s.copy()
    svals_full = [s.copy() for s in S]
    tdim = compute_truncate_dim(max_dim, canpre, S)
    lat.canonical = BlockList(list(range(nl)), list(range(nl)), [None] * nl)
    lat.match_dim = [0] * nl
    for l in range(nl):
        if V[l] is not None:
            col = 0
            for p in ket.same_index(0, l):
                cols = ket.mats[p].shape[1]
                ket.mats[p] = V[l][:tdim[l], col:col + cols].copy()
                col += cols
        lat.left_dim[l] = tdim[l]
        m = U[l].shape[0]
        lat.match_dim[l] = m
        Ul = np.zeros((m, tdim[l]))
        k = min(tdim[l], U[l].shape[1])
        Ul[:, :k] = U[l][:, :k]
        lat.canonical.mats[l] = Ul * S[l][None, :tdim[l]]
    return {"svals": svals_full, "tdim": tdim, "discarded": _discarded(svals_full, tdim)}


def merge_lattice(lat: Lattice, source: Lattice, side: int) -> Lattice:
    """Left/RightMergeTensorLattice (real_tensor_lattice.cc:914-977): every ket
    block of `lat` whose left (side 0) / right (side 1) sector is s is replaced
    by canonical[s] @ block (side 0) or block @ canonical[s] (side 1), with
    canonical the per-sector blocks of `source`; that sector's dimension becomes
    the canonical block's rows (cols); then NormalizeTensorLattice
    (:491-494 -> real_matrix_block.cc:164-171) scales the whole ket by
    sqrt(1 / sum of squares)."""
    C = source.canonical.mats
    mats = [m.copy() for m in lat.ket.mats]
    left_dim, right_dim = list(lat.left_dim), list(lat.right_dim)
    if side == 0:
        for sec in range(len(left_dim)):
            for k, li in enumerate(lat.ket.left):
                if li == sec:
                    mats[k] = C[sec] @ mats[k]
            left_dim[sec] = C[sec].shape[0]
    else:
        for sec in range(len(right_dim)):
            for k, ri in enumerate(lat.ket.right):
                if ri == sec:
                    mats[k] = mats[k] @ C[sec]
            right_dim[sec] = C[sec].shape[1]
    total = 0.0
    for m in mats:
        total += float(np.sum(m * m))
    f = np.sqrt(1.0 / total)
    out = Lattice(physics_dim=lat.physics_dim, left_block=list(lat.left_block), left_dim=left_dim,
                  right_block=list(lat.right_block), right_dim=right_dim, physics_index=lat.physics_index.copy(),
                  ket=BlockList(list(lat.ket.left), list(lat.ket.right), [m * f for m in mats]))
    return out


def _discarded(svals: list, tdim: list) -> float:
    tot = 0.0
    for s, t in zip(svals, tdim):
        s = np.asarray(s)
        tot += float(np.sum(s[t:] ** 2))
    return tot


# ----------------------------------------------------------------------------------
# a4: Lanczos (RealTensorLanczos::LanczosMethod, real_tensor_lanczos.cc:14-201)
# ----------------------------------------------------------------------------------
def lanczos(lat: Lattice, W: np.ndarray, L: list, R: list, niter: int,
            precision: float = 1e-15, zero_tol: float = 1e-15) -> dict:
    """Runs the reference Lanczos on `lat` (its ket is the start vector and receives
    the ground vector).  Returns energy, iterations and the alpha/beta lists."""
    n = lat.psi_dim()
    if n < 100:
        H = compute_effect_hamilton(lat, W, L, R)
        w, v = np.linalg.eigh(H)
        lat.ket.unvectorize(v[:, 0].copy())
        return {"energy": float(w[0]), "iters": 0, "alpha": [], "beta": []}
    psi = [lat.ket.vectorize().copy()]
    h = np.zeros(n)
    alpha, beta = [], []
    old = 10000.0
    work = Lattice(lat.physics_dim, lat.left_block, lat.left_dim, lat.right_block, lat.right_dim,
                   lat.physics_index, lat.ket.copy())
    energy = None
    for i in range(niter):
        work.ket.unvectorize(psi[i])
        multiply_effect_hamilton(work, W, L, R, h)
        a = float(psi[i] @ h)
        h -= a * psi[i]
        b = float(np.sqrt(h @ h))
        alpha.append(a)
        beta.append(b)
        dim = i + 1
        T = np.diag(alpha) + np.diag(beta[:dim - 1], 1) + np.diag(beta[:dim - 1], -1)
        ev, evec = np.linalg.eigh(T)
        new = float(ev[0])
        if beta[i] < zero_tol or abs(new - old) < precision or dim == niter:
            energy = new
            vec = np.zeros(n)
            for k in range(dim):
                vec += psi[k] * evec[k, 0]
            lat.ket.unvectorize(vec)
            return {"energy": energy, "iters": dim, "alpha": alpha, "beta": beta}
        old = new
        nxt = h / beta[i]
        h = -beta[i] * psi[i]
        for k in range(dim):
            nxt -= (psi[k] @ nxt) * psi[k]
        nxt /= np.sqrt(nxt @ nxt)
        psi.append(nxt)
    return {"energy": energy, "iters": niter, "alpha": alpha, "beta": beta}


# ----------------------------------------------------------------------------------
# Seeded synthetic operands with a given block structure (bench / large parity cases)
# ----------------------------------------------------------------------------------
_SM_G = np.uint64(0x9E3779B97F4A7C15)
_SM_M1 = np.uint64(0xBF58476D1CE4E5B9)
_SM_M2 = np.uint64(0x94D049BB133111EB)


def splitmix_uniform(seed: int, start: int, count: int) -> np.ndarray:
    """Values `start .. start+count-1` of the splitmix64 stream mapped to [-1, 1)
    (identical to probe::SplitMix and to the library's generator)."""
    with np.errstate(over="ignore"):
        k = np.arange(start + 1, start + count + 1, dtype=np.uint64)
        z = np.uint64(seed) + k * _SM_G
        z = (z ^ (z >> np.uint64(30))) * _SM_M1
        z = (z ^ (z >> np.uint64(27))) * _SM_M2
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (2.0 / 9007199254740992.0) - 1.0
