"""Exact diagonalisation of the spin-less Bose-Hubbard model in a fixed-N
sector (test infrastructure): an algorithm-independent check of DMRG energies
for small lattices.

Conventions follow the reference's MPO (model/hamiltonian/
real_spinless_bose_square_hamiltonian.cc): H = sum over bonds <p0,p1> of
J (b+_p0 b_p1 + b_p0 b+_p1) + sum_i [mu n_i + U n_i (n_i - 1)], J = Jx on
x-bonds and Jy on y-bonds, sites ordered p = j + i * Ny, periodic wraps only
for a dimension of more than two sites."""
from __future__ import annotations

import itertools

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as sla


def bonds(nx: int, ny: int, px: bool, py: bool):
    out = []
    for i in range(nx):
        for j in range(ny):
            p0 = j + i * ny
            if i + 1 < nx:
                out.append((p0, j + (i + 1) * ny, "x"))
            elif nx > 2 and px:
                out.append((j, p0, "x"))
            if j + 1 < ny:
                out.append((p0, (j + 1) + i * ny, "y"))
            elif ny > 2 and py:
                out.append((i * ny, p0, "y"))
    return out


def ground_energy(nx: int, ny: int, nboson: int, d: int, jx: float, jy: float, u: float, mu: float,
                  px: bool = False, py: bool = False) -> float:
    L = nx * ny
    states = [s for s in itertools.product(range(d), repeat=L) if sum(s) == nboson]
    index = {s: k for k, s in enumerate(states)}
    rows, cols, vals = [], [], []
    for k, s in enumerate(states):
        diag = sum(mu * n + u * n * (n - 1) for n in s)
        rows.append(k)
        cols.append(k)
        vals.append(diag)
        for a, b, kind in bonds(nx, ny, px, py):
            J = jx if kind == "x" else jy
            if J == 0:
                continue
            for src, dst in ((a, b), (b, a)):  # b+_dst b_src
                if s[src] == 0 or s[dst] == d - 1:
                    continue
                t = list(s)
                amp = np.sqrt(t[src]) * np.sqrt(t[dst] + 1)
                t[src] -= 1
                t[dst] += 1
                rows.append(index[tuple(t)])
                cols.append(k)
                vals.append(J * amp)
    n = len(states)
    H = sp.csr_matrix((vals, (rows, cols)), shape=(n, n))
    if n < 400:
        return float(np.linalg.eigvalsh(H.toarray())[0])
    return float(sla.eigsh(H, k=1, which="SA")[0][0])


def ground_energy_spinful(nx: int, ny: int, nup: int, ndown: int, d: int, jx: float, jy: float, u_uu: float,
                          u_dd: float, u_ud: float, mu: float, px: bool = False, py: bool = False,
                          flux: float = 0.0) -> float:
    """Two-component bosons in the (N_up, N_down) sector, the reference's
    spinful model (model/hamiltonian/complex_spinful_bose_square_hamiltonian.cc):
    per species s, J (a+ a + h.c.) on the bonds of bonds(), mu n + U_s/2 n(n-1)
    on site; U_ud n_up n_down.  With a flux, a boson hopping along y from row j
    to row j+1 (mod Ny) of column x picks up phi = exp(i 2 pi (x+1) flux) and the
    reverse hop conj(phi) (the reference's Peierls phase, :297-331).  A state
    lists (n_up, n_down) per lattice site."""
    L = nx * ny
    occ = [s for s in itertools.product(range(d), repeat=L)]
    ups = [s for s in occ if sum(s) == nup]
    dns = [s for s in occ if sum(s) == ndown]
    states = [(a, b) for a in ups for b in dns]
    index = {s: k for k, s in enumerate(states)}
    U = (u_uu, u_dd)
    rows, cols, vals = [], [], []
    for k, (a, b) in enumerate(states):
        diag = 0.0
        for sp_, occ_s in enumerate((a, b)):
            diag += sum(mu * n + 0.5 * U[sp_] * n * (n - 1) for n in occ_s)
        diag += u_ud * sum(x * y for x, y in zip(a, b))
        rows.append(k)
        cols.append(k)
        vals.append(diag)
        for p0, p1, kind in bonds(nx, ny, px, py):
            J = jx if kind == "x" else jy
            if J == 0:
                continue
            phase = {(p0, p1): 1.0, (p1, p0): 1.0}
            if kind == "y" and flux != 0.0:
                phi = np.exp(2j * np.pi * (p0 // ny + 1) * flux)
                lo, hi = (p0, p1) if (p0 % ny + 1) % ny == p1 % ny else (p1, p0)  # hi = row j + 1 of lo
                phase = {(lo, hi): phi, (hi, lo): np.conj(phi)}
            for sp_ in range(2):
                s = (a, b)[sp_]
                for src, dst in ((p0, p1), (p1, p0)):
                    if s[src] == 0 or s[dst] == d - 1:
                        continue
                    t = list(s)
                    amp = np.sqrt(t[src]) * np.sqrt(t[dst] + 1)
                    t[src] -= 1
                    t[dst] += 1
                    new = (tuple(t), b) if sp_ == 0 else (a, tuple(t))
                    rows.append(index[new])
                    cols.append(k)
                    vals.append(J * amp * phase[(src, dst)])
    n = len(states)
    H = sp.csr_matrix((np.asarray(vals, dtype=complex if flux != 0.0 else float), (rows, cols)), shape=(n, n))
    if n < 400:
        return float(np.linalg.eigvalsh(H.toarray())[0])
    return float(sla.eigsh(H, k=1, which="SA")[0][0].real)
