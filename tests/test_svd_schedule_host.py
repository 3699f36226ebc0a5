"""The batched SVD's pair-solve schedule (svd.cu, build_pair_schedule), checked
independently of the library's own checks: each of the 63 steps rotates 32
disjoint column pairs covering all 64 columns, every two columns share exactly
one step (a cyclic sweep of the pair's Gram matrix), in each half-warp the 16
columns addressed first, and the 16 addressed second, are distinct mod 16
(8-byte shared-memory banks), and the seat lanes match the circle seating that
the solve's register-resident rotation accumulation follows."""
import numpy as np

from dmrgcc_b200 import capi


def seat_column(seat, r):
    return 0 if seat == 0 else (seat - 1 - r) % 63 + 1


def fields(tab):
    return (tab & 63, (tab >> 6) & 63, (tab >> 12) & 1, (tab >> 13) & 31, (tab >> 18) & 1)


def test_pair_schedule_is_a_cyclic_sweep_without_bank_collisions():
    tab = capi.svd_pair_schedule().astype(np.int64)
    a, b, flip, _, _ = fields(tab)
    assert np.all(a < b) and np.all(tab >> 19 == 0)
    met = np.zeros((64, 64), dtype=np.int64)
    for r in range(63):
        assert sorted(np.concatenate([a[r], b[r]]).tolist()) == list(range(64))
        np.add.at(met, (a[r], b[r]), 1)
        first = np.where(flip[r] == 1, b[r], a[r])
        second = np.where(flip[r] == 1, a[r], b[r])
        for h in (slice(0, 16), slice(16, 32)):
            assert len(set((first[h] % 16).tolist())) == 16
            assert len(set((second[h] % 16).tolist())) == 16
    assert np.array_equal(met[np.triu_indices(64, 1)], np.ones(64 * 63 // 2, dtype=np.int64))


def test_seat_lanes_follow_the_circle_seating():
    tab = capi.svd_pair_schedule().astype(np.int64)
    a, b, flip, j, jflip = fields(tab)
    for r in range(63):
        assert sorted(j[r].tolist()) == list(range(32))
        for lane in range(32):
            s0, s1 = seat_column(j[r, lane], r), seat_column(63 - j[r, lane], r)
            assert {s0, s1} == {a[r, lane], b[r, lane]}
            first = b[r, lane] if flip[r, lane] else a[r, lane]
            assert jflip[r, lane] == (s0 != first)


def test_seat_shift_accumulates_the_rotation_product():
    """The solve's accumulation of Q = J_0 J_1 ... with each lane holding the two
    seats j, 63 - j of every row and moving them one seat per step (two shuffles)
    gives the same Q as rotating the columns of Q in place (two inner sweeps of
    random rotations, in the oriented form the log stores)."""
    tab = capi.svd_pair_schedule().astype(np.int64)
    a, b, flip, j, jflip = fields(tab)
    rng = np.random.default_rng(7)
    steps = 126
    theta = rng.uniform(-np.pi, np.pi, size=(steps, 32))
    direct = np.eye(64)
    log = np.zeros((steps, 32, 2))
    for t in range(steps):
        r = t % 63
        for lane in range(32):
            c, s = np.cos(theta[t, lane]), np.sin(theta[t, lane])
            p, q = (b[r, lane], a[r, lane]) if flip[r, lane] else (a[r, lane], b[r, lane])
            qp, qq = direct[:, p].copy(), direct[:, q].copy()
            direct[:, p], direct[:, q] = c * qp - s * qq, s * qp + c * qq
            log[t, j[r, lane]] = (c, -s if jflip[r, lane] else s)
    # the register form: q1[row, lane] = seat lane, q2[row, lane] = seat 63 - lane
    rows = np.arange(64)[:, None]
    lanes = np.arange(32)[None, :]
    q1 = (rows == lanes).astype(float)
    q2 = (rows == 63 - lanes).astype(float)
    for t in range(steps):
        c, s = log[t, :, 0][None, :], log[t, :, 1][None, :]
        f, g = c * q1 - s * q2, s * q1 + c * q2
        up_src = np.where(lanes == 0, g, f)
        up = np.concatenate([up_src[:, :1], up_src[:, :-1]], axis=1)      # lane k <- lane k - 1
        dn = np.concatenate([g[:, 1:], g[:, -1:]], axis=1)                # lane k <- lane k + 1
        q1 = np.where(lanes == 0, f, up)
        q2 = np.where(lanes == 31, f, dn)
    reg = np.zeros((64, 64))
    for lane in range(32):
        reg[:, seat_column(lane, steps)] = q1[:, lane]
        reg[:, seat_column(63 - lane, steps)] = q2[:, lane]
    assert np.allclose(reg, direct, atol=1e-13)


def _tiles(nb, meas):
    """measure matrix (nb x nb, symmetric) -> the planner's tile order (bi <= bj, row-major)"""
    return np.array([meas[i, j] for i in range(nb) for j in range(i, nb)])


def test_guided_rounds_cover_every_unconverged_pair_once():
    """The measure-guided sweep (svd.cu, problem_rounds): every round is a
    matching of column blocks, every block pair whose measure is above tol is
    solved exactly once, every block unconverged only within itself takes part
    in some pair, and a sweep never needs more rounds than the full round-robin
    order plus one round per such block.  Random measure patterns, from a few
    unconverged pairs (the late sweeps) to all of them (the first)."""
    rng = np.random.default_rng(5)
    tol = 1e-14
    for cols in (20, 64, 100, 384, 550, 668):
        nb = (cols + 31) // 32
        nbe = max(2, nb + (nb & 1))
        for frac in (0.0, 0.05, 0.3, 1.0):
            meas = np.where(rng.random((nb, nb)) < frac, rng.uniform(2, 1e6, (nb, nb)) * tol,
                            rng.uniform(0, 0.9, (nb, nb)) * tol)
            meas = np.triu(meas) + np.triu(meas, 1).T
            rounds = capi.svd_plan_rounds(cols, _tiles(nb, meas), tol)
            seen = {}
            in_pair = set()
            for rd in rounds:
                used = [b for pr in rd for b in pr]
                assert len(used) == len(set(used)), "a block twice in one round"
                for bi, bj in rd:
                    assert 0 <= bi < bj < nbe
                    seen[(bi, bj)] = seen.get((bi, bj), 0) + 1
                    in_pair.update((bi, bj))
            need = {(i, j) for i in range(nb) for j in range(i + 1, nb) if meas[i, j] > tol}
            for pr in need:
                assert seen.get(pr) == 1, (cols, frac, pr)
            internal = [i for i in range(nb) if meas[i, i] > tol]
            for i in internal:
                assert i in in_pair
            if not need and not internal:
                assert rounds == []
            assert len(rounds) <= (nbe - 1) + len(internal)
