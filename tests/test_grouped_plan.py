"""The grouped Cholesky / solve plans (sdpvibe_b200.grouped) run on the CPU emulation of their kernels
(tests/grouped_emu.py) give, block by block, exactly the oracle's restatement of the reference's recursion
(sdpvibe/batched.py:243-352): factor, tile inverses and their exponents, L^-1 B and L^-T B -- for blocks of
different sizes in one plan, both orientations of the right-hand-side products (m <= 64 and m > 64)."""
import numpy as np
import pytest

import oracle as O
from oracle import mp as OM
import grouped_emu as emu
from sdpvibe_b200 import grouped as G


def _spd_blocks(rng, ns, L):
    out = []
    for n in ns:
        Gm = rng.integers(-40, 41, size=(n, n)).astype(object)
        d = rng.integers(-20, 21, size=n)
        A = Gm.dot(Gm.T) + np.eye(n, dtype=object) * (50 * n)
        vals = [int(A[i, j]) for i in range(n) for j in range(n)]
        exps = [int(d[i] + d[j]) for i in range(n) for j in range(n)]
        m, e = O.mpf_norm(O.to_limbs(vals, L), np.array(exps, np.int64), L)
        out.append((m.reshape(L, 1, n, n), e.reshape(1, n, n)))
    return out


def _rand_rhs(rng, L, n, m):
    vals = [int(v) for v in rng.integers(-(1 << 60), 1 << 60, size=n * m)]
    m_, e_ = O.mpf_norm(O.to_limbs(vals, L), rng.integers(-30, 30, size=n * m).astype(np.int64), L)
    return m_.reshape(L, 1, n, m), e_.reshape(1, n, m)


def _grouped(refs, L, m, rhs, lower):
    sizes = [r.npad // 32 for r in refs]
    e = refs[0].efx
    fplan = G.factor_plan(sizes, L, e, 1)
    lay = fplan.lay
    Fa = np.zeros((L, lay.T, 32, 32), np.int32)
    for b, r in enumerate(refs):
        pos = G.tile_positions(sizes[b])
        t0 = lay.tile(b, 0, 0)
        Fa.reshape(L, -1)[:, t0 * 1024:t0 * 1024 + pos.size] = r.P.reshape(L, -1)[:, pos]
    Xa, xe = emu.run_factor(fplan, Fa)
    splan = G.solve_plan(sizes, L, e, m, lower)
    Pa = np.zeros((L, lay.D, 32, m), np.int32)
    Pe = np.zeros((lay.D, m), np.int64)
    for b, (P, cE) in enumerate(rhs):
        r0 = lay.diag(b, 0)
        Pa[:, r0:r0 + sizes[b]] = P.reshape(L, sizes[b], 32, m)
        Pe[r0:r0 + sizes[b]] = cE[0][None, :]
    emu.run_solve(splan, Pa, Pe, Fa, Xa, xe)
    return lay, Fa, Xa, xe, Pa, Pe


@pytest.mark.parametrize("ns,m,L", [((20, 40, 70, 100, 150), 3, 8), ((33, 170), 70, 6), ((250,), 5, 4)])
def test_grouped_plan_matches_oracle_recursion(ns, m, L):
    rng = np.random.default_rng(sum(ns) + m)
    refs, rhs_l, rhs_u, out_l, out_u = [], [], [], [], []
    for (Am, Ae) in _spd_blocks(rng, ns, L):
        ref = OM.Chol.__new__(OM.Chol)
        # the oracle's equilibration and recursion, keeping the padded fixed-point input
        orig = OM.bchol
        def keep(P, e, bt=32, refine=1, _o=orig, _r=ref):
            if not hasattr(_r, "P"):                          # the outermost call's input
                _r.P = P
            return _o(P, e, bt, refine)
        OM.bchol = keep
        try:
            OM.Chol.__init__(ref, Am, Ae)
        finally:
            OM.bchol = orig
        refs.append(ref)
        Bm, Be = _rand_rhs(rng, L, Am.shape[2], m)
        P, cE = ref._to_bmp(Bm, Be)
        rhs_l.append((P, cE))
        rhs_u.append((P, cE))
        out_l.append(OM.btrsm_left(ref.Lt, ref.efx, P, cE, ref.tiles, 32, 0))
        out_u.append(OM.btrsm_left_T(ref.Lt, ref.efx, P, cE, ref.tiles, 32, 0))
    for lower, rhs, outs in ((True, rhs_l, out_l), (False, rhs_u, out_u)):
        lay, Fa, Xa, xe, Pa, Pe = _grouped(refs, L, m, rhs, lower)
        for b, r in enumerate(refs):
            s = r.npad // 32
            pos = G.tile_positions(s)
            t0 = lay.tile(b, 0, 0)
            dense = np.zeros((L, s * 32 * s * 32), np.int32)
            dense[:, pos] = Fa.reshape(L, -1)[:, t0 * 1024:t0 * 1024 + pos.size]
            assert np.array_equal(dense.reshape(L, 1, 32 * s, 32 * s), r.Lt), ("factor", b)
            for j, t in enumerate(r.tiles):
                assert np.array_equal(Xa[:, lay.diag(b, j)], t.X[:, 0]), ("inverse", b, j)
                assert int(xe[lay.diag(b, j)]) == int(t.Xe[0, 0]), ("inverse exponent", b, j)
            Pr, Per = outs[b]
            r0 = lay.diag(b, 0)
            got = Pa[:, r0:r0 + s].reshape(L, 1, 32 * s, m)
            assert np.array_equal(got, Pr), ("solve", lower, b)
            assert np.array_equal(Pe[r0:r0 + s], np.broadcast_to(OM.expt(Per, 1, m), (s, m))), ("solve exps", lower, b)


def test_schedule_merges_blocks_of_every_size():
    """Column waves of the factorisation serve all blocks; the solve waves of blocks of 1..5 tiles are as
    many as the longest program (13 operations for 5 tiles)."""
    plan = G.FactorPlan([1, 2, 3, 4, 5], 4, -(32 * 4 - 40), 1)
    tiles = [st for kind, st in plan.stages if kind == "tile"]
    assert len(tiles) == 5 and tiles[0]["n"] == 5 and tiles[4]["n"] == 1
    progs = [G.solve_program(s, True) for s in (1, 2, 3, 4, 5)]
    assert len(G.schedule(progs)) == max(len(p) for p in progs) == 13
    assert G.column_groups(5, 4) == [(0, 3), (3, 4)] and G.column_groups(32, 31) == [(0, 16), (16, 24), (24, 28),
                                                                                   (28, 30), (30, 31)]
