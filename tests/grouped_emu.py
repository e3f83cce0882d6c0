"""CPU emulation of the grouped Cholesky / solve kernels -- TEST INFRASTRUCTURE ONLY.

Runs a plan of ``sdpvibe_b200.grouped`` (its host tables: copy descriptors, grouped-GEMM items, rounding
descriptors) with numpy arenas and the oracle's primitives in place of the device kernels: exact products
and the CRT through the oracle's residue path, roundings through its shift_round / add_same, the base tiles
through its chol_tiles / trinv_tiles.  It states what each device kernel computes (the comments name the
kernel), so a plan checked here against the oracle's recursion checks the schedule, and the GPU run of
the same plan checks the kernels.
"""
import numpy as np

import oracle as O
from oracle import mp as OM


def _flat(a):
    return a.reshape(a.shape[0], -1)


def copy(desc, srcs, dst):
    """grp_copy: dst[r][c] = src[r][c] (or dst[c][r]) per descriptor"""
    d2 = _flat(dst)
    for sid, sbase, sld, dbase, dld, rows, cols, trans in desc.tolist():
        s2 = _flat(srcs[sid])
        r = np.arange(rows)[:, None]
        c = np.arange(cols)[None, :]
        v = s2[:, sbase + r * sld + c]
        if trans:
            d2[:, dbase + c * dld + r] = v
        else:
            d2[:, dbase + r * dld + c] = v


def product_wave(g, srcs, L):
    """grp_copy x 2, residues, sdpv_rns_gemm_grouped, sdpv_crt_block -> (CRT words (W, Rout w), bit lengths)"""
    T = O.tables(L)
    ws = np.zeros((L, g.RA + g.RB, g.kp), np.int32)       # big side rows, then the small side's from row RA
    copy(g.desc, srcs, ws)
    big, small = ws[:, :g.RA], ws[:, g.RA:]
    Wd = np.zeros((T.W, g.Rout * g.w), np.int32)
    bl = np.zeros((g.Rout * g.w,), np.int64)
    for b0, nbig, s0, nsmall, klen, o0, c0, _ in g.items_np.tolist():
        A = big[:, b0:b0 + nbig, :klen]
        B = small[:, s0:s0 + nsmall, :klen]
        acc = OM.exact_acc(T, A, B)                              # (n, nbig, nsmall)
        words, bits = O.crt_block(T, acc, nsmall, 0, nsmall, nbig)
        r = np.arange(nbig)[:, None]
        j = np.arange(nsmall)[None, :]
        pos = ((o0 + r) * g.w + j) if g.out_mode == 1 else ((o0 + j) * g.w + c0 + r)
        Wd[:, pos.reshape(-1)] = words
        bl[pos.reshape(-1)] = bits
    return T, Wd, bl


def finish_fixed(g, Wd, ar, L, xe):
    """grp_finish_fixed: out = base + sum_i sign_i round(W_i / 2^s_i), s_i = cst_i - xe[idx_i]"""
    for d in g.finish.tolist():
        oid, ob, old, bid, bb, bld, rows, cols, ns = d[:9]
        r = np.arange(rows)[:, None]
        c = np.arange(cols)[None, :]
        acc = _flat(ar[bid])[:, bb + r * bld + c].reshape(L, -1) if bid >= 0 else np.zeros((L, rows * cols), np.int32)
        for i in range(ns):
            cb, sg, cst, ei = d[9 + 4 * i:13 + 4 * i]
            s = cst - (int(xe[ei]) if ei >= 0 else 0)
            v, _ = O.shift_round(Wd[:, (cb + r * g.w + c).reshape(-1)], np.full(rows * cols, s, np.int64), L)
            acc = O.add_same(acc, v, int(sg))
        _flat(ar[oid])[:, (ob + r * old + c).reshape(-1)] = acc


def run_factor(plan, Fa):
    """run_factor of the plan on the numpy factor arena Fa (L, T, 32, 32), in place -> (Xa, xe)"""
    L, e, lay = plan.L, plan.e, plan.lay
    WL, LF = L + 24, L
    F = 32 * LF
    Xa = np.zeros((L, lay.D, 32, 32), np.int32)
    xe = np.zeros((lay.D,), np.int64)
    Ya = np.zeros((L, plan.ntemp, 32, 32), np.int32)
    Ra = np.zeros_like(Ya)
    ar = [Fa, Xa, Ya, Ra]
    tri = np.tril(np.ones((32, 32), bool))
    for kind, st in plan.stages:
        if kind == "tile":
            for fb, xi in zip(st["fbase"].tolist(), st["xidx"].tolist()):
                t = fb // 1024
                # grp_tile_widen: exact shift to -F in WL words, zero above the diagonal
                Wt, _ = O.shift_round(_flat(Fa[:, t]), np.full(1024, -F - e, np.int64), WL)
                Wt = np.ascontiguousarray(Wt.T.reshape(1, 32, 32, WL)).view(np.uint32)
                Wt[0, ~tri] = 0
                Lw, RINV = O.chol_tiles(Wt, 32, WL, LF)
                Xw = O.trinv_tiles(Lw, RINV, 32, WL, LF)
                # grp_tile_narrow: factor to e (zero upper), inverse to its own exponent
                Ls, _ = O.shift_round(Lw.view(np.int32).reshape(1024, WL).T, np.full(1024, e + F, np.int64), L)
                Ls = Ls.reshape(L, 32, 32)
                Ls[:, ~tri] = 0
                Fa[:, t] = Ls
                Xs = Xw.view(np.int32).reshape(1024, WL).T
                ex = int(O.bitlen(Xs).max()) - F - (32 * L - 32)
                xv, _ = O.shift_round(Xs, np.full(1024, ex + F, np.int64), L)
                Xa[:, xi] = xv.reshape(L, 32, 32)
                xe[xi] = ex
            continue
        T, Wd, bl = product_wave(st, ar, L)
        finish_fixed(st, Wd, ar, L, xe)
    return Xa, xe


def run_solve(plan, Pa, Pe, Fa, Xa, xe):
    """run_solve of the plan on numpy arenas, in place"""
    L, m = plan.L, plan.m
    hr = 32 * L - 32
    ar = [Pa, Fa, Xa]
    P2 = _flat(Pa)

    def ent(rt, r, c):
        return rt * 32 * m + r * m + c

    for kind, st in plan.stages:
        if kind == "merge":
            # grp_merge: common column exponents over the node's row tiles
            for rt0, nrt, c0, nc in st["desc"].tolist():
                for c in range(c0, c0 + nc):
                    ee = Pe[rt0:rt0 + nrt, c].max()
                    for t in range(rt0, rt0 + nrt):
                        pos = np.array([ent(t, r, c) for r in range(32)])
                        v, _ = O.shift_round(P2[:, pos], np.full(32, ee - Pe[t, c], np.int64), L)
                        P2[:, pos] = v
                        Pe[t, c] = ee
            continue
        T, Wd, bl = product_wave(st, ar, L)
        # grp_solve_round: a group's 'col' exponents over all its rows, then its entries rounded into the
        # destination row tiles (leaf store, or the aligned difference with the base rows)
        for row0, rows, c0, nc, eA, eidx, ebrt, mode, brt0, drt0 in st.round.tolist():
            for c in range(c0, c0 + nc):
                mx = int(bl[(row0 + np.arange(rows)) * st.w + c].max())
                su = mx - hr
                eu = eA + (int(xe[eidx]) if eidx >= 0 else 0) + int(Pe[ebrt, c]) + su
                for t in range(rows // 32):
                    u, _ = O.shift_round(Wd[:, (row0 + 32 * t + np.arange(32)) * st.w + c], np.full(32, su, np.int64), L)
                    pos = np.array([ent(drt0 + t, r, c) for r in range(32)])
                    if mode == 0:
                        P2[:, pos] = u
                        Pe[drt0 + t, c] = eu
                        continue
                    bpos = np.array([ent(brt0 + t, r, c) for r in range(32)])
                    eb = int(Pe[brt0 + t, c])
                    e2 = max(eb, eu) + 1
                    bv, _ = O.shift_round(P2[:, bpos], np.full(32, e2 - eb, np.int64), L)
                    uv, _ = O.shift_round(u, np.full(32, e2 - eu, np.int64), L)
                    P2[:, pos] = O.add_same(bv, uv, -1 if mode == 1 else 1)
                    Pe[drt0 + t, c] = e2
