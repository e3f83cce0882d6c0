"""Grouped batched Cholesky factorisation and triangular solves over a device work list.

Blocks of different sizes are factored and solved together: no bucket of equal sizes, no padding of a
block beyond its own multiple of 32.  Every block's result is bit-identical to the reference's recursive
bchol / btrsm_right / btrsm_left / btrsm_left_T on that block alone (sdpvibe/batched.py:243-352),
because every product, rounding point and sum is the same:

* Factorisation (fixed point at one exponent e).  With the split rule of the recursion (a range of s tiles
  splits after ceil(s/2) tiles, sdpvibe/batched.py:265) the recursion hands tile (i, j), i >= j, one rounded
  product  round_e(sum_{k in g} L_ik L_jk^T)  per range g = [lo, mid) of every tree node whose right half
  holds j (`column_groups`): btrsm_right's update and bchol's Schur complement are both of that form.  The
  subtractions are exact (fixed exponent, sdpvibe/batched.py:82-92), so their order is free.  A column j is
  then: its updates, the base tile (chol_tiles + trinv_tiles), and the panel leaf X = round(B X_j^T) with
  `refine` correction steps (sdpvibe/batched.py:291-299) -- the same column program for every block, so
  column j of all blocks runs as one wave.
* Solves (per-column exponents).  L^-1 B and L^-T B round per column over node-shaped row ranges and rescale
  both halves of every node to a common exponent (sdpvibe/batched.py:313-352), so their rounding depends on
  the tree: each block runs the program of its own tree (`solve_program`), and a greedy scheduler merges the
  programs of all blocks into waves of one operation kind (the kind of the block with the longest remaining
  program).

A wave of products is: tile copies of both operand sides into one workspace (grp_copy), its residues
(sdpv_residues_u8), one grouped narrow residue GEMM over an item table (sdpv_rns_gemm_grouped: up to 128
rows of one side against up to 64 rows of the other, K per item), one CRT (sdpv_crt_block) and the rounding
kernel of the wave (grp_finish_fixed, or grp_solve_round: column exponents and rounding of a group in one
CTA); base-tile waves are grp_tile_widen, sdpv_chol_tiles, sdpv_trinv_tiles and grp_tile_narrow; merges
are grp_merge.  Plans (host tables uploaded once) are cached per
block-size sequence.
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .rns import dev
from .mpmat import lib_ctx

BT = 32
LI = 24                         # extra words of the base tiles' wide fixed point (sdpvibe/batched.py:243)
F_AR, X_AR, Y_AR, R_AR = 0, 1, 2, 3          # factorisation arenas
P_AR, PF_AR, PX_AR = 0, 1, 2                  # solve arenas: solve state, factor, inverses
MAX_SOURCES = 7
RES_BUDGET = 2 << 30            # residue bytes of one wave's operands before the moduli are split


def split_point(lo, hi):
    """The recursion's split of tiles [lo, hi): n1 = ceil((n // 2) / 32) * 32 for n = 32 (hi - lo)."""
    return lo + (hi - lo + 1) // 2


def column_groups(s, j):
    """The tile ranges [lo, mid) whose rounded products tile column j of an s-tile block receives."""
    out, lo, hi = [], 0, s
    while hi - lo > 1:
        mid = split_point(lo, hi)
        if j >= mid:
            out.append((lo, mid))
            lo = mid
        else:
            hi = mid
    return out


def solve_program(s, lower):
    """Operation sequence of one block's L^-1 B (lower) or L^-T B solve, in dependency order."""
    ops = []

    def rec(lo, hi):
        if hi - lo == 1:
            ops.append(("leaf", lo))
            return
        mid = split_point(lo, hi)
        first, second = ((lo, mid), (mid, hi)) if lower else ((mid, hi), (lo, mid))
        rec(*first)
        ops.append(("upd", lo, mid, hi))
        rec(*second)
        ops.append(("merge", lo, mid, hi))
    rec(0, s)
    return ops


def schedule(programs):
    """Merge per-block programs into waves of one kind: each wave takes the next operation of every block
    whose next operation has the kind of the block with the longest remaining program."""
    pos = [0] * len(programs)
    waves = []
    while True:
        live = [b for b, p in enumerate(programs) if pos[b] < len(p)]
        if not live:
            return waves
        crit = max(live, key=lambda b: len(programs[b]) - pos[b])
        kind = programs[crit][pos[crit]][0]
        wave = [(b, programs[b][pos[b]]) for b in live if programs[b][pos[b]][0] == kind]
        for b, _ in wave:
            pos[b] += 1
        waves.append((kind, wave))


class Layout:
    """Arena positions of the blocks: s[b] tiles per side; lower tile (b, i, j) of the factor arena,
    diagonal tile / solve row tile (b, i)."""

    def __init__(self, sizes):
        self.s = [int(x) for x in sizes]
        self.toff = np.concatenate([[0], np.cumsum([s * (s + 1) // 2 for s in self.s])]).astype(np.int64)
        self.doff = np.concatenate([[0], np.cumsum(self.s)]).astype(np.int64)
        self.T, self.D = int(self.toff[-1]), int(self.doff[-1])

    def tile(self, b, i, j):
        return int(self.toff[b]) + i * (i + 1) // 2 + j

    def diag(self, b, i):
        return int(self.doff[b]) + i


def _chunks(seq, n):
    return [seq[a:a + n] for a in range(0, len(seq), n)]


class _Gemm:
    """One wave of grouped products: operand bands gathered into a big-side and a small-side workspace,
    the item table of the grouped residue GEMM and the accumulator rows of its outputs."""

    def __init__(self, TB, out_mode, w):
        self.TB, self.out_mode, self.w = TB, out_mode, w
        self.copies = ([], [])          # (arena, src base, src ld, row, col, rows, cols, trans) per side
        self.rows = [0, 0]
        self.kp = 32
        self.items = []
        self.out_rows = 0

    def band(self, side, srcs, trans=False):
        """A band of 32 rows: srcs = [(arena, tile base entry, ld)] along K (32 columns each).  Returns its
        first workspace row."""
        r0 = self.rows[side]
        for kk, (aid, base, ld) in enumerate(srcs):
            self.copies[side].append((aid, base, ld, r0, 32 * kk, 32, 32, trans))
        self.rows[side] += 32
        self.kp = max(self.kp, 32 * len(srcs))
        return r0

    def rows_of(self, side, srcs, m):
        """m rows from 32 x m solve tiles transposed: row c of the band is column c of the tiles; srcs along K."""
        r0 = self.rows[side]
        for kk, (aid, base, ld) in enumerate(srcs):
            for c0 in range(0, m, 32):
                self.copies[side].append((aid, base + c0, ld, r0 + c0, 32 * kk, 32, min(32, m - c0), True))
        self.rows[side] += m
        self.kp = max(self.kp, 32 * len(srcs))
        return r0

    def item(self, big_row0, big_rows, small_row0, small_rows, klen, out_row0, out_col0=0):
        self.items.append((big_row0, big_rows, small_row0, small_rows, klen, out_row0, out_col0, 0))

    def take_out_rows(self, n):
        r0 = self.out_rows
        self.out_rows += n
        return r0

    def finalize(self):
        """one copy table for both sides: the small side's rows follow the big side's RA rows in one
        workspace (one gather, one residue decomposition)"""
        kp = self.kp
        self.RA, self.RB = -(-max(self.rows[0], 1) // 32) * 32, max(self.rows[1], 1)
        off = (0, self.RA)
        self.desc = np.array([(a, b, ld, (r + off[side]) * kp + c, kp, rr, cc, int(t))
                              for side in (0, 1) for a, b, ld, r, c, rr, cc, t in self.copies[side]],
                             dtype=np.int64).reshape(-1, 8)
        self.items_np = np.array(self.items, dtype=np.int32).reshape(-1, 8)
        if self.out_mode == 1:
            self.out_rows = self.RA
        self.Rout = max(self.out_rows, 1)
        return self


def _np_desc(rows, width):
    return np.array(rows, dtype=np.int64).reshape(-1, width)


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(dev)


class _DevGemm:
    pass


def _to_device(g):
    d = _DevGemm()
    for k in ("TB", "out_mode", "w", "kp", "RA", "RB", "Rout", "nfin", "nround"):
        setattr(d, k, getattr(g, k, None))
    d.desc, d.ndesc = _dev(g.desc), len(g.desc)
    d.items, d.nitems = _dev(g.items_np), len(g.items_np)
    for k in ("finish", "round"):
        v = getattr(g, k, None)
        setattr(d, k, _dev(v) if v is not None else None)
    return d


class _Plan:
    def device_stages(self):
        """the stages with their tables on the current device (uploaded once)"""
        key = torch.cuda.current_device()
        cache = self.__dict__.setdefault("_dev_stages", {})
        if key not in cache:
            out = []
            for kind, st in self.stages:
                if kind == "gemm":
                    out.append((kind, _to_device(st)))
                else:
                    out.append((kind, {k: (_dev(v) if isinstance(v, np.ndarray) else v) for k, v in st.items()}))
            cache[key] = out
        return cache[key]


# ------------------------------------------------------------------ factorisation plan
class FactorPlan(_Plan):
    """Waves of the factorisation of blocks with s[b] tiles per side at limb count L, fixed-point exponent e.
    With `tree` and `row0` (per block) only rows >= row0[b] are computed, against a factor of tree[b] tiles
    already in the arena (columns j < tree[b]): the right solve X L^T = B of sdpvibe/batched.py:291-305 with
    B's row tiles below the factor's."""

    def __init__(self, sizes, L, e, refine, tree=None, row0=None):
        self.lay = lay = Layout(sizes)
        self.L, self.e, self.refine = L, e, refine
        nb = len(lay.s)
        self.tree = list(tree) if tree is not None else lay.s
        self.row0 = list(row0) if row0 is not None else [0] * nb
        self.stages = []
        self.ntemp = 1
        for j in range(max(self.tree)):
            blocks = [b for b in range(nb) if self.tree[b] > j]
            self._update(j, blocks)
            diag = [b for b in blocks if self.row0[b] <= j]
            if diag:
                self.stages.append(("tile", {"fbase": np.array([lay.tile(b, j, j) * 1024 for b in diag], np.int64),
                                             "xidx": np.array([lay.diag(b, j) for b in diag], np.int64),
                                             "n": len(diag)}))
            leaf = [b for b in blocks if lay.s[b] > max(j + 1, self.row0[b])]
            if leaf:
                self._leaf(j, leaf)

    def _rows(self, b, first):
        return list(range(max(first, self.row0[b]), self.lay.s[b]))

    def _gemm_stage(self, g, fin):
        g.finalize()
        g.finish = _np_desc(fin, 40)
        g.nfin = len(fin)
        self.stages.append(("gemm", g))

    def _update(self, j, blocks):
        lay, e = self.lay, self.e
        g = _Gemm(TB=32, out_mode=1, w=32)
        srcs = {}
        for b in blocks:
            rows = self._rows(b, j)
            for lo, mid in column_groups(self.tree[b], j):
                if not rows:
                    continue
                srow = g.band(1, [(F_AR, lay.tile(b, j, k) * 1024, 32) for k in range(lo, mid)])
                for ch in _chunks(rows, 4):
                    r0 = None
                    for i in ch:
                        r = g.band(0, [(F_AR, lay.tile(b, i, k) * 1024, 32) for k in range(lo, mid)])
                        r0 = r if r0 is None else r0
                        srcs.setdefault(lay.tile(b, i, j), []).append((r * 32, -1, -e, -1))
                    g.item(r0, 32 * len(ch), srow, 32, 32 * (mid - lo), r0)
        if not g.items:
            return
        fin = []
        for t, ss in srcs.items():
            assert len(ss) <= MAX_SOURCES
            row = [F_AR, t * 1024, 32, F_AR, t * 1024, 32, 32, 32, len(ss)]
            for s in ss:
                row += list(s)
            fin.append(row + [0] * (40 - len(row)))
        self._gemm_stage(g, fin)

    def _leaf(self, j, blocks):
        """X = round(B X_j^T); refine x { R = B - round(X L_jj^T); X = X + round(R X_j^T) }  (B = tile (i, j))."""
        lay, e = self.lay, self.e
        tiles = [(b, i) for b in blocks for i in self._rows(b, j + 1)]
        self.ntemp = max(self.ntemp, len(tiles))
        tmp = {bi: q for q, bi in enumerate(tiles)}

        def wave(small_of, big_of, out_of, base_of, sign, cst, eidx_of):
            g = _Gemm(TB=32, out_mode=1, w=32)
            fin = []
            for b in blocks:
                srow = g.band(1, [small_of(b)])
                for ch in _chunks(self._rows(b, j + 1), 4):
                    r0 = None
                    for i in ch:
                        r = g.band(0, [big_of(b, i)])
                        r0 = r if r0 is None else r0
                        oa, ob = out_of(b, i)
                        ba, bb = base_of(b, i)
                        row = [oa, ob, 32, ba, bb, 32, 32, 32, 1, r * 32, sign, cst, eidx_of(b)]
                        fin.append(row + [0] * (40 - len(row)))
                    g.item(r0, 32 * len(ch), srow, 32, 32, r0)
            self._gemm_stage(g, fin)

        F = lambda b, i: (F_AR, lay.tile(b, i, j) * 1024)
        Y = lambda b, i: (Y_AR, tmp[(b, i)] * 1024)
        R = lambda b, i: (R_AR, tmp[(b, i)] * 1024)
        Xj = lambda b: (X_AR, lay.diag(b, j) * 1024, 32)
        Ljj = lambda b: (F_AR, lay.tile(b, j, j) * 1024, 32)
        none = lambda b, i: (-1, 0)
        xe = lambda b: lay.diag(b, j)
        first_out = Y if self.refine else F
        wave(Xj, lambda b, i: F(b, i) + (32,), first_out, none, 1, 0, xe)
        for it in range(self.refine):
            wave(Ljj, lambda b, i: Y(b, i) + (32,), R, F, -1, -e, lambda b: -1)
            wave(Xj, lambda b, i: R(b, i) + (32,), F if it == self.refine - 1 else Y, Y, 1, 0, xe)


# ------------------------------------------------------------------ solve plan
class SolvePlan(_Plan):
    """Waves of L^-1 B (lower) or L^-T B for blocks with s[b] tiles and m right-hand sides; refine = 0."""

    def __init__(self, sizes, L, e, m, lower):
        self.lay = lay = Layout(sizes)
        self.L, self.e, self.m, self.lower = L, e, m, lower
        progs = [solve_program(s, lower) for s in lay.s]
        self.stages = []
        for kind, wave in schedule(progs):
            if kind == "merge":
                d = []
                for b, (_, lo, mid, hi) in wave:
                    for c0 in range(0, m, 32):
                        d.append((lay.diag(b, lo), hi - lo, c0, min(32, m - c0)))
                self.stages.append(("merge", {"desc": _np_desc(d, 4), "n": len(d)}))
            else:
                self._products(kind, wave)

    def _products(self, kind, wave):
        lay, m, e, lower = self.lay, self.m, self.e, self.lower
        narrow_rhs = m <= 64
        if narrow_rhs:
            TB = -(-m // 16) * 16
            g = _Gemm(TB=TB, out_mode=1, w=TB)
        else:
            g = _Gemm(TB=32 if kind == "leaf" else 64, out_mode=2, w=m)
        rnd = []
        for q, (b, op) in enumerate(wave):
            if kind == "leaf":
                j = op[1]
                a_bands = [[(PX_AR, lay.diag(b, j) * 1024, 32)]]
                a_trans = not lower
                p_tiles = [(P_AR, lay.diag(b, j) * 32 * m, m)]
                out_rts = [lay.diag(b, j)]
                eA, eA_idx, eB_rt, mode = 0, lay.diag(b, j), lay.diag(b, j), 0
            else:
                _, lo, mid, hi = op
                if lower:
                    out_range, k_range = range(mid, hi), range(lo, mid)
                    a_bands = [[(PF_AR, lay.tile(b, i, k) * 1024, 32) for k in k_range] for i in out_range]
                else:
                    out_range, k_range = range(lo, mid), range(mid, hi)
                    a_bands = [[(PF_AR, lay.tile(b, t, i) * 1024, 32) for t in k_range] for i in out_range]
                a_trans = not lower
                p_tiles = [(P_AR, lay.diag(b, k) * 32 * m, m) for k in k_range]
                out_rts = [lay.diag(b, i) for i in out_range]
                eA, eA_idx, eB_rt, mode = e, -1, lay.diag(b, k_range[0]), 1
            klen = 32 * len(p_tiles)
            if narrow_rhs:
                srow = g.rows_of(1, p_tiles, m)
                rows0 = []
                for ch in _chunks(a_bands, 4):
                    r0 = None
                    for band in ch:
                        r = g.band(0, band, a_trans)
                        r0 = r if r0 is None else r0
                        rows0.append(r)
                    g.item(r0, 32 * len(ch), srow, m, klen, r0)
            else:
                prow = g.rows_of(0, p_tiles, m)
                rows0 = []
                for ch in _chunks(a_bands, 2):
                    s0 = None
                    for band in ch:
                        r = g.band(1, band, a_trans)
                        s0 = r if s0 is None else s0
                    o0 = g.take_out_rows(32 * len(ch))
                    rows0 += [o0 + 32 * u for u in range(len(ch))]
                    for p0 in range(0, m, 128):
                        g.item(prow + p0, min(128, m - p0), s0, 32 * len(ch), klen, o0, p0)
            assert all(b - a == 32 for a, b in zip(rows0, rows0[1:])), "a group's output rows are consecutive"
            for c0 in range(0, m, 32):
                rnd.append((rows0[0], 32 * len(rows0), c0, min(32, m - c0), eA, eA_idx, eB_rt, mode, out_rts[0],
                            out_rts[0]))
        g.finalize()
        g.round, g.nround = _np_desc(rnd, 10), len(rnd)
        g.finish, g.nfin = None, 0
        self.stages.append(("gemm", g))


# ------------------------------------------------------------------ execution
def _ptrs(tensors):
    """host arrays of the arenas' device pointers and plane strides (entries), as the C ABI takes them"""
    arr = (ctypes.c_void_p * 4)(*([t.data_ptr() for t in tensors] + [None] * (4 - len(tensors))))
    planes = (ctypes.c_int64 * 4)(*([t[0].numel() for t in tensors] + [0] * (4 - len(tensors))))
    keep = (arr, planes)
    return ctypes.cast(arr, ctypes.c_void_p), ctypes.cast(planes, ctypes.c_void_p), len(tensors), keep


def _residue_products(R, g, ws, acc):
    """acc <- residues of the wave's grouped products: the workspace's rows decomposed once (moduli split into
    groups within the residue budget), the big side its first RA rows, the small side the rest."""
    rows = g.RA + g.RB
    per_mod = 2 * g.kp * rows
    GR = R.n if R.n * per_mod <= RES_BUDGET else max(16, (RES_BUDGET // per_mod) // 16 * 16)
    small_off = g.RA * g.kp
    for g0 in range(0, R.n, GR):
        G = min(GR, R.n - g0)
        rh, rl = R.residues(ws, 0, g.kp, g0, G, spread=True, unsigned=True)
        hp, lp = rh.data_ptr(), rl.data_ptr()
        _lib.call("sdpv_rns_gemm_grouped", R.handle, ctypes.c_void_p(hp), ctypes.c_void_p(lp), g.RA, rh.stride(0),
                  ctypes.c_void_p(hp + small_off), ctypes.c_void_p(lp + small_off), g.RB, rh.stride(0), g.kp, g.TB,
                  g.out_mode, _lib.ptr(g.items), g.nitems, _lib.ptr(acc), g.w, g.Rout, g0, G, _lib.stream())
        del rh, rl


def _product_wave(g, arenas, L):
    """gather (both sides, one launch), residues (one launch), grouped GEMM, CRT -> (CRT words (W, Rout w),
    bit lengths)"""
    R = lib_ctx(L)
    arr, planes, n, _keep = _ptrs(arenas)
    ws = torch.empty((L, g.RA + g.RB, g.kp), dtype=torch.int32, device=dev)
    _lib.call("sdpv_grp_copy", arr, planes, n, _lib.ptr(ws), ws[0].numel(), L, _lib.ptr(g.desc), g.ndesc, _lib.stream())
    acc = torch.empty((R.n, g.Rout, g.w), dtype=torch.int16, device=dev)
    _residue_products(R, g, ws, acc)
    del ws
    Wd, bl, _ = R.crt_block(acc, g.w, 0, g.w, g.Rout)
    return R, Wd, bl


def run_factor(plan, Fa, Xa=None, xe=None):
    """Factor the blocks held in the factor arena Fa (L, T, 32, 32) in place; returns (X arena, xe)."""
    L, e = plan.L, plan.e
    lay = plan.lay
    WL, LF = L + LI, L
    if Xa is None:
        Xa = torch.empty((L, lay.D, BT, BT), dtype=torch.int32, device=dev)
        xe = torch.empty((lay.D,), dtype=torch.int64, device=dev)
    Ya = torch.empty((L, plan.ntemp, BT, BT), dtype=torch.int32, device=dev)
    Ra = torch.empty_like(Ya)
    arenas = [Fa, Xa, Ya, Ra]
    for kind, st in plan.device_stages():
        if kind == "tile":
            n = st["n"]
            Wb = torch.empty((n, BT, BT, WL), dtype=torch.int32, device=dev)
            _lib.call("sdpv_grp_tile_widen", _lib.ptr(Fa), Fa[0].numel(), L, e, WL, LF, _lib.ptr(st["fbase"]), n,
                      _lib.ptr(Wb), _lib.stream())
            RINV = torch.empty((n, BT, WL), dtype=torch.int32, device=dev)
            _lib.call("sdpv_chol_tiles", _lib.ptr(Wb), _lib.ptr(RINV), n, BT, WL, LF, _lib.stream())
            Xw = torch.empty_like(Wb)
            scratch = Xw if WL <= 64 else torch.empty_like(Wb)   # the shared-memory inverse needs no scratch
            _lib.call("sdpv_trinv_tiles", _lib.ptr(Wb), _lib.ptr(RINV), _lib.ptr(Xw), _lib.ptr(scratch), n, BT, WL, LF,
                      _lib.stream())
            _lib.call("sdpv_grp_tile_narrow", _lib.ptr(Wb), _lib.ptr(Xw), WL, LF, _lib.ptr(Fa), Fa[0].numel(), L, e,
                      _lib.ptr(st["fbase"]), _lib.ptr(Xa), Xa[0].numel(), _lib.ptr(st["xidx"]), _lib.ptr(xe), n,
                      _lib.stream())
            continue
        R, Wd, bl = _product_wave(st, arenas, L)
        arr, planes, n, _keep = _ptrs(arenas)
        _lib.call("sdpv_grp_finish_fixed", _lib.ptr(Wd), R.W, Wd.shape[1], st.w, arr, planes, n, L, _lib.ptr(xe),
                  _lib.ptr(st.finish), st.nfin, _lib.stream())
    return Xa, xe


def run_solve(plan, Pa, Pe, Fa, Xa, xe):
    """Solve in place on the solve arena Pa (L, RT, 32, m) with exponents Pe (RT, m)."""
    L, m = plan.L, plan.m
    arenas = [Pa, Fa, Xa]
    for kind, st in plan.device_stages():
        if kind == "merge":
            _lib.call("sdpv_grp_merge", _lib.ptr(Pa), Pa[0].numel(), _lib.ptr(Pe), m, L, _lib.ptr(st["desc"]), st["n"],
                      _lib.stream())
            continue
        R, Wd, bl = _product_wave(st, arenas, L)
        _lib.call("sdpv_grp_solve_round", _lib.ptr(Wd), _lib.ptr(bl), R.W, Wd.shape[1], st.w, _lib.ptr(Pa), Pa[0].numel(),
                  _lib.ptr(Pe), m, L, _lib.ptr(xe), _lib.ptr(st.round), st.nround, _lib.stream())


_PLANS = {}


def factor_plan(sizes, L, e, refine):
    key = ("f", tuple(sizes), L, e, refine)
    if key not in _PLANS:
        _PLANS[key] = FactorPlan(sizes, L, e, refine)
    return _PLANS[key]


def solve_plan(sizes, L, e, m, lower):
    key = ("s", tuple(sizes), L, e, m, lower)
    if key not in _PLANS:
        _PLANS[key] = SolvePlan(sizes, L, e, m, lower)
    return _PLANS[key]


# ------------------------------------------------------------------ dense <-> arena
_IDX = {}


def tile_positions(s):
    """flat positions (in an s*32 x s*32 row-major matrix) of the lower tiles' entries, in arena order"""
    n = 32 * s
    idx = []
    for i in range(s):
        for j in range(i + 1):
            r = np.arange(32)[:, None] + 32 * i
            c = np.arange(32)[None, :] + 32 * j
            idx.append((r * n + c).reshape(-1))
    return np.concatenate(idx)


def _tile_index(s):
    key = ("t", s, torch.cuda.current_device())
    if key not in _IDX:
        _IDX[key] = torch.from_numpy(tile_positions(s)).to(dev)
    return _IDX[key]


def dense_to_arena(P, Fa, lay, b0):
    """P (L, nb, n, n) fixed point -> the factor arena tiles of blocks b0 .. b0 + nb - 1 (all of s = n / 32)."""
    L, nb, n, _ = P.shape
    s = n // 32
    T_b = s * (s + 1) // 2
    t0 = int(lay.toff[b0])
    idx = _tile_index(s)
    Fa.view(L, -1)[:, t0 * 1024:(t0 + nb * T_b) * 1024].view(L, nb, T_b * 1024).copy_(
        P.reshape(L, nb, n * n).index_select(2, idx))


def arena_to_dense(Fa, lay, b0, nb, s):
    """the lower tiles of blocks b0 .. b0 + nb - 1 -> dense (L, nb, 32 s, 32 s) with zero upper tiles"""
    L = Fa.shape[0]
    n = 32 * s
    T_b = s * (s + 1) // 2
    t0 = int(lay.toff[b0])
    out = torch.zeros((L, nb, n * n), dtype=torch.int32, device=dev)
    out.index_copy_(2, _tile_index(s), Fa.view(L, -1)[:, t0 * 1024:(t0 + nb * T_b) * 1024].view(L, nb, T_b * 1024))
    return out.view(L, nb, n, n)


# ------------------------------------------------------------------ public objects
class Factorisation:
    """Cholesky factors of batches of equilibrated fixed-point blocks, all factored by one grouped plan.
    batches: (L, nb_q, n_q, n_q) int32 limb planes at the fixed-point exponent e, n_q a multiple of 32; the
    factorisation runs as one CUDA-graph replay per sequence of batch shapes (graphs.run)."""

    def __init__(self, batches, e, refine=1):
        from . import graphs
        L = batches[0].shape[0]
        self.L, self.e, self.refine = L, int(e), refine
        self.batches = [(int(P.shape[1]), int(P.shape[2]) // BT) for P in batches]
        self.sizes = [s for nb, s in self.batches for _ in range(nb)]
        self.lay = lay = Layout(self.sizes)
        self.b0 = [int(x) for x in np.cumsum([0] + [nb for nb, _ in self.batches])[:-1]]
        plan = factor_plan(self.sizes, L, self.e, refine)

        def fn(ins):
            Fa = torch.empty((L, lay.T, BT, BT), dtype=torch.int32, device=dev)
            for P, b0 in zip(ins, self.b0):
                dense_to_arena(P.contiguous(), Fa, lay, b0)
            Xa, xe = run_factor(plan, Fa)
            return [Fa, Xa, xe]
        self.Fa, self.Xa, self.xe = graphs.run(("gfactor", L, tuple(self.batches), self.e, refine), fn, list(batches))

    def dense(self, q):
        """batch q's factor as dense limb planes (L, nb, n, n), zero above the diagonal"""
        nb, s = self.batches[q]
        return arena_to_dense(self.Fa, self.lay, self.b0[q], nb, s)

    def _index(self, key, make):
        """a device index tensor of this layout, made once (no host-device copy on later calls)"""
        ck = (tuple(self.batches), key, torch.cuda.current_device())
        if ck not in _IDX:
            _IDX[ck] = torch.from_numpy(np.ascontiguousarray(make(), dtype=np.int64)).to(dev)
        return _IDX[ck]

    def diag_tile(self, q, j):
        """batch q's diagonal tile j: (inverse limbs (L, nb, 32, 32), its exponents (nb,), factor limbs)"""
        nb, _ = self.batches[q]
        bs = range(self.b0[q], self.b0[q] + nb)
        di = self._index(("d", q, j), lambda: [self.lay.diag(b, j) for b in bs])
        ti = self._index(("t", q, j), lambda: [self.lay.tile(b, j, j) for b in bs])
        return self.Xa.index_select(1, di), self.xe.index_select(0, di), self.Fa.index_select(1, ti)

    def diagonal(self, q):
        """limbs of the diagonal of batch q's factor, (L, nb, n)"""
        nb, s = self.batches[q]

        def make():
            b = np.arange(self.b0[q], self.b0[q] + nb)[:, None]
            i = np.arange(BT * s)[None, :]
            t = self.lay.toff[b] + (i // BT) * (i // BT + 1) // 2 + i // BT
            return (t * 1024 + (i % BT) * (BT + 1)).reshape(-1)
        idx = self._index(("diag", q), make)
        return self.Fa.view(self.L, -1).index_select(1, idx).view(self.L, nb, BT * s)


def factor_from_tiles(Lf, e, Xs, xes):
    """A Factorisation object over an existing factor: Lf (L, nb, n, n) at exponent e, the diagonal tiles'
    inverses Xs[j] (L, nb, 32, 32) with exponents xes[j] (nb,) -- the form the reference's bchol returns."""
    fac = Factorisation.__new__(Factorisation)
    L, nb, n, _ = Lf.shape
    s = n // BT
    fac.L, fac.e, fac.refine = L, int(e), None
    fac.batches = [(nb, s)]
    fac.sizes = [s] * nb
    fac.lay = lay = Layout(fac.sizes)
    fac.b0 = [0]
    fac.Fa = torch.empty((L, lay.T, BT, BT), dtype=torch.int32, device=dev)
    dense_to_arena(Lf.contiguous(), fac.Fa, lay, 0)
    fac.Xa = torch.empty((L, lay.D, BT, BT), dtype=torch.int32, device=dev)
    fac.xe = torch.empty((lay.D,), dtype=torch.int64, device=dev)
    for j in range(s):
        di = torch.tensor([lay.diag(b, j) for b in range(nb)], device=dev)
        fac.Xa.index_copy_(1, di, Xs[j].contiguous())
        fac.xe.index_copy_(0, di, xes[j].contiguous())
    return fac


def right_solve(fac, Bm, refine=1):
    """X with X L^T = B for fac's one batch: Bm (L, nb, mrows, n) at fac's exponent, n = fac's padded size
    (sdpvibe/batched.py:291-305): the factorisation's column program on B's row tiles, placed below the
    factor in a larger arena."""
    L, nb, mr, n = Bm.shape
    s = n // BT
    rb = -(-mr // BT)
    assert fac.batches == [(nb, s)]
    lay = Layout([s + rb] * nb)
    plan = FactorPlan([s + rb] * nb, L, fac.e, refine, tree=[s] * nb, row0=[s] * nb)
    Fa = torch.zeros((L, lay.T, BT, BT), dtype=torch.int32, device=dev)
    big = torch.zeros((L, nb, BT * (s + rb), BT * (s + rb)), dtype=torch.int32, device=dev)
    big[:, :, :n, :n] = arena_to_dense(fac.Fa, fac.lay, 0, nb, s)
    big[:, :, n:n + mr, :n] = Bm
    dense_to_arena(big, Fa, lay, 0)
    Xa = torch.zeros((L, lay.D, BT, BT), dtype=torch.int32, device=dev)
    xe = torch.zeros((lay.D,), dtype=torch.int64, device=dev)
    for b in range(nb):
        Xa[:, lay.diag(b, 0):lay.diag(b, 0) + s] = fac.Xa[:, fac.lay.diag(b, 0):fac.lay.diag(b, 0) + s]
        xe[lay.diag(b, 0):lay.diag(b, 0) + s] = fac.xe[fac.lay.diag(b, 0):fac.lay.diag(b, 0) + s]
    run_factor(plan, Fa, Xa, xe)
    return arena_to_dense(Fa, lay, 0, nb, s + rb)[:, :, n:n + mr, :n].contiguous()


def solve(fac, rhs, lower, Fa=None, Xa=None, xe=None):
    """L^-1 B (lower) or L^-T B for every batch of fac: rhs = [(limbs (L, nb_q, n_q, m), column exponents
    (nb_q, m))] at the batches' padded sizes, all with the same m; returns the solutions in the same form
    (sdpvibe/batched.py:322-352 with refine = 0, per block).  Fa, Xa, xe default to fac's arenas (a caller
    replaying a graph passes its static copies)."""
    Fa = fac.Fa if Fa is None else Fa
    Xa = fac.Xa if Xa is None else Xa
    xe = fac.xe if xe is None else xe
    L, lay = fac.L, fac.lay
    m = int(rhs[0][0].shape[-1])
    plan = solve_plan(fac.sizes, L, fac.e, m, lower)
    Pa = torch.empty((L, lay.D, BT, m), dtype=torch.int32, device=dev)
    Pe = torch.empty((lay.D, m), dtype=torch.int64, device=dev)
    for (Pm, pe), (nb, s), b0 in zip(rhs, fac.batches, fac.b0):
        r0 = lay.diag(b0, 0)
        Pa[:, r0:r0 + nb * s].view(L, nb, s * BT, m).copy_(Pm)
        Pe[r0:r0 + nb * s].view(nb, s, m).copy_(pe[:, None, :].expand(nb, s, m))
    run_solve(plan, Pa, Pe, Fa, Xa, xe)
    out = []
    for (nb, s), b0 in zip(fac.batches, fac.b0):
        r0 = lay.diag(b0, 0)
        out.append((Pa[:, r0:r0 + nb * s].reshape(L, nb, s * BT, m), Pe[r0:r0 + nb * s].view(nb, s, m)[:, 0].contiguous()))
    return out
