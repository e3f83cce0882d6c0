"""Multiprecision dense Cholesky and triangular solves of one matrix: drop-in for ``sdpvibe.linalg``
(sdpvibe/linalg.py:1-138).  Matrices are ``MP`` block-floating arrays (mpmat); a Cholesky input is SPD,
equilibrated (|a_ij| <= 1) and in fixed point with exponent fx_exp(L).

The reference defines these results by a recursion over halves split after ceil((n // 2) / 32) * 32 rows.
Here they are evaluated from that split rule directly, not by recursing:
* chol / trsm_right: column by column (32 wide).  Column j receives one rounded product per range
  [lo, mid) of ``grouped.column_groups`` (the split tree's left halves to its left); the products are at a
  fixed exponent, so one residue GEMM serves all rows below, and the exact differences commute.  Then the
  diagonal tile is factored (``basecase.chol_tile``) and the rows below are solved against it, by
  substitution on CUDA cores (``basecase.trsv_tile``) or with the tile inverse and `refine` corrections.
* trsm_left: the operation program of ``grouped.solve_program`` (leaves, updates with their per-column
  'col' rounding and aligned differences, rescales of both halves of a node), run on MP row tiles.
* chol_inv: the inverse built over the same split tree, child products at a common ('mat') exponent.
"""
import torch

from . import grouped
from .mpmat import MP, gemm_nt, add, rescale, from_ints, neg
from .basecase import chol_inv_tile, chol_tile, trsv_tile, apply_tile_inverse
from .rns import dev

BT = 32


def fx_exp(L):
    """exponent of the equilibrated fixed-point format (sdpvibe/linalg.py:19)"""
    return -(32 * L - 40)


def _split(n, bt):
    return (n // 2 + bt - 1) // bt * bt


def _ntiles(n, bt):
    """number of diagonal tiles chol() produces for an n x n matrix"""
    return 1 if n <= bt else -(-n // bt)


def _band(W, r0, r1, c0, c1, e):
    return MP(W[:, r0:r1, c0:c1].contiguous(), e)


def _leaf_right(Bj, t, e, leaf, refine):
    """X with X L_jj^T = Bj for a band of rows Bj (fixed point at e)"""
    if leaf == "gemm" and t.X is not None:
        X = gemm_nt(Bj, t.X, out_exp=e)                                      # Bj X_jj^T
        for _ in range(refine):                                              # X + (Bj - X L_jj^T) X_jj^T
            Rr = add(Bj, gemm_nt(X, t.Lmp, out_exp=e), -1, out_exp=e)
            X = add(X, gemm_nt(Rr, t.X, out_exp=e), 1, out_exp=e)
        return X.limbs
    m = Bj.shape[0]
    out, _ = trsv_tile(t, Bj.limbs, torch.full((m,), e, dtype=torch.int64, device=dev), out_exp=e)
    return out


def _columns(W, e, s, tiles, first_row, tree, leaf, refine, factor):
    """The column program on the working copy W (L, rows, 32 tree): rows >= first_row get their updates and
    leaves; with factor, the diagonal tiles are factored on the way (tiles filled in)."""
    rows = W.shape[1]
    for j in range(tree):
        c0, c1 = BT * j, BT * (j + 1)
        r0 = max(c0, first_row)
        for lo, mid in grouped.column_groups(tree, j):
            if r0 >= rows:
                break
            P = gemm_nt(_band(W, r0, rows, BT * lo, BT * mid, e), _band(W, c0, c1, BT * lo, BT * mid, e), out_exp=e)
            W[:, r0:rows, c0:c1] = add(_band(W, r0, rows, c0, c1, e), P, -1, out_exp=e).limbs
        if factor:
            Lt, t = chol_tile(_band(W, c0, c1, c0, c1, e), want_inverse=factor == "inverse")[:2]
            W[:, c0:c1, c0:c1] = Lt.limbs
            tiles.append(t)
        rb = max(c1, first_row)
        if rb < rows:
            W[:, rb:rows, c0:c1] = _leaf_right(_band(W, rb, rows, c0, c1, e), tiles[j], e, leaf, refine)


def chol(A, bt=32, tile_inverses=False, panel_leaf="subst", refine=0):
    """(L, tiles) of an equilibrated fixed-point SPD matrix, n a multiple of bt (sdpvibe/linalg.py:83-96)"""
    n, L = A.shape[0], A.L
    e = fx_exp(L)
    assert bt == BT and n % BT == 0, "pad n to a multiple of the tile size"
    W = A.limbs.clone()
    tiles = []
    _columns(W, e, n // BT, tiles, 0, n // BT, panel_leaf, refine, "inverse" if tile_inverses else "plain")
    s = n // BT
    for i in range(s):                                                       # the factor is lower triangular
        W[:, BT * i:BT * (i + 1), BT * (i + 1):] = 0
    return MP(W, e), tiles


def trsm_right(B, Lf, tiles, bt=32, leaf="subst", refine=0):
    """X with X L^T = B, fixed point (sdpvibe/linalg.py:99-118)"""
    n = Lf.shape[0]
    e = fx_exp(Lf.L)
    m = B.shape[0]
    s = n // BT
    W = torch.zeros((Lf.L, n + m, n), dtype=torch.int32, device=dev)
    W[:, :n] = Lf.limbs
    W[:, n:] = B.limbs
    _columns(W, e, s, list(tiles), n, s, leaf, refine, None)
    return MP(W[:, n:].contiguous(), e)


def trsm(X, B, kc=4096):
    """P = X B with X = L^-1; per-column exponents (sdpvibe/linalg.py:67-70)"""
    Bt = MP(B.limbs.transpose(1, 2).contiguous(), 0)
    return gemm_nt(X, Bt, out_exp="col", kc=kc, bt_rowexp=B.exp)


def _rows_t(P):
    """P (r x m, per-column exponents) as the transposed operand of gemm_nt with its row exponents"""
    return MP(P.limbs.transpose(1, 2).contiguous(), 0), P.exp


def trsm_left(Lf, B, tiles, bt=32, leaf="gemm", refine=0):
    """P = L^-1 B; B (n x m) with per-column exponents, P likewise (sdpvibe/linalg.py:121-138).
    leaf: 'gemm' (explicit tile inverses on the tensor cores) or 'subst' (substitution on CUDA cores)"""
    n, m = B.shape
    s = n // BT
    rows = [MP(B.limbs[:, BT * i:BT * (i + 1)].contiguous(), B.exp) for i in range(s)]
    for op in grouped.solve_program(s, True):
        if op[0] == "leaf":
            j = op[1]
            t = tiles[j]
            if leaf == "gemm" and t.X is not None:
                rows[j] = apply_tile_inverse(t, rows[j], refine)
            else:
                out, ex = trsv_tile(t, rows[j].limbs.transpose(1, 2).contiguous(), rows[j].exp)
                rows[j] = MP(out.transpose(1, 2).contiguous(), ex)
            continue
        _, lo, mid, hi = op
        if op[0] == "upd":
            left = MP(torch.cat([r.limbs for r in rows[lo:mid]], 1), rows[lo].exp)
            Pt, pexp = _rows_t(left)
            U = gemm_nt(_band(Lf.limbs, BT * mid, BT * hi, BT * lo, BT * mid, Lf.uniform_exp()), Pt, out_exp="col",
                        bt_rowexp=pexp)
            Bb = MP(torch.cat([r.limbs for r in rows[mid:hi]], 1), rows[mid].exp)
            D = add(Bb, U, -1, out_exp="align")
            rows[mid:hi] = [MP(D.limbs[:, BT * q:BT * (q + 1)].contiguous(), D.exp) for q in range(hi - mid)]
        else:                                                                # rescale both halves to one exponent
            ee = torch.maximum(rows[lo].exp, rows[mid].exp)
            rows[lo:hi] = [rescale(r, ee) for r in rows[lo:hi]]
    return MP(torch.cat([r.limbs for r in rows], 1), rows[0].exp)


def _stack(tl, tr_, bl, br, L):
    """2 x 2 blocks [[tl, tr_], [bl, br]] (None = zero) at the largest block exponent"""
    parts = [p for p in (tl, tr_, bl, br) if p is not None]
    e = max(p.uniform_exp() for p in parts)
    h = (tl.shape[0], br.shape[0])
    w = (tl.shape[1], br.shape[1])
    out = torch.zeros((L, h[0] + h[1], w[0] + w[1]), dtype=torch.int32, device=dev)
    for p, r, c in ((tl, 0, 0), (tr_, 0, w[0]), (bl, h[0], 0), (br, h[0], w[0])):
        if p is not None:
            out[:, r:r + p.shape[0], c:c + p.shape[1]] = (p if p.uniform_exp() == e else rescale(p, e)).limbs
    return MP(out, e)


def chol_inv(A, bt=32, stats=None):
    """(L, X = L^-1) of an equilibrated fixed-point SPD matrix (sdpvibe/linalg.py:39-64).  For a node of n
    rows split at n1: L21 = A21 X11^T, S = A22 - L21 L21^T at the fixed point, then X21 = -X22 (L21 X11)
    with both products at a common ('mat') exponent; a leaf of fewer than bt rows is padded with the
    fixed-point identity."""
    L = A.L
    e = fx_exp(L)
    assert A.uniform_exp() == e

    def node(M):
        n = M.shape[0]
        if n <= bt:
            if n == bt:
                return chol_inv_tile(M)
            P = torch.zeros((L, bt, bt), dtype=torch.int32, device=dev)
            P[:, :n, :n] = M.limbs
            P[:, torch.arange(n, bt), torch.arange(n, bt)] = from_ints([[1 << (32 * L - 40)]], e, L).limbs[:, 0, :1]
            Lt, Xt = chol_inv_tile(MP(P, e))
            return Lt[:n, :n], Xt[:n, :n]
        n1 = _split(n, bt)
        L11, X11 = node(M[:n1, :n1])
        L21 = gemm_nt(M[n1:, :n1], X11, out_exp=e)
        L22, X22 = node(add(M[n1:, n1:], gemm_nt(L21, L21, out_exp=e), -1, out_exp=e))
        X21 = neg(gemm_nt(X22, gemm_nt(L21, X11.t(), out_exp="mat").t(), out_exp="mat"))
        return _stack(L11, None, L21, L22, L), _stack(X11, None, X21, X22, L)

    return node(A)
