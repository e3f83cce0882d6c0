"""Tiled Cholesky factorisation of one large N x N MPF matrix (Q of the solver) with the interface of
``mpf.Chol``: drop-in for ``sdpvibe.blockchol`` (sdpvibe/blockchol.py:1-94).

The factor is defined by the right-looking blocked algorithm over b x b tiles of the lower triangle,

    for k:  D_k = Chol(A_kk);  L_ik = (D_k^-1 A_ik^T)^T (i > k);  A_ij <- A_ij - L_ik L_jk^T (i >= j > k, in k order)

with every product exact then rounded (mpf.gemm) and every difference rounded (mpf.add), so its bits are
fixed by that sequence of rounded operations; it agrees with the monolithic factorisation to working
precision only.  The peak memory is about half of Q plus one column of tiles.  How the operations are
issued is this module's own:
* the panel of step k is one triangular solve: the columns of a solve are independent (per-column
  alignment, exponents and rescaling), so the transposed tiles A_ik^T side by side give each tile's
  columns exactly what a solve of that tile alone gives;
* each panel tile is aligned (one exponent per row) and decomposed into residues once, and the trailing
  update's products L_ik L_jk^T are residue GEMMs of those operands, reconstructed and renormalised by one
  CRT each -- the arithmetic of mpf.gemm(L_ik, L_jk, transB=True), whose row alignment of L_jk as the
  transposed operand is the one it gets as the left operand.
"""
import torch

from .mpf import MPF, Chol, add, gemm, top_max, aligned, _row_exponents
from .mpmat import lib_ctx, KC_MAX


def _block(Q, r0, r1, c0, c1):
    return MPF(Q.m[:, r0:r1, c0:c1].contiguous(), Q.e[r0:r1, c0:c1].contiguous())


def _mirror_lower(A):
    """the symmetric matrix whose lower triangle is A's"""
    n = A.shape[-1]
    low = torch.tril(torch.ones(n, n, dtype=torch.bool, device=A.e.device))
    return MPF(torch.where(low, A.m, A.m.transpose(-1, -2)).contiguous(),
               torch.where(low, A.e, A.e.transpose(-1, -2)).contiguous())


def _cat(parts, dim):
    """MPF matrices side by side (dim 1) or stacked (dim 0)"""
    return MPF(torch.cat([p.m for p in parts], dim + 1), torch.cat([p.e for p in parts], dim))


class _PanelOperand:
    """One panel tile (M x K MPF) with its rows aligned to a common exponent each and decomposed into
    residues once, for all the products it enters."""

    def __init__(self, A):
        L = A.L
        self.M, K = A.shape
        self.R = R = lib_ctx(L)
        self.L = L
        self.rexp = _row_exponents(top_max(A, over_rows=False), L)[0]          # (M,)
        Am = aligned(A, self.rexp[None], per_col=False, transpose=False).view(L, self.M, K)
        self.res = [R.residues(Am, k0, min(KC_MAX, K - k0), spread=True, unsigned=True) for k0 in range(0, K, KC_MAX)]

    def times_t(self, other):
        """self @ other^T, exact and renormalised per entry (mpf.gemm(self, other, transB=True))"""
        R, M, N = self.R, self.M, other.M
        acc = torch.empty((R.n, M, N), dtype=torch.int16, device=self.rexp.device)
        for q, ((ah, al), (bh, bl)) in enumerate(zip(self.res, other.res)):
            R.accumulate(ah, al, bh, bl, acc, fresh=q == 0, unsigned=True)
        Om, Oe = R.crt_norm(acc, N, 0, N, M, self.rexp, other.rexp[None, :], self.L, rows_per_block=M)
        return MPF(Om.view(self.L, M, N), Oe.view(M, N))


class BlockChol:
    """Q = L L^T with L in b x b tiles: diagonal factors D[k] (mpf.Chol) and off-diagonal tiles Lo[i, k]"""

    def __init__(self, holder, b=2048):
        """holder: a list holding Q (MPF (N, N), lower triangle valid); Q is taken out of it so that its
        memory goes as soon as the tiles are cut"""
        Q = holder.pop()
        N = Q.shape[0]
        self.N, self.b, self.L = N, b, Q.L
        self.cuts = cuts = list(range(0, N, b)) + [N]
        self.T = T = len(cuts) - 1
        rest = {(i, j): _block(Q, cuts[i], cuts[i + 1], cuts[j], cuts[j + 1]) for i in range(T) for j in range(i + 1)}
        del Q
        self.D, self.Lo = [], {}
        for k in range(T):
            dk = Chol(_mirror_lower(rest.pop((k, k))))
            self.D.append(dk)
            below = list(range(k + 1, T))
            if not below:
                break
            widths = [cuts[i + 1] - cuts[i] for i in below]
            sol = dk.solve_lower(_cat([rest.pop((i, k)).T for i in below], 1))   # (b_k, sum of panel rows)
            ops = {}
            c0 = 0
            for i, w in zip(below, widths):
                self.Lo[i, k] = MPF(sol.m[:, :, c0:c0 + w], sol.e[:, c0:c0 + w]).T
                ops[i] = _PanelOperand(self.Lo[i, k])
                c0 += w
            for i in below:
                for j in below[:below.index(i) + 1]:
                    rest[i, j] = add(rest[i, j], ops[i].times_t(ops[j]), -1)
            del ops, sol

    def _rows(self, B, k):
        return MPF(B.m[:, self.cuts[k]:self.cuts[k + 1]].contiguous(), B.e[self.cuts[k]:self.cuts[k + 1]].contiguous())

    def solve_lower(self, B):
        """L^-1 B for B: MPF (N, m): forward substitution over the tile rows (differences in column order)"""
        y = []
        for k in range(self.T):
            r = self._rows(B, k)
            for j, yj in enumerate(y):
                r = add(r, gemm(self.Lo[k, j], yj), -1)
            y.append(self.D[k].solve_lower(r))
        return _cat(y, 0)

    def solve_upper(self, Y):
        """L^-T Y: back substitution over the tile rows (differences in increasing row order)"""
        x = [None] * self.T
        for k in range(self.T - 1, -1, -1):
            r = self._rows(Y, k)
            for i in range(k + 1, self.T):
                r = add(r, gemm(self.Lo[i, k], x[i], transA=True), -1)
            x[k] = self.D[k].solve_upper(r)
        return _cat(x, 0)

    def solve(self, B):
        return self.solve_upper(self.solve_lower(B))

    def log2_cond(self):
        """log2 of SDPB's condition estimate (max / min diagonal entry of L)^2 over all diagonal tiles"""
        from .solver import chol_log2_cond_parts
        parts = [chol_log2_cond_parts(dk) for dk in self.D]
        return 2 * (max(h for h, _ in parts) - min(lo for _, lo in parts))
