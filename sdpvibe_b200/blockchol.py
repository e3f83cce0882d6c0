"""Tiled Cholesky factorisation of one large N x N MPF matrix (Q of the solver) with the interface of
``mpf.Chol`` (drop-in for ``sdpvibe.blockchol``, sdpvibe/blockchol.py:1-94).

The monolithic ``mpf.Chol`` needs about 9 N^2 MPF entries at its peak (fixed-point copy, padding,
recursion); the tiled form keeps the lower triangle as b x b tiles and factorises right-looking,

    for k:  L_kk = chol(A_kk);  L_ik = (L_kk^-1 A_ik^T)^T  (i > k);  A_ij -= L_ik L_jk^T  (i >= j > k),

overwriting tiles as it goes (peak about N^2 / 2 + O(b N) entries).  Every step is one of the exact
primitives (``Chol`` of a tile, its triangular solves, ``gemm``, ``add``) in the reference's order, so
the factor and the solves are the reference's bit for bit; they agree with the monolithic factorisation
to working precision only (a different rounding order).
"""
import torch

from .mpf import MPF, Chol, gemm, add


def _block(Q, r0, r1, c0, c1):
    return MPF(Q.m[:, r0:r1, c0:c1].contiguous(), Q.e[r0:r1, c0:c1].contiguous())


def _mirror_lower(A):
    """the symmetric matrix whose lower triangle is A's"""
    n = A.shape[-1]
    low = torch.tril(torch.ones(n, n, dtype=torch.bool, device=A.e.device))
    return MPF(torch.where(low, A.m, A.m.transpose(-1, -2)).contiguous(),
               torch.where(low, A.e, A.e.transpose(-1, -2)).contiguous())


def _rows(B, r0, r1):
    return MPF(B.m[:, r0:r1].contiguous(), B.e[r0:r1].contiguous())


def _stack_rows(parts):
    return MPF(torch.cat([p.m for p in parts], 1), torch.cat([p.e for p in parts], 0))


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
        A = {(i, j): _block(Q, cuts[i], cuts[i + 1], cuts[j], cuts[j + 1]) for i in range(T) for j in range(i + 1)}
        del Q
        self.D = []
        for k in range(T):
            ck = Chol(_mirror_lower(A.pop((k, k))))
            self.D.append(ck)
            for i in range(k + 1, T):
                A[i, k] = ck.solve_lower(A[i, k].T).T
            for i in range(k + 1, T):
                for j in range(k + 1, i + 1):
                    A[i, j] = add(A[i, j], gemm(A[i, k], A[j, k], transB=True), -1)
        self.Lo = A

    def solve_lower(self, B):
        """L^-1 B for B: MPF (N, m)"""
        y = []
        for k in range(self.T):
            r = _rows(B, self.cuts[k], self.cuts[k + 1])
            for j in range(k):
                r = add(r, gemm(self.Lo[k, j], y[j]), -1)
            y.append(self.D[k].solve_lower(r))
        return _stack_rows(y)

    def solve_upper(self, Y):
        """L^-T Y"""
        x = [None] * self.T
        for k in reversed(range(self.T)):
            r = _rows(Y, self.cuts[k], self.cuts[k + 1])
            for i in range(k + 1, self.T):
                r = add(r, gemm(self.Lo[i, k], x[i], transA=True), -1)
            x[k] = self.D[k].solve_upper(r)
        return _stack_rows(x)

    def solve(self, B):
        return self.solve_upper(self.solve_lower(B))

    def log2_cond(self):
        """log2 of SDPB's condition estimate (max / min diagonal entry of L)^2 over all diagonal tiles"""
        from .solver import chol_log2_cond_parts
        parts = [chol_log2_cond_parts(ck) for ck in self.D]
        return 2 * (max(h for h, _ in parts) - min(lo for _, lo in parts))
