"""Adjoints of the multiprecision building blocks and the objective's sensitivity to the constraint data.
The reference has no counterpart (it has no differentiation); the quantities are defined here.

  gemm_vjp(A, B, G, transA, transB)   C = op(A) op(B):  (dA, dB) = (G op(B)^T, op(A)^T G) mapped back
                                      through the transposes -- two exact-then-rounded residue GEMMs; no
                                      residues are kept from the forward product (they are recomputed)
  chol_solve_vjp(ch, x, gx)           x = S^-1 r with S = L L^T (mpf.Chol):  gr = S^-1 gx with the same
                                      factor (S symmetric), gS = -gr x^T
  objective_sensitivity(solver, dirs) the first-order change of the primal objective c.x + const along
                                      directions (dB_g, dc_g) of the constraint data at the solver's current
                                      iterate, by linear response: d(obj) = sum_g dc_g . x_g
                                      - sum_g x_g^T dB_g y  (the envelope value, exact at an optimal
                                      primal-dual pair, where c - B y = sum A_p Y-pairings).

Everything stays in MPF on the GPU; the scalar results are mpmath numbers on the host.
"""
import numpy as np
import torch

from . import mpf as F
from .mpf import MPF, gemm, add, dot
from .solver import flat_rows, bexpand


def gemm_vjp(A, B, G, transA=False, transB=False):
    """cotangents of A and B for C = op(A) op(B) given the cotangent G of C (all MPF, 2-d or batched)"""
    # dop(A) = G op(B)^T, dop(B) = op(A)^T G; then undo the transposes
    if not transA:
        dA = gemm(G, B, transB=not transB)                       # G op(B)^T
    else:
        dA = gemm(B, G, transA=transB, transB=True)               # (G op(B)^T)^T = op(B) G^T
    if not transB:
        dB = gemm(A, G, transA=not transA)                        # op(A)^T G
    else:
        dB = gemm(G, A, transA=True, transB=transA)               # (op(A)^T G)^T = G^T op(A)
    return dA, dB


def chol_solve_vjp(ch, x, gx):
    """(gr, gS) for x = S^-1 r solved with the factor ch of S: gr = S^-1 gx, gS = -gr x^T"""
    gr = ch.solve(gx)
    gS = -gemm(gr, x, transB=True)
    return gr, gS


def random_directions(sdp, count, seed=1, L=None):
    """count Gaussian directions (dB_g, dc_g) over every chunk's padded data, each scaled to unit norm over
    all chunks jointly (float64 values, exact in MPF); padded entries are zero"""
    rng = np.random.default_rng(seed)
    L = L or sdp.L
    out = []
    for _ in range(count):
        parts = []
        sq = 0.0
        for g in sdp.groups:
            mask = g.xmask.cpu().numpy()                          # (nb, P) live rows
            dB = rng.standard_normal((g.nb, g.P, sdp.N)) * mask[:, :, None]
            dc = rng.standard_normal((g.nb, g.P, 1)) * mask[:, :, None]
            parts.append((dB, dc))
            sq += float((dB * dB).sum() + (dc * dc).sum())
        s = 1.0 / np.sqrt(sq)
        out.append([(F.from_float(dB * s, L), F.from_float(dc * s, L)) for dB, dc in parts])
    return out


def objective_sensitivity(solver, directions):
    """linear response of the primal objective along each direction at the solver's current iterate"""
    res = []
    for d in directions:
        tot = 0
        for gi, (g, (dB, dc)) in enumerate(zip(solver.sdp.groups, d)):
            x = solver.st[gi]["xs"]["x"]                             # (nb, P, 1)
            dBy = gemm(dB, bexpand(solver.y, g.nb))                    # (nb, P, 1) = dB_g y
            tot = tot + dot(dc, x) - dot(dBy, x)
        res.append(tot)
    return res
