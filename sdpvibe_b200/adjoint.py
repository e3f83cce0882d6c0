"""Sensitivity of the primal objective to the constraint data (B, c) at a fixed iterate, by hand-written
adjoints of the multiprecision GEMM and of the Schur-complement solve.  The reference has no
differentiation; the quantities are defined here.

The differentiated function.  At a primal-dual iterate (x, X, y, Y) of SDPB's problem
    min c.x  s.t.  X = sum_p A_p x_p >= 0,  B^T x = b          (dual: Tr(A_p Y) + (B y)_p = c_p)
the Newton system of the solver (sdpvibe/solver.py:870-933, with R = beta mu I - X Y) reduces to
    S dx - B dy = rhs,   B^T dx = p,    S_pq = Tr(A_p X^-1 A_q Y) (factor L_S),
    rhs = -(c - Tr(A Y) - B y) - diag(V^T Z V),   p = b - B^T x,
solved as in the solver: P = L_S^-1 B, Q = P^T P, dy = Q^-1 (p - P^T L_S^-1 rhs), dx = L_S^-T (L_S^-1 rhs + P dy).
    f(B, c) = const + c . (x + dx(B, c))
is the primal objective after a full Newton step from the fixed iterate: smooth in (B, c) at any iterate,
and at an optimal, strictly complementary solution its derivative is the envelope value below (the
implicit-function derivative of the optimum).  S and the Z-term do not depend on (B, c).

Its adjoint.  With K = [[S, -B], [B^T, 0]] and z = (dx, dy), c.dz' = lambda^T (dr - dK z) for
K^T lambda = (c, 0); lambda = (u, -v) where (u, v) is the same solve with rhs = c and p = 0:
    v = Q^-1 (-P^T L_S^-1 c),  u = L_S^-T (L_S^-1 c + P v)         (triangular solves with the same factors)
    df = dc . (x + dx - u) + u^T dB (y + dy) + (x + dx)^T dB v
    grad_c = x + dx - u,   grad_B = u (y + dy)^T + (x + dx) v^T   (the GEMM adjoint of C = B W, W = [y+dy, v])
Residues are recomputed in the backward products (none are stored by the forward).  A directional
derivative along (dB, dc) is one GEMM dB [y+dy, v] plus dot products.

The plain linear-response (envelope) value  dc . x - x^T dB y  is computed beside it.

  gemm_vjp, chol_solve_vjp        adjoints of the building blocks
  NewtonObjective(solver, L)      f and its adjoint at the solver's current iterate, at L limbs (L larger than
                                  the solver's widens the iterate and the data exactly: finite differences
                                  at twice the working precision)
  iter_directions(sdp, count)     Gaussian unit directions in (B, c) from one numpy generator
  envelope_sensitivity            the plain linear-response value

  ObjectiveFunction / objective      the same f behind torch.autograd.Function: float64 carrier tensors of the
                                  chunks' (B, c) enter the graph, f comes out as a float64 scalar, and
                                  backward() gives the carriers the adjoint gradient rounded to float64;
                                  the exact MPF gradient stays on the objective (`last_gradient`)

torch's autograd tracks floating-point tensors only and the MPF limb planes are int32, so the exact 832-bit
cotangents travel as MPF payloads beside the float64 graph.  Everything stays in MPF on the GPU; scalar
results are mpmath numbers.
"""
import mpmath as mp
import numpy as np
import torch

from . import mpf as F
from .mpf import MPF, EZ, Chol, gemm, add, dot, symmetrize, total
from .solver import (Solver, SDP, Group, flat_rows, bexpand, masked, add_diag, diag_of, copy_lower_to_upper)


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


# ------------------------------------------------------------------ exact widening to more limbs
def widen(A, L2):
    """the same values with L2 >= L limbs: L2 - L zero low limbs, exponents lowered by 32 (L2 - L)"""
    L = A.L
    assert L2 >= L
    if L2 == L:
        return A
    m = torch.cat([torch.zeros((L2 - L, *A.shape), dtype=torch.int32, device=A.m.device), A.m], 0)
    return MPF(m, torch.where(A.e == EZ, A.e, A.e - 32 * (L2 - L)))


def widen_sdp(sdp, L2):
    """the SDP with every array widened to L2 limbs (same values)"""
    out = SDP.__new__(SDP)
    out.const, out.b, out.N, out.L = sdp.const, widen(sdp.b, L2), sdp.N, L2
    out.total_psd_rows, out.nblocks = sdp.total_psd_rows, sdp.nblocks
    out.groups = []
    for g in sdp.groups:
        h = Group()
        h.__dict__.update(g.__dict__)
        h.c, h.B = widen(g.c, L2), widen(g.B, L2)
        h.V = {k: [widen(v, L2) for v in vs] for k, vs in g.V.items()}
        out.groups.append(h)
    return out


def _hcat(*cols):
    """MPF arrays (..., n, 1) side by side -> (..., n, k)"""
    return MPF(torch.cat([c.m for c in cols], -1), torch.cat([c.e for c in cols], -1))


def _col(A, j):
    return MPF(A.m[..., j:j + 1].contiguous(), A.e[..., j:j + 1].contiguous())


class _Prec:
    """mpmath working precision for L limbs inside a with-block"""

    def __init__(self, L):
        self.bits = F.NBITS(L) + 64

    def __enter__(self):
        self.old = mp.mp.prec
        mp.mp.prec = max(self.old, self.bits)

    def __exit__(self, *a):
        mp.mp.prec = self.old


class NewtonObjective:
    """f(B, c) = const + c . (x + dx(B, c)) at the solver's current iterate, with its adjoint.

    forward(Bs, cs) evaluates f at per-chunk data (default: the SDP's own) and keeps the factors;
    backward() returns (grad_B, grad_c) per chunk at that data; directional(dBs, dcs) the derivative
    along a direction together with the envelope value."""

    def __init__(self, solver, L=None, beta=0):
        L = L or solver.L
        self.L, self.beta = L, beta
        with _Prec(L):
            if L == solver.L:
                view, sdp = solver, solver.sdp
            else:
                sdp = widen_sdp(solver.sdp, L)
                view = Solver.__new__(Solver)
                view.sdp, view.L, view.p = sdp, L, solver.p
                view.S = lambda v: F.scalar(v, L)
            self.sdp = sdp
            self.y = widen(solver.y, L)
            it = []
            musum = mp.mpf(0)
            for gi, g in enumerate(sdp.groups):
                xs = solver.st[gi]["xs"]
                x, X, Y = widen(xs["x"], L), widen(xs["X"][0], L), widen(xs["Y"][0], L)
                mk2 = g.Xmask[0][:, :, None] & g.Xmask[0][:, None, :]
                mXY = masked(-gemm(X, Y), mk2)
                musum += total(diag_of(mXY))
                it.append((g, x, X, Y, mk2, mXY))
            mu = -musum / sdp.total_psd_rows
            self.parts = []
            for g, x, X, Y, mk2, mXY in it:
                cX = Chol(X)
                AXI, AY = view.pairings(g, g.V, [cX], [Y])
                cs = Chol(view.schur(g, AXI, AY))
                ayd = view.seg_diag(g, AY, [g.K])                    # Tr(A_p Y)
                Pres = masked(add(view.cmws(g, g.V, x)[0], X, -1), mk2)
                Rb = mXY if not beta else add_diag(mXY, view.S(mp.mpf(beta) * mu), g.Xmask[0])
                Z = symmetrize(cX.solve(add(gemm(Pres, Y), Rb, -1)))
                Vx = g.V["Vx"][0]
                tz = view.seg_diag(g, [gemm(Vx, gemm(Z, Vx), transA=True)], [g.K])
                self.parts.append(dict(g=g, x=x, cs=cs, ayd=ayd, tz=tz))
        self._fw = None

    def forward(self, Bs=None, cs=None):
        sdp, y = self.sdp, self.y
        G = sdp.groups
        Bs = Bs or [g.B for g in G]
        cs = cs or [g.c for g in G]
        with _Prec(self.L):
            pvec, Q, sol = sdp.b, None, []
            for pt, B, c in zip(self.parts, Bs, cs):
                g, ch = pt["g"], pt["cs"]
                By = gemm(B, bexpand(y, g.nb))
                dres = add(add(-pt["ayd"], By, -1), c)
                pvec = add(pvec, gemm(flat_rows(B), flat_rows(pt["x"]), transA=True), -1)
                P = ch.solve_lower(B)
                w = ch.solve_lower(add(-dres, pt["tz"], -1))
                q = gemm(flat_rows(P), flat_rows(P), transA=True)
                Q = q if Q is None else add(Q, q)
                sol.append((P, w))
            dy = pvec
            for P, w in sol:
                dy = add(dy, gemm(flat_rows(P), flat_rows(w), transA=True), -1)
            cholQ = Chol(copy_lower_to_upper(Q))
            del Q
            dy = cholQ.solve(dy)
            f, xn = mp.mpf(sdp.const), []
            for pt, (P, w), c in zip(self.parts, sol, cs):
                g = pt["g"]
                dx = pt["cs"].solve_upper(add(w, gemm(P, bexpand(dy, g.nb))))
                xn.append(add(pt["x"], dx))
                f += dot(c, xn[-1])
        self._fw = dict(Bs=Bs, cs=cs, P=[s[0] for s in sol], cholQ=cholQ, dy=dy, xn=xn)
        self._adj = None
        return f

    def _adjoint(self):
        """(u per chunk, v) of K^T lambda = (c, 0), lambda = (u, -v)"""
        if self._adj is None:
            fw = self._fw
            assert fw is not None, "forward() first"
            with _Prec(self.L):
                r, ws = None, []
                for pt, P, c in zip(self.parts, fw["P"], fw["cs"]):
                    w = pt["cs"].solve_lower(c)
                    ws.append(w)
                    t = gemm(flat_rows(P), flat_rows(w), transA=True)
                    r = t if r is None else add(r, t)
                v = fw["cholQ"].solve(-r)
                us = [pt["cs"].solve_upper(add(w, gemm(P, bexpand(v, pt["g"].nb))))
                      for pt, P, w in zip(self.parts, fw["P"], ws)]
                self._adj = dict(u=us, v=v, W=_hcat(add(self.y, fw["dy"]), v, self.y))
        return self._adj

    def backward(self):
        """[(grad_B_g, grad_c_g)] at the last forward's data"""
        fw, ad = self._fw, self._adjoint()
        out = []
        with _Prec(self.L):
            W2 = _hcat(_col(ad["W"], 0), _col(ad["W"], 1))                  # [y + dy, v]
            for pt, B, u, xn in zip(self.parts, fw["Bs"], ad["u"], fw["xn"]):
                nb = pt["g"].nb
                gB, _ = gemm_vjp(B, bexpand(W2, nb), _hcat(u, xn))            # u (y+dy)^T + (x+dx) v^T
                out.append((gB, add(xn, u, -1)))
        return out

    def directional(self, dBs, dcs):
        """(adjoint derivative of f, envelope value) along the direction (dB_g, dc_g) per chunk"""
        fw, ad = self._fw, self._adjoint()
        da, de = mp.mpf(0), mp.mpf(0)
        with _Prec(self.L):
            for pt, dB, dc, u, xn in zip(self.parts, dBs, dcs, ad["u"], fw["xn"]):
                x = pt["x"]
                T = gemm(dB, bexpand(ad["W"], pt["g"].nb))                  # dB [y + dy, v, y]
                da += dot(dc, add(xn, u, -1)) + dot(u, _col(T, 0)) + dot(xn, _col(T, 1))
                de += dot(dc, x) - dot(x, _col(T, 2))
        return da, de


def iter_directions(sdp, count, seed=1, L=None, host=False):
    """count Gaussian directions [(dB_g, dc_g) per chunk] from one numpy generator, each scaled to unit
    norm over all chunks jointly (float64 values, exact in MPF); padded entries are zero.  Yields one
    direction at a time (a direction is as large as B); host=True yields the float64 arrays instead."""
    rng = np.random.default_rng(seed)
    L = L or sdp.L
    for _ in range(count):
        parts, sq = [], 0.0
        for g in sdp.groups:
            mask = g.xmask.cpu().numpy()                          # (nb, P) live rows
            dB = rng.standard_normal((g.nb, g.P, sdp.N)) * mask[:, :, None]
            dc = rng.standard_normal((g.nb, g.P, 1)) * mask[:, :, None]
            parts.append((dB, dc))
            sq += float((dB * dB).sum() + (dc * dc).sum())
        s = 1.0 / np.sqrt(sq)
        parts = [(dB * s, dc * s) for dB, dc in parts]
        yield parts if host else direction_to_mpf(parts, L)


def direction_to_mpf(parts, L):
    """host float64 direction [(dB_g, dc_g)] -> MPF on the device (exact)"""
    return [(F.from_float(dB, L), F.from_float(dc, L)) for dB, dc in parts]


def random_directions(sdp, count, seed=1, L=None):
    return list(iter_directions(sdp, count, seed, L))


def envelope_sensitivity(solver, directions):
    """plain linear response sum_g dc_g . x_g - x_g^T dB_g y at the solver's current iterate, per direction"""
    res = []
    for d in directions:
        tot = 0
        for gi, (g, (dB, dc)) in enumerate(zip(solver.sdp.groups, d)):
            x = solver.st[gi]["xs"]["x"]                             # (nb, P, 1)
            dBy = gemm(dB, bexpand(solver.y, g.nb))                    # (nb, P, 1) = dB_g y
            tot = tot + dot(dc, x) - dot(dBy, x)
        res.append(tot)
    return res


class ObjectiveFunction(torch.autograd.Function):
    """f(B, c) of a NewtonObjective in torch's autograd.  Inputs: the objective, then per chunk float64
    carriers (B_g (nb, P, N), c_g (nb, P, 1)) -- their values are not read: f is evaluated exactly at the
    objective's MPF data.  Output: f rounded to float64.  Backward: grad_out times the adjoint gradient
    (grad_B, grad_c) of every chunk, rounded to float64 from the exact MPF values, which are kept on the
    objective as `last_gradient`."""

    @staticmethod
    def forward(ctx, fo, *carriers):
        f = fo.forward()
        ctx.fo = fo
        ctx.n = len(carriers)
        ctx.dev = carriers[0].device if carriers else torch.device("cuda")
        return torch.tensor(float(f), dtype=torch.float64, device=ctx.dev)

    @staticmethod
    def backward(ctx, gout):
        grads = ctx.fo.backward()
        ctx.fo.last_gradient = grads
        out = [None]
        for gB, gc in grads:
            for G in (gB, gc):
                out.append(gout * torch.from_numpy(np.ascontiguousarray(G.to_float())).to(ctx.dev))
        return tuple(out[:ctx.n + 1])


def objective(fo, carriers):
    """f as a float64 tensor in torch's graph: carriers = [(B_g, c_g)] float64 tensors (requires_grad)"""
    flat = [t for pair in carriers for t in pair]
    return ObjectiveFunction.apply(fo, *flat)
