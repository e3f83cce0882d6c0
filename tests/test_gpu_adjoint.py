"""Adjoints of the multiprecision building blocks and the objective sensitivity (sdpvibe_b200.adjoint; no
counterpart in the reference): the GEMM vector-Jacobian products satisfy <G, dA B> = <gemm_vjp_A, dA> to
working precision; the Cholesky-solve adjoint matches central finite differences; the derivative of the
objective after a Newton step, by its adjoint at working precision, agrees with central finite
differences taken at twice the precision to at least 40 digits; the envelope value equals its defining
formula evaluated in mpmath."""
import mpmath as mp
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rand(rng, shape, L, lo=-3, hi=3):
    from sdpvibe_b200.solver import _rand_host_mpf, _host_mpf
    return _host_mpf(_rand_host_mpf(rng, shape, L, spread=hi), L)


def _inner(A, B):
    a, b = A.to_mp().reshape(-1), B.to_mp().reshape(-1)
    return mp.fsum(x * y for x, y in zip(a, b))


@pytest.mark.parametrize("tA,tB", [(False, False), (True, False), (False, True), (True, True)])
def test_gemm_vjp_identity(tA, tB):
    from sdpvibe_b200.adjoint import gemm_vjp
    from sdpvibe_b200.mpf import gemm
    L = 8
    mp.mp.prec = 32 * L + 64
    rng = np.random.default_rng(int(tA) * 2 + int(tB))
    M, K, N = 6, 9, 5
    A = _rand(rng, (K, M) if tA else (M, K), L)
    B = _rand(rng, (N, K) if tB else (K, N), L)
    G = _rand(rng, (M, N), L)
    dA = _rand(rng, A.shape, L)
    dB = _rand(rng, B.shape, L)
    gA, gB = gemm_vjp(A, B, G, tA, tB)
    assert gA.shape == A.shape and gB.shape == B.shape
    lhsA = _inner(G, gemm(dA, B, tA, tB))
    lhsB = _inner(G, gemm(A, dB, tA, tB))
    for lhs, rhs in ((lhsA, _inner(gA, dA)), (lhsB, _inner(gB, dB))):
        assert abs(lhs - rhs) <= mp.mpf(2) ** -(32 * L - 20) * (abs(lhs) + 1)


def test_chol_solve_vjp_central_differences():
    from sdpvibe_b200.adjoint import chol_solve_vjp
    from sdpvibe_b200.mpf import MPF, Chol, add, from_float, gemm
    L = 26
    mp.mp.prec = 32 * L + 64
    rng = np.random.default_rng(3)
    nb, n, m = 2, 40, 3
    G = rng.standard_normal((nb, n, n))
    S = from_float(G @ np.swapaxes(G, 1, 2) + n * np.eye(n), L)
    r = from_float(rng.standard_normal((nb, n, m)), L)
    gx = from_float(rng.standard_normal((nb, n, m)), L)
    D = rng.standard_normal((nb, n, n))
    dS = from_float((D + np.swapaxes(D, 1, 2)) / 2, L)
    dr = from_float(rng.standard_normal((nb, n, m)), L)
    ch = Chol(S)
    x = ch.solve(r)
    gr, gS = chol_solve_vjp(ch, x, gx)
    h = 2 ** -120

    def obj(Sm, rm):
        return _inner(gx, Chol(Sm).solve(rm))
    fd_S = (obj(add(S, dS.shift(-120)), r) - obj(add(S, dS.shift(-120), -1), r)) / (2 * mp.mpf(h))
    fd_r = (obj(S, add(r, dr.shift(-120))) - obj(S, add(r, dr.shift(-120), -1))) / (2 * mp.mpf(h))
    for fd, an in ((fd_S, _inner(gS, dS)), (fd_r, _inner(gr, dr))):
        assert abs(fd - an) <= mp.mpf(2) ** -200 * (abs(an) + 1), (float(fd), float(an))


def test_envelope_sensitivity_formula():
    from conftest import golden
    from test_gpu_solver import _sdp_from_fixture
    from sdpvibe_b200.adjoint import envelope_sensitivity, random_directions
    from sdpvibe_b200.solver import Solver
    g = golden("solver_tiny")
    sdp, L = _sdp_from_fixture(g)
    sol = Solver(sdp, L)
    sol.run(max_iter=2)
    dirs = random_directions(sdp, 3, seed=1)
    got = envelope_sensitivity(sol, dirs)
    y = sol.y.to_mp().reshape(-1)
    for d, v in zip(dirs, got):
        ref = mp.mpf(0)
        for gi, (dB, dc) in enumerate(d):
            x = sol.st[gi]["xs"]["x"].to_mp()
            B = dB.to_mp()
            c = dc.to_mp()
            for b in range(x.shape[0]):
                for p in range(x.shape[1]):
                    ref += c[b, p, 0] * x[b, p, 0] - x[b, p, 0] * mp.fsum(B[b, p, k] * y[k] for k in range(len(y)))
        assert abs(v - ref) <= mp.mpf(2) ** -(32 * L - 40) * (abs(ref) + 1)


def test_newton_objective_adjoint_vs_finite_differences():
    """f(B, c) = c.(x + dx) at the iterate of 4 solver iterations (L = 16, 510 bits): the adjoint's
    directional derivatives against central differences at L = 32 with h = 2^-250 (truncation ~2^-500),
    along 3 Gaussian unit directions; the materialised gradient (GEMM adjoint) gives the same numbers"""
    from sdpvibe_b200.adjoint import NewtonObjective, iter_directions, widen, envelope_sensitivity
    from sdpvibe_b200.mpf import add, dot
    from sdpvibe_b200.solver import Solver
    from sdpvibe_b200.synthetic import ising_like_sdp
    L, L2, k = 16, 32, 250
    sdp, _ = ising_like_sdp(L, nblocks=10, N=20)
    sol = Solver(sdp, L)
    sol.run(max_iter=4)
    fo = NewtonObjective(sol)
    f0 = fo.forward()
    grads = fo.backward()
    hi = NewtonObjective(sol, L=L2)
    assert abs(hi.forward() - f0) <= mp.mpf(10) ** -60 * abs(f0)                  # the same function
    mp.mp.prec = 32 * L2 + 64
    worst = mp.inf
    for d in iter_directions(sdp, 3, seed=1):
        da, de = fo.directional([dB for dB, _ in d], [dc for _, dc in d])
        assert abs(de - envelope_sensitivity(sol, [d])[0]) <= mp.mpf(2) ** -(32 * L - 40) * (abs(de) + 1)
        dg = sum(dot(gB, dB) + dot(gc, dc) for (gB, gc), (dB, dc) in zip(grads, d))
        assert abs(dg - da) <= mp.mpf(2) ** -(32 * L - 60) * (abs(da) + 1)
        wd = [(widen(dB, L2).shift(-k), widen(dc, L2).shift(-k)) for dB, dc in d]
        fp = hi.forward([add(g.B, dB) for g, (dB, _) in zip(hi.sdp.groups, wd)],
                        [add(g.c, dc) for g, (_, dc) in zip(hi.sdp.groups, wd)])
        fm = hi.forward([add(g.B, dB, -1) for g, (dB, _) in zip(hi.sdp.groups, wd)],
                        [add(g.c, dc, -1) for g, (_, dc) in zip(hi.sdp.groups, wd)])
        fd = (fp - fm) * mp.mpf(2) ** (k - 1)
        digits = -mp.log10(abs(da - fd) / abs(fd)) if da != fd else mp.inf
        worst = min(worst, digits)
    assert worst >= 40, float(worst)


def _strictly_feasible_sdp(L, seed=5):
    """a small SDP (dims 1, 1, 2; N = 4) with a strictly feasible primal point (x0: 1 on the diagonal pair
    segments, so X0 = sum_k v_k v_k^T per diagonal block > 0) and dual point (Y0 = I, y0 Gaussian):
    c = Tr(A_p I) + B y0, b = B^T x0.  It has an optimal primal-dual pair with zero gap."""
    from sdpvibe_b200.mpf import add, from_float, gemm, zeros
    from sdpvibe_b200.solver import SDP, Solver, bexpand, flat_rows
    rng = np.random.default_rng(seed)
    N = 4
    blocks = []
    for dim, K, he, ho in ((1, 6, 3, 2), (1, 5, 3, 2), (2, 4, 2, 2)):
        npair = dim * (dim + 1) // 2
        blocks.append(dict(dim=dim, K=K, Ve=rng.standard_normal((he, K)), Vo=rng.standard_normal((ho, K)),
                           c=np.zeros((K * npair, 1)), B=rng.standard_normal((K * npair, N))))
    sdp = SDP(blocks, np.zeros((N, 1)), 0, L)
    helper = Solver(sdp, L)
    y0 = from_float(rng.standard_normal((N, 1)), L)
    b = None
    for g in sdp.groups:
        Vx = g.V["Vx"][0]
        ayd = helper.seg_diag(g, [gemm(Vx, Vx, transA=True)], [g.K])          # Tr(A_p I)
        g.c = add(ayd, gemm(g.B, bexpand(y0, g.nb)))
        x0 = np.zeros((g.nb, g.P, 1))
        for c, r, off in helper.segments(g):
            if c == r:
                x0[:, off:off + g.K, 0] = 1.0
        x0 = from_float(x0 * g.xmask.cpu().numpy()[:, :, None], L)
        t = gemm(flat_rows(g.B), flat_rows(x0), transA=True)
        b = t if b is None else add(b, t)
    sdp.b = b
    return sdp


def test_newton_objective_derivative_is_envelope_value_at_optimum():
    """at an optimal primal-dual pair (gap < 1e-30) the adjoint derivative of f = c.(x + dx) equals the
    plain linear-response value dc.x - x^T dB y (the derivative of the optimal value), and f equals the
    primal objective"""
    from sdpvibe_b200.adjoint import NewtonObjective, iter_directions
    from sdpvibe_b200.solver import Solver
    L = 12
    sdp = _strictly_feasible_sdp(L)
    sol = Solver(sdp, L, maxIterations=300)
    res = sol.run()
    assert res["terminateReason"] == "found primal-dual optimal solution", res["terminateReason"]
    fo = NewtonObjective(sol)
    f0 = fo.forward()
    pobj = res["primalObjective"]
    assert abs(f0 - pobj) <= mp.mpf(10) ** -25 * (abs(pobj) + 1)
    for d in iter_directions(sdp, 3, seed=1):
        da, de = fo.directional([dB for dB, _ in d], [dc for _, dc in d])
        assert abs(da - de) <= mp.mpf(10) ** -12 * abs(de), (mp.nstr(da, 20), mp.nstr(de, 20))


def test_objective_behind_autograd_function():
    """f through torch.autograd: backward() gives the float64 carriers the adjoint gradient; its directional
    derivative matches the exact adjoint's to float64 accuracy, and the exact MPF gradient is kept."""
    import torch
    from sdpvibe_b200.adjoint import NewtonObjective, iter_directions, objective
    from sdpvibe_b200.solver import Solver
    from sdpvibe_b200.synthetic import ising_like_sdp
    L = 16
    sdp, _ = ising_like_sdp(L, nblocks=10, N=20)
    sol = Solver(sdp, L)
    sol.run(max_iter=3)
    fo = NewtonObjective(sol)
    carriers = [(torch.from_numpy(g.B.to_float()).cuda().requires_grad_(),
                 torch.from_numpy(g.c.to_float()).cuda().requires_grad_()) for g in sdp.groups]
    f = objective(fo, carriers)
    assert abs(float(f) - float(fo.forward())) <= 1e-12 * abs(float(f))
    f.backward()
    host = next(iter_directions(sdp, 1, seed=3, host=True))
    dev = next(iter_directions(sdp, 1, seed=3))
    lin = sum(float((B.grad.cpu().numpy() * dB).sum() + (c.grad.cpu().numpy() * dc).sum())
              for (B, c), (dB, dc) in zip(carriers, host))
    exact, _ = fo.directional(*zip(*dev))
    assert abs(lin - float(exact)) <= 1e-9 * (abs(float(exact)) + 1e-30)
    assert len(fo.last_gradient) == len(sdp.groups)
