"""Per-kernel timing of the multiprecision hot path on one GPU (CUDA events, after warm-up).

  python -m sdpvibe_b200.kernel_bench --kernel syrk --N 274 --K 7000 --L 27 --reps 20
  kernels: residues | align (the Gram chunk's column alignment) | gemm | syrk | crt | mpfgemm | bgemm (--nb stacked blocks) | cholsolve (batched
  Cholesky + solve over uneven blocks) | tiles (--nb 32 x 32 base tiles: factorisation and inverse) |
  solve (mpf.Chol of --nb SPD blocks of size --M, then L^-1 B with B (nb, M, N): per-kernel device time of
  the eager sequence and the time of its CUDA-graph replay)

Inputs are seeded random limb planes / residues of the given shape; rates are algorithmic (the
reference's operation counts: moduli x 4 digit products x 2 ops per multiply-add; decomposition
bytes = limb bytes read + residue bytes written).
"""
import argparse
import json

import numpy as np
import torch


def _events(fn, reps, warmup=3):
    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        fn()
        e.record()
        e.synchronize()
        ts.append(s.elapsed_time(e))
    return ts


def cholsolve_inputs(blocks, nmin, nmax, nrhs, seed=0):
    """SPD blocks A_b = G G^T + n I (G Gaussian, float64, numpy seed), n_b ~ U[nmin, nmax], with nrhs
    right-hand sides U(-1, 1); all values exact float64.  Returns a list of (n, A, B) numpy arrays."""
    rng = np.random.default_rng(seed)
    ns = rng.integers(nmin, nmax + 1, size=blocks)
    out = []
    for n in ns:
        G = rng.standard_normal((n, n))
        A = G @ G.T + n * np.eye(n)
        A = (A + A.T) / 2
        out.append((int(n), A, rng.uniform(-1.0, 1.0, size=(n, nrhs))))
    return out


def cholsolve_buckets(cases, L, bt=32):
    """group blocks by padded size (multiple of bt) as the reference's callers do (one batched Chol per
    size): each block is padded with the identity, its right-hand sides with zero rows.
    Returns [(npad, [block indices], A MPF (nb, npad, npad), B MPF (nb, npad, nrhs))]."""
    from . import mpf
    by = {}
    for i, (n, _, _) in enumerate(cases):
        by.setdefault(max(bt, -(-n // bt) * bt), []).append(i)
    res = []
    for npad in sorted(by):
        idx = by[npad]
        nrhs = cases[idx[0]][2].shape[1]
        A = np.zeros((len(idx), npad, npad))
        B = np.zeros((len(idx), npad, nrhs))
        for q, i in enumerate(idx):
            n, Ai, Bi = cases[i]
            A[q] = np.eye(npad)
            A[q, :n, :n] = Ai
            B[q, :n] = Bi
        res.append((npad, idx, mpf.from_float(A, L), mpf.from_float(B, L)))
    return res


def spd_tile_fx(L, seed=0):
    """one 32 x 32 SPD tile G G^T + 2^30 I (G integer, |g| < 2^20) scaled below 1, in wide fixed point
    (WL = L + 24 words, 32 L fraction bits), entry-major (32, 32, WL) int32"""
    WL, F = L + 24, 32 * L
    rng = np.random.default_rng(seed)
    G = [[int(v) for v in row] for row in rng.integers(-(1 << 20), 1 << 20, size=(32, 32))]
    A = [[sum(G[i][k] * G[j][k] for k in range(32)) + ((1 << 30) if i == j else 0) for j in range(32)]
         for i in range(32)]
    sh = F - (max(A[i][i] for i in range(32)).bit_length() + 1)
    out = np.zeros((32, 32, WL), np.uint32)
    for i in range(32):
        for j in range(32):
            u = (A[i][j] << sh) % (1 << (32 * WL))
            out[i, j] = [(u >> (32 * w)) & 0xffffffff for w in range(WL)]
    return out.view(np.int32)


def _tiles(a):
    from . import _lib
    from .basecase import tile_factor
    WL, LF = a.L + 24, a.L
    W = torch.from_numpy(spd_tile_fx(a.L)).cuda()[None].expand(a.nb, 32, 32, WL).contiguous()
    Lw, X, RINV = tile_factor(W, WL, LF)
    work = W.clone()

    def chol():
        work.copy_(W)
        _lib.call("sdpv_chol_tiles", _lib.ptr(work), _lib.ptr(RINV), a.nb, 32, WL, LF, _lib.stream())
    Xo, scratch = torch.empty_like(Lw), torch.empty_like(Lw)

    def inv():
        _lib.call("sdpv_trinv_tiles", _lib.ptr(Lw), _lib.ptr(RINV), _lib.ptr(Xo), _lib.ptr(scratch), a.nb, 32, WL,
                  LF, _lib.stream())
    tc = _events(chol, a.reps, a.warmup)
    ti = _events(inv, a.reps, a.warmup)
    return dict(nb=a.nb, WL=WL, chol_ms=min(tc), chol_ms_mean=float(np.mean(tc)), trinv_ms=min(ti),
                trinv_ms_mean=float(np.mean(ti)))


def _solve(a):
    from . import _trace, graphs, mpf
    rng = np.random.default_rng(1)
    n, nb, m = a.M, a.nb, a.N
    G = rng.standard_normal((nb, n, n))
    A = mpf.from_float(G @ np.swapaxes(G, 1, 2) + n * np.eye(n), a.L)
    B = mpf.from_float(rng.standard_normal((nb, n, m)), a.L)
    ch = mpf.Chol(A)
    graphs.ENABLED = False
    ch.solve_lower(B)
    torch.cuda.synchronize()
    names = [k for k in _lib_names() if k.startswith("sdpv_")]
    with _trace.Trace(timed=names) as tr:
        t_eager = _events(lambda: ch.solve_lower(B), 1, 0)[0]
    kms = {k: round(sum(tr.kernel_ms(k)), 3) for k in sorted(tr.events, key=lambda k: -sum(tr.kernel_ms(k)))}
    graphs.ENABLED = True
    tg = _events(lambda: ch.solve_lower(B), a.reps, max(2, a.warmup))
    return dict(nb=nb, n=n, m=m, eager_ms=t_eager, graph_ms=min(tg), launches=tr.total_launches,
                launches_by_entry=dict(tr.launches), kernel_ms=kms)


def _lib_names():
    from . import _lib
    return list(_lib._SIGS)


def _cholsolve(a, rng):
    """batched Cholesky + 2 triangular solves (nrhs right-hand sides) over uneven SPD blocks"""
    from . import mpf, _trace
    cases = cholsolve_inputs(a.blocks, a.nmin, a.nmax, a.nrhs)
    buckets = cholsolve_buckets(cases, a.L)

    def step():
        for _, _, A, B in buckets:
            ch = mpf.Chol(A)
            ch.solve(B)

    def chol_only():
        for _, _, A, _ in buckets:
            mpf.Chol(A)
    ts = _events(step, a.reps, a.warmup)
    tc = _events(chol_only, a.reps, a.warmup)
    names = ("sdpv_chol_tiles", "sdpv_trinv_tiles", "sdpv_residues", "sdpv_rns_gemm", "sdpv_crt_block",
             "sdpv_crt_norm", "sdpv_shift_round", "sdpv_add_same", "sdpv_bitlen", "sdpv_badd_align",
             "sdpv_mpf_norm", "sdpv_mpf_mul", "sdpv_mpf_add", "sdpv_top_max", "sdpv_align", "sdpv_align_t",
             "sdpv_align_rows", "sdpv_residues_rows")
    with _trace.Trace(timed=names) as tr:
        step()
        torch.cuda.synchronize()
    kms = {n: round(sum(tr.kernel_ms(n)), 3) for n in names if tr.launches[n]}
    ns = np.array([c[0] for c in cases], dtype=np.float64)
    mac_chol = float((ns ** 3 / 6).sum())
    mac_solve = float((2 * ns ** 2 / 2 * a.nrhs).sum())
    t = min(ts)
    return dict(blocks=a.blocks, nrhs=a.nrhs, buckets={int(b[0]): len(b[1]) for b in buckets},
                ms=t, ms_mean=float(np.mean(ts)), ms_chol=min(tc),
                mp_mac_chol=mac_chol, mp_mac_solve=mac_solve,
                mp_mac_per_s=(mac_chol + mac_solve) / (t * 1e-3),
                launches=tr.total_launches, ms_per_launch=t / max(1, tr.total_launches),
                launches_by_entry=dict(tr.launches), kernel_ms=kms)


def main():
    from .mpmat import lib_ctx
    from . import mpf

    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel", default="syrk", choices=("residues", "align", "gemm", "syrk", "crt", "mpfgemm", "cholsolve",
                                                             "bgemm", "tiles", "solve"))
    ap.add_argument("--nb", type=int, default=1, help="bgemm: number of stacked blocks")
    ap.add_argument("--blocks", type=int, default=600, help="cholsolve: number of SPD blocks")
    ap.add_argument("--nmin", type=int, default=8)
    ap.add_argument("--nmax", type=int, default=160)
    ap.add_argument("--nrhs", type=int, default=8)
    ap.add_argument("--L", type=int, default=27)
    ap.add_argument("--M", type=int, default=274)
    ap.add_argument("--N", type=int, default=274)
    ap.add_argument("--K", type=int, default=7000)
    ap.add_argument("--reps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--packed", action="store_true", help="contiguous residue planes (no channel spreading)")
    a = ap.parse_args()
    dev = "cuda"
    rng = np.random.default_rng(0)
    R = lib_ctx(a.L)
    out = {"kernel": a.kernel, "L": a.L, "M": a.M, "N": a.N, "K": a.K, "n_mod": R.n}
    if a.kernel in ("residues", "gemm", "syrk"):
        X = torch.from_numpy(rng.integers(-(1 << 31), 1 << 31, size=(a.L, a.N, a.K), dtype=np.int64)
                             .astype(np.int32)).to(dev)
        if a.kernel == "residues":
            ts = _events(lambda: R.residues(X, 0, a.K, spread=not a.packed, unsigned=not a.packed), a.reps, a.warmup)
            bytes_ = a.N * a.K * (4 * a.L + 2 * R.n)
            out.update(ms=min(ts), ms_mean=float(np.mean(ts)), gbs=bytes_ / (min(ts) * 1e-3) / 1e9)
        else:
            Ah, Al = R.residues(X, 0, a.K, spread=not a.packed, unsigned=not a.packed)
            if a.kernel == "syrk":
                acc = torch.zeros((R.n, a.N, a.N), dtype=torch.int16, device=dev)
                ts = _events(lambda: R.accumulate(Ah, Al, None, None, acc, syrk=True, unsigned=not a.packed), a.reps,
                             a.warmup)
                ops = R.n * 8 * (a.N * (a.N + 1) // 2) * a.K
            else:
                Y = torch.from_numpy(rng.integers(-(1 << 31), 1 << 31, size=(a.L, a.M, a.K), dtype=np.int64)
                                     .astype(np.int32)).to(dev)
                Bh, Bl = R.residues(Y, 0, a.K, spread=not a.packed, unsigned=not a.packed)
                acc = torch.zeros((R.n, a.M, a.N), dtype=torch.int16, device=dev)
                ts = _events(lambda: R.accumulate(Bh, Bl, Ah, Al, acc, unsigned=not a.packed), a.reps, a.warmup)
                ops = R.n * 8 * a.M * a.N * a.K
            out.update(ms=min(ts), ms_mean=float(np.mean(ts)), tops=ops / (min(ts) * 1e-3) / 1e12)
    elif a.kernel == "align":
        # a Gram chunk: K rows x N columns of (L-1)-limb MPF entries, columns rounded to their top - NB and
        # transposed into L limb planes (sdpv_align_t)
        La = a.L - 1
        mm = rng.integers(-(1 << 31), 1 << 31, size=(La, a.K, a.N), dtype=np.int64).astype(np.int32)
        P = mpf.MPF(torch.from_numpy(mm).to(dev), torch.from_numpy(rng.integers(-8, 9, size=(a.K, a.N))).to(dev))
        target = (mpf.top_max(P, over_rows=True)[0] - mpf.NBITS(La))[None].contiguous()
        ld = -(-a.K // 4) * 4
        ts = _events(lambda: mpf.aligned(P, target, per_col=True, transpose=True, Lout=a.L, ld=ld), a.reps, a.warmup)
        bytes_ = a.N * a.K * (4 * La + 8 + 4 * a.L)
        out.update(ms=min(ts), ms_mean=float(np.mean(ts)), gbs=bytes_ / (min(ts) * 1e-3) / 1e9)
    elif a.kernel == "bgemm":
        # batched residue GEMM of nb stacked blocks (M x K) (N x K), as the Cholesky/trsm recursion issues
        X = torch.from_numpy(rng.integers(-(1 << 31), 1 << 31, size=(a.L, a.nb * a.M, a.K), dtype=np.int64)
                             .astype(np.int32)).to(dev)
        Y = torch.from_numpy(rng.integers(-(1 << 31), 1 << 31, size=(a.L, a.nb * a.N, a.K), dtype=np.int64)
                             .astype(np.int32)).to(dev)
        Ah, Al = R.residues(X, 0, a.K, spread=True, unsigned=True)
        Bh, Bl = R.residues(Y, 0, a.K, spread=True, unsigned=True)
        acc = torch.zeros((R.n, a.nb * a.M, a.N), dtype=torch.int16, device=dev)
        ts = _events(lambda: R.accumulate(Ah, Al, Bh, Bl, acc, nb=a.nb, fresh=True, unsigned=True), a.reps, a.warmup)
        tr = _events(lambda: R.residues(X, 0, a.K, spread=True, unsigned=True), a.reps, a.warmup)
        ops = R.n * 8 * a.nb * a.M * a.N * a.K
        out.update(nb=a.nb, ms=min(ts), ms_mean=float(np.mean(ts)), tops=ops / (min(ts) * 1e-3) / 1e12,
                   items=((a.M + 127) // 128) * ((a.N + 127) // 128) * a.nb * R.n, ms_residues_A=min(tr))
    elif a.kernel == "cholsolve":
        out.update(_cholsolve(a, rng))
    elif a.kernel == "tiles":
        out.update(_tiles(a))
    elif a.kernel == "solve":
        out.update(_solve(a))
    elif a.kernel == "crt":
        m = torch.tensor(R.mods, dtype=torch.int64, device=dev)[:, None, None]
        acc = (torch.randint(0, 1 << 30, (R.n, a.M, a.N), device=dev) % m).to(torch.int16)
        rexp = torch.zeros(a.M, dtype=torch.int64, device=dev)
        cexp = torch.zeros(a.N, dtype=torch.int64, device=dev)
        ts = _events(lambda: R.crt_norm(acc, a.N, 0, a.N, a.M, rexp, cexp, a.L - 1), a.reps, a.warmup)
        tb = _events(lambda: R.crt_block(acc, a.N, 0, a.N, a.M), a.reps, a.warmup)
        out.update(ms=min(ts), ms_mean=float(np.mean(ts)), entries_per_s=a.M * a.N / (min(ts) * 1e-3),
                   ms_block=min(tb), block_entries_per_s=a.M * a.N / (min(tb) * 1e-3))
    else:
        L = a.L

        def rand(shape):
            n = int(np.prod(shape))
            mm = rng.integers(-(1 << 31), 1 << 31, size=(L, n), dtype=np.int64).astype(np.int32)
            mm[-1] = (mm[-1] & ((1 << 29) - 1)) | (1 << 29)
            return mpf.MPF(torch.from_numpy(mm).to(dev).view(L, *shape),
                           torch.from_numpy(rng.integers(-4, 5, size=n)).to(dev).view(*shape))
        A, B = rand((a.M, a.K)), rand((a.K, a.N))
        ts = _events(lambda: mpf.gemm(A, B), a.reps, a.warmup)
        out.update(ms=min(ts), ms_mean=float(np.mean(ts)), mp_mac_per_s=a.M * a.N * a.K / (min(ts) * 1e-3))
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
