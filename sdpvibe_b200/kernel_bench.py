"""Per-kernel timing of the multiprecision hot path on one GPU (CUDA events, after warm-up).

  python -m sdpvibe_b200.kernel_bench --kernel syrk --N 274 --K 7000 --L 27 --reps 20
  kernels: residues | gemm | syrk | crt | mpfgemm

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


def main():
    from .mpmat import ctx
    from . import mpf

    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel", default="syrk", choices=("residues", "gemm", "syrk", "crt", "mpfgemm"))
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
    R = ctx(a.L)
    out = {"kernel": a.kernel, "L": a.L, "M": a.M, "N": a.N, "K": a.K, "n_mod": R.n}
    if a.kernel in ("residues", "gemm", "syrk"):
        X = torch.from_numpy(rng.integers(-(1 << 31), 1 << 31, size=(a.L, a.N, a.K), dtype=np.int64)
                             .astype(np.int32)).to(dev)
        if a.kernel == "residues":
            ts = _events(lambda: R.residues(X, 0, a.K, spread=not a.packed), a.reps, a.warmup)
            bytes_ = a.N * a.K * (4 * a.L + 2 * R.n)
            out.update(ms=min(ts), ms_mean=float(np.mean(ts)), gbs=bytes_ / (min(ts) * 1e-3) / 1e9)
        else:
            Ah, Al = R.residues(X, 0, a.K, spread=not a.packed)
            if a.kernel == "syrk":
                acc = torch.zeros((R.n, a.N, a.N), dtype=torch.int16, device=dev)
                ts = _events(lambda: R.accumulate(Ah, Al, None, None, acc, syrk=True), a.reps, a.warmup)
                ops = R.n * 8 * (a.N * (a.N + 1) // 2) * a.K
            else:
                Y = torch.from_numpy(rng.integers(-(1 << 31), 1 << 31, size=(a.L, a.M, a.K), dtype=np.int64)
                                     .astype(np.int32)).to(dev)
                Bh, Bl = R.residues(Y, 0, a.K, spread=not a.packed)
                acc = torch.zeros((R.n, a.M, a.N), dtype=torch.int16, device=dev)
                ts = _events(lambda: R.accumulate(Bh, Bl, Ah, Al, acc), a.reps, a.warmup)
                ops = R.n * 8 * a.M * a.N * a.K
            out.update(ms=min(ts), ms_mean=float(np.mean(ts)), tops=ops / (min(ts) * 1e-3) / 1e12)
    elif a.kernel == "crt":
        m = torch.tensor(R.mods, dtype=torch.int64, device=dev)[:, None, None]
        acc = (torch.randint(0, 1 << 30, (R.n, a.M, a.N), device=dev) % m).to(torch.int16)
        rexp = torch.zeros(a.M, dtype=torch.int64, device=dev)
        cexp = torch.zeros(a.N, dtype=torch.int64, device=dev)
        ts = _events(lambda: R.crt_norm(acc, a.N, 0, a.N, a.M, rexp, cexp, a.L - 1), a.reps, a.warmup)
        out.update(ms=min(ts), ms_mean=float(np.mean(ts)), entries_per_s=a.M * a.N / (min(ts) * 1e-3))
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
