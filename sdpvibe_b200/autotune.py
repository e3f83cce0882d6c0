"""Offline autotuner of the launch-shape knobs (sdpv_tune_set): it times every candidate value on the
shapes the workloads issue and writes the fastest into ``tuning_b200.json`` beside this module, which the
library applies when it loads (``apply``).  The knobs only decide how work is cut into launches and work
items; every choice gives the same bits.

    python -m sdpvibe_b200.autotune [--reps 5]      (on the GPU the table is for)

Knobs and their shapes:
  crt_ctas    CTAs per SM of the CRT: crt_block of the triangular solves' products (90 x 32 x 1000
              entries), crt_norm of the Gram step (274 x 274)
  narrow_max  short-side limit of the narrow residue-GEMM items: the solves' block products
              (90 x 32 x 1000, K 32; 30 x 64 x 1000, K 64; 131 x 96 x 8, K 64)
  pack_max    block size limit for packing small blocks into one GEMM tile: the Cholesky recursion of
              the c2 buckets (106 x 32 x 32, K 32; 131 x 64 x 32, K 64; 98 x 16 x 16, K 16)
  res_warps   reducer warps of the decomposition kernel: the Gram chunk's residues (274 x 7000 entries,
              L + 1 = 27 limbs, unsigned digits) and the solver's (1000 x 1000, L = 26, API digits)
  moduli_group  the prime split: the library's own contexts take the least multiple of G primes with
              M > 4 kmax 2^(2(32 L - 1)) (sdpvibe/rns.py:166-173 with G = 16): at L = 26, 128 / 120 / 116 /
              113 moduli for G = 16 / 8 / 4 / 1.  Every product is exact whatever the moduli, so the rounded
              results are the same bits; the work of the decomposition, the residue GEMMs and the CRT
              scales with the count.  Timed on an mp GEMM (512^3), a grouped Cholesky + solve of 60
              uneven blocks and a Gram chunk (274 columns, 1750 rows); RNS(L) built by a caller keeps the
              reference's G = 16 and its residue format.

The digit split of a residue (r = 128 hi + lo, two int8 digits) is fixed by the int8 operands of the tensor
cores: every split into two digits below 256 has the same products and bounds.  The residue GEMM's 128 x 128
tile, its 3-stage ring and its single-CTA MMA are fixed by shared memory (three 64 KB stages) and TMEM (384
accumulator columns per tile); a two-CTA (cta_group::2) variant is not built.
"""
import argparse
import json
import os

import numpy as np
import torch

from . import _lib

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning_b200.json")
KNOBS = {"crt_ctas": (0, [1, 2, 3, 4]), "narrow_max": (1, [0, 32, 48, 64]), "pack_max": (2, [0, 32, 64]),
         "res_warps": (3, [8, 16]), "moduli_group": (4, [16, 8, 4, 1])}


def set_knob(name, value):
    _lib.call("sdpv_tune_set", KNOBS[name][0], int(value))


def get_knob(name):
    import ctypes
    v = ctypes.c_int(0)
    _lib.check(_lib.lib().sdpv_tune_get(KNOBS[name][0], ctypes.byref(v)), "sdpv_tune_get")
    return v.value


def apply(path=TABLE):
    """set the knobs from a table written by this tuner on the same GPU model (silently keeps the defaults
    when there is none)"""
    if not os.path.exists(path) or not torch.cuda.is_available():
        return None
    with open(path) as f:
        table = json.load(f)
    if table.get("device") != torch.cuda.get_device_name():
        return None
    for name, value in table["knobs"].items():
        if name in KNOBS:
            set_knob(name, value)
    return table["knobs"]


def _time(fn, reps):
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        fn()
        b.record()
        b.synchronize()
        ts.append(a.elapsed_time(b))
    return float(np.median(ts))


def _gemm_case(R, nb, M, N, K, rng):
    def res(rows):
        m = torch.tensor(R.mods, dtype=torch.int64)[:, None, None]
        r = torch.from_numpy(rng.integers(0, 1 << 30, size=(R.n, rows, K))) % m
        r = torch.where(r > m // 2, r - m, r)
        lo = ((r + 64) & 127) - 64
        return ((r - lo) >> 7).to(torch.int8).cuda(), lo.to(torch.int8).cuda()
    Ah, Al = res(nb * M)
    Bh, Bl = res(nb * N)
    acc = torch.empty((R.n, nb * M, N), dtype=torch.int16, device="cuda")
    return lambda: R.accumulate(Ah, Al, Bh, Bl, acc, nb=nb, fresh=True)


def _res_case(L, rows, K, unsigned):
    from .mpmat import lib_ctx
    R = lib_ctx(L)
    X = torch.randint(-(1 << 31), (1 << 31) - 1, (L, rows, K), dtype=torch.int32, device="cuda")
    return lambda: R.residues(X, 0, K, spread=True, unsigned=unsigned)


def _rows_case(L, nI, K):
    from .mpmat import lib_ctx
    R = lib_ctx(L)
    Rp = -(-K // 128) * 128
    Xr = torch.randint(0, 256, (nI, Rp, 128 if L <= 31 else 256), dtype=torch.uint8, device="cuda")
    return lambda: R.residues_rows(Xr, nI, Rp, 0, K)


def _mpgemm_case(L, n):
    from . import mpf
    A = mpf.from_float(np.random.default_rng(0).standard_normal((n, n)), L)
    return lambda: mpf.gemm(A, A)


def _cholsolve_case(L, nblocks):
    from . import mpf
    from .kernel_bench import cholsolve_inputs, cholsolve_buckets
    pairs = [(A, B) for _, _, A, B in cholsolve_buckets(cholsolve_inputs(nblocks, 8, 160, 8), L)]
    return lambda: mpf.chol_solve_many(pairs)


def _gram_case(L, N, rows):
    from . import mpf
    V = mpf.from_float(np.random.default_rng(2).standard_normal((rows, N)), L)

    def run():
        acc = mpf.GramAcc(N, L)
        acc.add(V)
        return acc.result()
    return run


def tune(reps=5, L=26):
    from .mpmat import lib_ctx
    R = lib_ctx(L)
    rng = np.random.default_rng(0)
    m = torch.tensor(R.mods, dtype=torch.int64, device="cuda")[:, None, None]
    acc_s = (torch.randint(0, 1 << 30, (R.n, 2880, 1000), device="cuda") % m).to(torch.int16)
    acc_g = (torch.randint(0, 1 << 30, (R.n, 274, 274), device="cuda") % m).to(torch.int16)
    z274 = torch.zeros(274, dtype=torch.int64, device="cuda")
    cases = {
        "crt_ctas": [lambda: R.crt_block(acc_s, 1000, 0, 1000, 2880),
                     lambda: R.crt_norm(acc_g, 274, 0, 274, 274, z274, z274, L - 1)],
        "narrow_max": [_gemm_case(R, 90, 32, 1000, 32, rng), _gemm_case(R, 30, 64, 1000, 64, rng),
                       _gemm_case(R, 131, 96, 8, 64, rng)],
        "pack_max": [_gemm_case(R, 106, 32, 32, 32, rng), _gemm_case(R, 131, 64, 32, 64, rng),
                     _gemm_case(R, 98, 16, 16, 16, rng)],
        "res_warps": [_res_case(27, 274, 7000, True), _res_case(26, 1000, 1000, False), _rows_case(27, 274, 7000)],
        "moduli_group": [_mpgemm_case(L, 512), _cholsolve_case(L, 60), _gram_case(L, 274, 1750)],
    }
    knobs, timings = {}, {}
    for name, (_, values) in KNOBS.items():
        default = get_knob(name)
        res = {}
        for v in values:
            set_knob(name, v)
            res[v] = sum(_time(fn, reps) for fn in cases[name])
        best = min(values, key=lambda v: res[v])
        set_knob(name, default)
        knobs[name] = best
        timings[name] = {str(v): round(t, 4) for v, t in res.items()}
    return {"device": torch.cuda.get_device_name(), "L": L, "knobs": knobs, "ms": timings}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--out", default=TABLE)
    a = ap.parse_args()
    table = tune(a.reps)
    with open(a.out, "w") as f:
        json.dump(table, f, indent=1)
    print(json.dumps(table))


if __name__ == "__main__":
    main()
