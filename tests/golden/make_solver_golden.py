"""Golden iterates of the reference's SDPB iteration (sdpvibe/solver.py Solver.run) on a tiny SDP.

Usage (in a container that has the reference tree; CPU only, slow: the Triton interpreter):
    python tests/golden/make_solver_golden.py

The reference package runs on CPU torch through ``_refenv`` (Triton interpreter, CUDA C strings as
host code).  Its GPU-only plumbing is replaced by stand-ins that do not touch the arithmetic: the
chunk store (sdpvibe/store.py: CUDA copy streams) by a dict, torch.cuda.synchronize by a no-op, and the
memory plan gets a fixed budget so that every chunk is resident, as on a large GPU.  The SDP data are
seeded numpy arrays of normalised MPF limbs; the fixture stores them with, for every iteration, the
scalars SDPB prints, the step lengths, y and each chunk's corrector direction (dx, dX, dY).
"""
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refenv as R  # noqa: E402,F401  (must come before torch / triton)
import mpmath as mp  # noqa: E402
import numpy as np  # noqa: E402
import torch  # noqa: E402

import sdpvibe.store as store  # noqa: E402


class DictStore:
    """resident-only stand-in for sdpvibe.store.Store (the methods the solver calls)"""

    def __init__(self, host_keys=(), ahead=1):
        self.d = {}

    def is_host(self, key):
        return False

    def put(self, key, obj):
        self.d[key] = obj

    def get(self, key):
        return self.d[key]

    def drop(self, key):
        self.d.pop(key, None)

    def prefetch(self, key):
        pass

    def stream(self, items, nxt=()):
        for keys in items:
            yield tuple(self.d.get(k) for k in keys)


store.Store = DictStore
torch.cuda.synchronize = lambda *a, **k: None          # CPU run: nothing to wait for
import sdpvibe.solver as S  # noqa: E402
from sdpvibe import mpf as F  # noqa: E402

# block shapes: two dim-1 blocks of different K (padding inside a chunk), one dim-2, one dim-3
BLOCKS = [dict(dim=1, K=3, he=2, ho=1), dict(dim=1, K=2, he=1, ho=1),
          dict(dim=2, K=3, he=2, ho=1), dict(dim=3, K=2, he=1, ho=1)]
N, L, ITERS, SEED = 5, 8, 3, 11
T0 = time.time()


def rand_host(rng, shape, spread=4):
    """normalised random MPF host data, |value| in [2^u, 2^(u+1)), u ~ U[-spread, spread]"""
    n = int(np.prod(shape))
    nb = 32 * L - 2
    vals, exps = [], []
    for _ in range(n):
        v = (1 << (nb - 1)) | int.from_bytes(rng.bytes((nb + 7) // 8), "little") % (1 << (nb - 1))
        vals.append(-v if rng.random() < 0.5 else v)
        exps.append(int(rng.integers(-spread, spread + 1)) - nb + 1)
    m = np.array([[((v >> (32 * k)) + (1 << 31)) % (1 << 32) - (1 << 31) for v in vals] for k in range(L)],
                 dtype=np.int32).reshape(L, *shape)
    return m, np.array(exps, dtype=np.int64).reshape(shape)


def to_ref(H):
    m, e = H
    return F.MPF(torch.from_numpy(m.copy()), torch.from_numpy(e.copy()))


def mpstr(v):
    """exact binary representation of an mpmath value"""
    s, man, ex, _ = mp.mpf(v)._mpf_
    return f"{'-' if s else ''}{int(man)}*2^{int(ex)}"


def main():
    rng = np.random.default_rng(SEED)
    b = rand_host(rng, (N, 1))
    data = []
    for bl in BLOCKS:
        npair = bl["dim"] * (bl["dim"] + 1) // 2
        data.append((rand_host(rng, (bl["he"], bl["K"])) if bl["he"] else None,
                     rand_host(rng, (bl["ho"], bl["K"])) if bl["ho"] else None,
                     rand_host(rng, (bl["K"] * npair, 1)), rand_host(rng, (bl["K"] * npair, N))))
    mp.mp.prec = F.NBITS(L) + 64
    sdp = S.SDP.__new__(S.SDP)
    lay = S.Layout(BLOCKS, N, L, budget=1e12, stream="none")
    sdp._build(BLOCKS, lambda j: tuple(None if x is None else to_ref(x) for x in data[j]), to_ref(b),
               mp.mpf(0), L, lay)
    sol = S.Solver(sdp, L)
    out = {"b_m": b[0], "b_e": b[1], "N": N, "L": L, "iters": ITERS, "seed": SEED,
           "blk_dim": np.array([bl["dim"] for bl in BLOCKS]), "blk_K": np.array([bl["K"] for bl in BLOCKS])}
    for j, (Ve, Vo, c, B) in enumerate(data):
        for k, v in (("Ve", Ve), ("Vo", Vo), ("c", c), ("B", B)):
            if v is not None:
                out[f"blk{j}_{k}_m"], out[f"blk{j}_{k}_e"] = v
    out["chunk_blocks"] = np.array([j for c in lay.chunks for j in c])

    def snap(row):
        it = row["iteration"]
        for k in ("mu", "P-obj", "D-obj", "gap", "P-err", "p-err", "D-err", "R-err", "P-step", "D-step", "beta"):
            out[f"it{it}_{k}"] = np.array(row[k])
        aP, aD, _ = sol.last_steps
        out[f"it{it}_aP"], out[f"it{it}_aD"] = np.array(mpstr(aP)), np.array(mpstr(aD))
        out[f"it{it}_y_m"], out[f"it{it}_y_e"] = sol.y.m.numpy(), sol.y.e.numpy()
        for gi in range(len(sdp.groups)):
            dc = sdp.store.get(("dc", gi))
            for name, M in (("dx", dc["dx"]), ("dX", dc["dX"][0]), ("dY", dc["dY"][0])):
                out[f"it{it}_g{gi}_{name}_m"], out[f"it{it}_g{gi}_{name}_e"] = M.m.numpy(), M.e.numpy()
        print(f"  iteration {it}: mu {row['mu']} steps {row['P-step']} {row['D-step']} ({time.time() - T0:.0f} s)",
              flush=True)
        np.savez_compressed(os.path.join(HERE, "solver_tiny.npz"), **out, iters_done=it)
    res = sol.run(max_iter=ITERS, verbose=False, on_iteration=snap)
    out["terminate"] = np.array(res["terminateReason"])
    np.savez_compressed(os.path.join(HERE, "solver_tiny.npz"), **out, iters_done=ITERS)
    print("wrote solver_tiny.npz")


if __name__ == "__main__":
    main()
