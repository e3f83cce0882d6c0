"""Synthetic SDPs for benchmarks and tests (the reference's sdpvibe/synthetic.py builds block shapes the
same way; the PMP -> SDP conversion itself is outside this package).

``ising_like``: the "Ising-structured" SDP used for per-iteration timings: 300 blocks with dims 1 / 2 / 3
in the ratio 6 : 3 : 1, polynomial degree d ~ U[20, 40] per block (numpy seed), K = d + 1 sample points
x_k = k / (d + 1), even / odd bilinear bases of sizes floor(d/2) + 1 and floor((d-1)/2) + 1 (the rule of
sdpvibe/synthetic.py:16-17) built from damped monomials sqrt(e^-x_k) x_k^m (odd: an extra sqrt(x_k)),
random normalised B, c and b; N = 1000 free variables.
"""
import numpy as np


def ising_like_shapes(nblocks=300, N=1000, dmin=20, dmax=40, seed=0):
    rng = np.random.default_rng(seed)
    dims = [1] * (nblocks * 6 // 10) + [2] * (nblocks * 3 // 10)
    dims += [3] * (nblocks - len(dims))
    blocks = []
    for dim in dims:
        d = int(rng.integers(dmin, dmax + 1))
        blocks.append(dict(dim=dim, K=d + 1, he=d // 2 + 1, ho=(d - 1) // 2 + 1, d=d))
    return blocks, N


def damped_bases(d, he, ho):
    """(V_even (he, K), V_odd (ho, K)) float64: sqrt(e^-x) x^m and sqrt(x e^-x) x^m at x_k = k/(d+1)"""
    x = np.arange(d + 1, dtype=np.float64) / (d + 1)
    w = np.sqrt(np.exp(-x))
    Ve = np.stack([w * x ** m for m in range(he)])
    Vo = np.stack([w * np.sqrt(x) * x ** m for m in range(ho)]) if ho else None
    return Ve, Vo


def ising_like_sdp(L, nblocks=300, N=1000, seed=0):
    """(SDP, block shapes) of ising_like_shapes with its data"""
    from .solver import SDP, _rand_host_mpf
    blocks, N = ising_like_shapes(nblocks, N, seed=seed)
    rng = np.random.default_rng(seed + 1)
    data = []
    for bl in blocks:
        Ve, Vo = damped_bases(bl["d"], bl["he"], bl["ho"])
        npair = bl["dim"] * (bl["dim"] + 1) // 2
        data.append(dict(dim=bl["dim"], K=bl["K"], Ve=Ve, Vo=Vo, c=_rand_host_mpf(rng, (bl["K"] * npair, 1), L),
                         B=_rand_host_mpf(rng, (bl["K"] * npair, N), L)))
    b = _rand_host_mpf(rng, (N, 1), L)
    return SDP(data, b, 0, L), blocks
