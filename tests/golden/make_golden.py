"""Generate the golden vectors in tests/golden/*.npz by running the reference itself on CPU.

Usage (in a container that has the reference tree; about 15-25 minutes on 8 cores):
    python tests/golden/make_golden.py [case ...]

The reference package (sdpvibe) is imported from its own tree by ``_refenv`` and executed on CPU
torch: Triton kernels under Triton's interpreter, CUDA C kernel strings as host code.  Every case
stores its seeded inputs and the reference's outputs; tests compare the oracle and the CUDA path
with them bit for bit.  Inputs are seeded with Python's `random` / numpy generators only.
"""
import os
import random
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import _refenv as R  # noqa: E402  (must come before torch / triton)
import numpy as np  # noqa: E402
import torch  # noqa: E402

from sdpvibe import rns, limbops, mpmat, mpf, batched, basecase, linalg  # noqa: E402


def limbs_of(values, L):
    """Python ints -> (L, n) int32 two's-complement limb planes."""
    return np.array([[((v >> (32 * k)) + (1 << 31)) % (1 << 32) - (1 << 31) for v in values]
                     for k in range(L)], dtype=np.int32).reshape(L, len(values))


def save(name, **arrays):
    out = {}
    for k, v in arrays.items():
        if torch.is_tensor(v):
            v = v.cpu().numpy()
        out[k] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"  wrote {name}.npz ({sum(a.nbytes for a in out.values())} bytes raw)")


def rmpf(rng, shape, L, elo, ehi, zero_frac=0.0):
    """Random normalised MPF: NB-bit mantissas, random sign, exponents uniform in [elo, ehi]."""
    n = int(np.prod(shape))
    nb = mpf.NBITS(L)
    ints, exps = [], []
    for _ in range(n):
        if rng.random() < zero_frac:
            ints.append(0); exps.append(0); continue
        v = rng.getrandbits(nb) | (1 << (nb - 1))
        ints.append(-v if rng.random() < 0.5 else v)
        exps.append(rng.randint(elo, ehi))
    return mpf.from_ints(ints, exps, L, shape)


# ------------------------------------------------------------------ cases
def case_bitlen():
    # tests/test_rns_kernels.py:16-25 (values around powers of two, three limbs)
    values = [v for bit in range(1, 95) for v in
              ((1 << bit) - 1, 1 << bit, (1 << bit) + 1, -(1 << bit) + 1, -(1 << bit), -(1 << bit) - 1)]
    values += [0, 1, -1]
    X = torch.from_numpy(limbs_of(values, 3))
    save("bitlen", X=X, out=limbops.bitlen_words(X))


def case_shift_round():
    rng = random.Random(5)
    for (Lin, Lout) in ((3, 2), (3, 3), (3, 5), (24, 24), (24, 25), (27, 26), (8, 1)):
        vals, shifts = [], []
        special = [0, 1, 2, 31, 32, 33, 63, 64, 65, 95, 96, 97, -1, -31, -32, -33, -64, 1 << 30, -(1 << 30) + 7]
        for s in special:
            for v in (0, 1, -1, (1 << (32 * Lin - 1)) - 1, -(1 << (32 * Lin - 1)), 3 << 40, -(3 << 40),
                      rng.randrange(-(1 << (32 * Lin - 1)), 1 << (32 * Lin - 1))):
                vals.append(v); shifts.append(s)
        for _ in range(300):
            vals.append(rng.randrange(-(1 << (32 * Lin - 1)), 1 << (32 * Lin - 1)))
            shifts.append(rng.randint(-40, 32 * Lin + 8))
        # ties: exact halves must round toward +infinity
        for _ in range(40):
            s = rng.randint(1, 32 * Lin - 2)
            q = rng.randrange(-(1 << (32 * Lin - 2 - s)), 1 << (32 * Lin - 2 - s)) if 32 * Lin - 2 - s > 0 else 0
            vals.append((q << s) + (1 << (s - 1))); shifts.append(s)
        X = torch.from_numpy(limbs_of(vals, Lin))
        s = torch.tensor(shifts, dtype=torch.int64)
        B = len(vals)
        out = torch.empty((Lout, B), dtype=torch.int32)
        flag = torch.empty((B,), dtype=torch.int32)
        limbops._shift_round_kernel[(-(-B // 256),)](X, s, out, flag, B, LIN=Lin, LOUT=Lout, BB=256,
                                                     PERENTRY=True)
        save(f"shift_round_{Lin}_{Lout}", X=X, s=s, out=out, flag=flag)


def case_add_same():
    rng = random.Random(9)
    for L in (1, 4, 24):
        lim = 1 << (32 * L - 1)
        a = [rng.randrange(-lim, lim) for _ in range(200)] + [lim - 1, -lim, 0, -1]
        b = [rng.randrange(-lim, lim) for _ in range(200)] + [1, -1, 0, lim - 1]
        A = torch.from_numpy(limbs_of(a, L)); Bm = torch.from_numpy(limbs_of(b, L))
        save(f"add_same_{L}", A=A, B=Bm, plus=limbops.add_same(A, Bm, 1), minus=limbops.add_same(A, Bm, -1))


def case_residues():
    # tests/test_rns_kernels.py:28-52
    for L in (1, 10, 24, 27, 28, 34):
        for K in (17, 65):
            rng = random.Random(123 + L + K)
            values = [[rng.randrange(-(1 << (32 * L - 1)), 1 << (32 * L - 1)) for _ in range(K)] for _ in range(3)]
            values[0][3:8] = [0, 1, -1, -(1 << (32 * L - 1)) + 1, (1 << (32 * L - 1)) - 1]
            X = torch.from_numpy(np.stack([limbs_of(r, L) for r in values], 1).copy())   # (L, 3, K)
            X[:, 0, 6] = 0
            X[-1, 0, 6] = -(1 << 31)                                                      # most negative value
            Rc = rns.RNS(L)
            out = {}
            for g0, G in ((0, Rc.n), (Rc.n - 16, 16)):
                hi, lo = Rc.residues(X, 3, K - 5, g0, G)
                out[f"hi_{g0}"] = hi; out[f"lo_{g0}"] = lo
            save(f"residues_L{L}_K{K}", X=X, k0=3, kc=K - 5, n=Rc.n, **out)


def case_crt_block():
    # tests/test_rns_kernels.py:55-80
    for L in (1, 10, 24, 27, 34):
        Rc = rns.RNS(L)
        rng = random.Random(41 + L)
        rows, N, start = 5, 13, 2
        limit = Rc.M // 4
        values = [[rng.randrange(-limit + 1, limit) for _ in range(N)] for _ in range(rows)]
        values[0][2:7] = [0, 1, -1, limit - 1, -limit + 1]
        values[1][2:7] = [1 << b for b in (0, 31, 32, 63, 64)]
        values[2][2:7] = [-(1 << b) for b in (0, 31, 32, 63, 64)]
        acc = torch.tensor([[[v % p for v in row] for row in values] for p in Rc.mods], dtype=torch.int16)
        out = {}
        for width in (1, 5, 11):
            W, bl, cnt = Rc.crt_block(acc, N, start, width, rows)
            out[f"W_{width}"] = W[:, :cnt]; out[f"bl_{width}"] = bl[:cnt]
        save(f"crt_block_L{L}", acc=acc, start=start, **out)


def case_accumulate():
    rng = np.random.default_rng(3)
    for L, (M, N, KC) in ((24, (70, 50, 48)), (26, (33, 130, 80))):
        Rc = rns.RNS(L)
        G = Rc.n
        m = np.array(Rc.mods)[:, None, None]
        ra = rng.integers(0, 1 << 30, size=(G, M, KC)) % m
        rb = rng.integers(0, 1 << 30, size=(G, N, KC)) % m
        ra = np.where(ra > m // 2, ra - m, ra); rb = np.where(rb > m // 2, rb - m, rb)
        split = lambda r: (((r + 64) & 127) - 64, (r - (((r + 64) & 127) - 64)) >> 7)
        alo, ahi = split(ra); blo, bhi = split(rb)
        t8 = lambda x: torch.from_numpy(x.astype(np.int8))
        acc0 = torch.from_numpy((rng.integers(0, 1 << 30, size=(G, M, N)) % m).astype(np.int16))
        acc = acc0.clone()
        Rc.accumulate(t8(ahi), t8(alo), t8(bhi), t8(blo), acc, 0)
        save(f"accumulate_L{L}", Ahi=t8(ahi), Alo=t8(alo), Bhi=t8(bhi), Blo=t8(blo), acc0=acc0, acc=acc)


def case_gemm_nt():
    # tests/test_gemm.py:199-214
    for L, cases in ((24, [(5, 7, 3, 'col'), (40, 33, 70, 'mat'), (9, 6, 20, -1000), (12, 70, 33, 'col')]),
                     (34, [(5, 7, 3, 'col'), (17, 9, 40, 'mat')])):
        rng = random.Random(1 + L)
        rint = lambda bits: rng.getrandbits(bits) * rng.choice([-1, 1])
        for ci, (M, N, K, mode) in enumerate(cases):
            A = [[rint(32 * L - 40) for _ in range(K)] for _ in range(M)]
            B = [[rint(32 * L - 40) for _ in range(K)] for _ in range(N)]
            Am, Bm = mpmat.from_ints(A, -1000, L), mpmat.from_ints(B, -1060, L)
            C = mpmat.gemm_nt(Am, Bm, out_exp=mode)
            save(f"gemm_nt_L{L}_{ci}", A=Am.limbs, B=Bm.limbs, eA=-1000, eB=-1060, mode=str(mode),
                 C=C.limbs, Ce=C.exp)
        # per-row exponents of Bt (the trsm path: gemm_nt(X, B^T, 'col', bt_rowexp=...))
        M, N, K = 8, 11, 13
        A = [[rint(32 * L - 40) for _ in range(K)] for _ in range(M)]
        B = [[rint(32 * L - 50) for _ in range(K)] for _ in range(N)]
        rowexp = torch.tensor([rng.randint(-40, 40) for _ in range(N)], dtype=torch.int64)
        Am, Bm = mpmat.from_ints(A, -7, L), mpmat.from_ints(B, 0, L)
        C = mpmat.gemm_nt(Am, Bm, out_exp="col", bt_rowexp=rowexp)
        save(f"gemm_nt_rowexp_L{L}", A=Am.limbs, B=Bm.limbs, eA=-7, rowexp=rowexp, C=C.limbs, Ce=C.exp)


def case_mpmat_add():
    rng = random.Random(7)
    L = 24
    rint = lambda bits: rng.getrandbits(bits) * rng.choice([-1, 1])
    A = [[rint(700) for _ in range(9)] for _ in range(4)]
    B = [[rint(700) for _ in range(9)] for _ in range(4)]
    Am, Bm = mpmat.from_ints(A, -900, L), mpmat.from_ints(B, -1000, L)
    ec = torch.tensor([rng.randint(-1100, -900) for _ in range(9)], dtype=torch.int64)
    Bc = mpmat.MP(Bm.limbs.clone(), ec)
    out = dict(A=Am.limbs, B=Bm.limbs, eA=-900, eB=-1000, ec=ec)
    for tag, (x, y, a, oe) in {"gen": (Am, Bm, -1, None), "col": (Am, Bc, 1, "col"), "mat": (Am, Bc, -1, "mat"),
                               "align": (Am, Bc, 1, "align"), "same": (Am, mpmat.MP(Bm.limbs, -900), -1, -900)}.items():
        C = mpmat.add(x, y, a, out_exp=oe)
        out[f"{tag}_C"] = C.limbs; out[f"{tag}_e"] = C.exp
    R = mpmat.rescale(Bc, -950)
    out["rescale_C"] = R.limbs
    save("mpmat_add", **out)


def case_badd():
    # tests/test_badd.py:149-188
    for L in (1, 4, 28, 34):
        for uniform in (False, True):
            rng = random.Random(19 + L)
            nb, rows, cols = 2, 3, 5
            limit = 1 << (32 * L - 1)
            edge = [0, 1, -1, limit - 1, -limit]
            a = [rng.randrange(-limit, limit) for _ in range(nb * rows * cols)]
            b = list(reversed(a))
            a[:5], b[:5] = edge, list(reversed(edge))
            a[10:14] = [limit - 1, -limit, limit - 1, -limit]
            b[10:14] = [-limit, limit - 1, limit - 1, -limit]
            ea = [-100] * (nb * cols)
            eb = [-100] * (nb * cols) if uniform else [-100 + d for d in (0, 1, 31, 32, 33, 63, 64, 65, -10000, 10000)]
            mk = lambda v, e: batched.BMP(torch.from_numpy(limbs_of(v, L)).view(L, nb, rows, cols),
                                          e[0] if uniform else torch.tensor(e, dtype=torch.int64).view(nb, cols))
            out = {}
            for sgn in (1, -1):
                o = batched.badd(mk(a, ea), mk(b, eb), sgn, out_exp="align")
                out[f"C_{sgn}"] = o.limbs; out[f"e_{sgn}"] = o.exp
            save(f"badd_L{L}_{'u' if uniform else 'n'}", A=limbs_of(a, L), B=limbs_of(b, L),
                 ea=np.array(ea), eb=np.array(eb), **out)


def case_mpf_elementwise():
    # tests/test_mpf_mul.py:115-139 plus mpf_add / mpf_norm
    for L in (1, 2, 10, 24, 26, 28, 34, 64):
        rng = random.Random(71 + L)
        bits = mpf.NBITS(L)
        edge = [0, 1, -1, (1 << bits) - 1, -((1 << bits) - 1), 1 << (bits - 1), -(1 << (bits - 1)),
                (1 << (bits - 1)) + 1]
        values = edge + [rng.randrange(-(1 << bits), 1 << bits) for _ in range(129)]
        a = mpf.from_ints(values, [rng.randrange(-2000, 2000) for _ in values], L, (len(values),))
        bv = list(reversed(values))
        b = mpf.from_ints(bv, [rng.randrange(-2000, 2000) for _ in bv], L, (len(bv),))
        # exponent gaps that exercise alignment in mpf_add
        gaps = [0, 1, 2, 31, 32, 33, 64, 32 * L, 32 * L + 3, 32 * (L + 3) + 5, -1, -33, -32 * L - 70]
        be = a.e.clone()
        for i in range(len(values)):
            be[i] = a.e[i] + gaps[i % len(gaps)]
        b2 = mpf.MPF(b.m.clone(), torch.where(b.e == mpf.EZ, b.e, be))
        sc = mpf.from_ints([(1 << bits) - 1], [5], L, (1,))
        wide = torch.from_numpy(limbs_of([rng.randrange(-(1 << (32 * (L + 3) - 1)), 1 << (32 * (L + 3) - 1))
                                          for _ in range(64)] + [0, 1, -1, 1 << 100, -(1 << 100)], L + 3))
        ein = torch.tensor([rng.randrange(-500, 500) for _ in range(wide.shape[1])], dtype=torch.int64)
        nrm = mpf.normalize(wide, ein, L)
        m1 = mpf.mul(a, b); ms = mpf.mul(a, sc); s1 = mpf.add(a, b2, 1); s2 = mpf.add(a, b2, -1)
        save(f"mpf_elem_L{L}", am=a.m, ae=a.e, bm=b2.m, be=b2.e, b0m=b.m, b0e=b.e, scm=sc.m, sce=sc.e,
             mul_m=mpf.mul(a, b).m, mul_e=mpf.mul(a, b).e, muls_m=ms.m, muls_e=ms.e,
             add_m=s1.m, add_e=s1.e, sub_m=s2.m, sub_e=s2.e, wide=wide, ein=ein, nrm_m=nrm.m, nrm_e=nrm.e)


def case_mpf_gemm():
    rng = random.Random(11)
    for tag, (L, shp, tA, tB, lo, hi) in {
            "2d": (24, (7, 9, 5), False, False, -4, 4),
            "2d_scaled": (26, (13, 21, 11), False, True, -300, 300),
            "3d": (10, (3, 6, 10, 4), True, False, -8, 8),
            "zeros": (24, (6, 5, 7), False, False, -4, 4)}.items():
        if len(shp) == 3:
            M, K, N = shp
            A = rmpf(rng, (K, M) if tA else (M, K), L, lo, hi, 0.3 if tag == "zeros" else 0.0)
            B = rmpf(rng, (N, K) if tB else (K, N), L, lo, hi, 0.3 if tag == "zeros" else 0.0)
        else:
            nb, M, K, N = shp
            A = rmpf(rng, (nb, K, M) if tA else (nb, M, K), L, lo, hi)
            B = rmpf(rng, (nb, N, K) if tB else (nb, K, N), L, lo, hi)
        C = mpf.gemm(A, B, tA, tB)
        save(f"mpf_gemm_{tag}", Am=A.m, Ae=A.e, Bm=B.m, Be=B.e, tA=tA, tB=tB, Cm=C.m, Ce=C.e)


def case_gramacc():
    # tests/test_gramacc.py:8-23 (chunk scale jumps; 60 > HEAD forces a flush)
    L, N = 8, 40
    rng = random.Random(13)
    for si, scales in enumerate(([0, 0, 0], [0, 10, -40], [0, 60, -5])):
        chunks = [rmpf(rng, (r, N), L, -8, 8).shift(sc) for r, sc in zip((60, 17, 33), scales)]
        acc = mpf.GramAcc(N, L)
        for c in chunks:
            acc.add(c)
        Q = acc.result()
        save(f"gramacc_{si}", **{f"P{i}m": c.m for i, c in enumerate(chunks)},
             **{f"P{i}e": c.e for i, c in enumerate(chunks)}, Qm=Q.m, Qe=Q.e, flushes=acc.flushes,
             Eref=acc.next_reference(), loss=acc.precision_loss())
    # with reference exponents from a previous accumulation
    chunks = [rmpf(rng, (r, N), L, -8, 8) for r in (25, 31)]
    acc = mpf.GramAcc(N, L)
    for c in chunks:
        acc.add(c)
    E = acc.next_reference()
    acc2 = mpf.GramAcc(N, L, E_ref=E)
    for c in chunks:
        acc2.add(c)
    Q = acc2.result()
    save("gramacc_eref", **{f"P{i}m": c.m for i, c in enumerate(chunks)},
         **{f"P{i}e": c.e for i, c in enumerate(chunks)}, Eref=E, Qm=Q.m, Qe=Q.e, flushes=acc2.flushes)


def spd_blocks(rng, nb, n, L, rowscale):
    """A = G G^T + n I from integer G (exact), optional power-of-two row/column scaling."""
    vals, exps = [], []
    for b in range(nb):
        G = [[rng.randint(-60, 60) for _ in range(n)] for _ in range(n)]
        d = [rng.randint(-rowscale, rowscale) for _ in range(n)]
        for i in range(n):
            for j in range(n):
                v = sum(G[i][k] * G[j][k] for k in range(n)) + (100 * n if i == j else 0)
                vals.append(v); exps.append(d[i] + d[j])
    return mpf.from_ints(vals, exps, L, (nb, n, n))


def case_chol():
    rng = random.Random(17)
    for tag, (L, nb, n, nr, rs) in {"n40": (8, 2, 40, 3, 30), "n32": (8, 3, 32, 2, 0),
                                     "n70": (6, 1, 70, 2, 60)}.items():
        A = spd_blocks(rng, nb, n, L, rs)
        ch = mpf.Chol(A)
        B = rmpf(rng, (nb, n, nr), L, -20, 20)
        lo, up = ch.solve_lower(B), ch.solve_upper(B)
        xs = ch.solve(B)
        tiles = {f"X{i}m": t.X.limbs for i, t in enumerate(ch.tiles)}
        tiles.update({f"X{i}e": t.X.exp for i, t in enumerate(ch.tiles)})
        save(f"chol_{tag}", Am=A.m, Ae=A.e, Bm=B.m, Be=B.e, Lt=ch.Lt.limbs, k=ch.k,
             lo_m=lo.m, lo_e=lo.e, up_m=up.m, up_e=up.e, x_m=xs.m, x_e=xs.e, **tiles)


def case_blockchol():
    # sdpvibe/blockchol.py: the tiled Cholesky of one N x N matrix (lower triangle valid) and its solves
    from sdpvibe.blockchol import BlockChol
    rng = random.Random(29)
    L, N, b, nr = 8, 70, 32, 3
    A = spd_blocks(rng, 1, N, L, 12)
    Q = mpf.MPF(A.m[:, 0].contiguous(), A.e[0].contiguous())
    ch = BlockChol([Q], b)
    B = rmpf(rng, (N, nr), L, -20, 20)
    lo, up, xs = ch.solve_lower(B), ch.solve_upper(B), ch.solve(B)
    save("blockchol_n70_b32", Qm=A.m[:, 0], Qe=A.e[0], b=b, Bm=B.m, Be=B.e, lo_m=lo.m, lo_e=lo.e, up_m=up.m,
         up_e=up.e, x_m=xs.m, x_e=xs.e, log2_cond=np.float64(ch.log2_cond()))


def case_bigfloat():
    # sdpvibe/_bigfloat.c via sdpvibe/sdp_io.py: a block written by write_block_bin (boost binary archive of
    # El::BigFloat records) and read back by read_block; plus raw records of every kind for the decoder
    from sdpvibe import sdp_io
    import struct
    rng = random.Random(31)
    for tag, (L, precision, dim, K, N, h) in {"L8_p200": (8, 200, 2, 3, 4, 2), "L26_p768": (26, 768, 1, 5, 3, 3)}.items():
        npair = dim * (dim + 1) // 2
        def host(shape, elo, ehi, zf=0.2):
            A = rmpf(rng, shape, L, elo, ehi, zf)
            return A.m.reshape(L, -1).T.contiguous().numpy(), A.e.reshape(-1).numpy()
        blk = {"dim": dim, "K": K, "B": host((K * npair, N), -30, 30), "c": host((K * npair,), -10, 10),
               "bilinear_bases_even": (h, host((h, K), -5, 5)), "bilinear_bases_odd": (0, None)}
        path = os.path.join("/tmp", f"block_{tag}.bin")
        sdp_io.write_block_bin(path, blk, precision, L, N)
        raw = open(path, "rb").read()
        r = sdp_io._BinReader(raw, L)
        _, _, Bl, Be = r.matrix()
        cl, ce = r.vector()
        bases = [r.matrix(), r.matrix()]
        save(f"bigfloat_block_{tag}", raw=np.frombuffer(raw, np.uint8), L=L, precision=precision, dim=dim, K=K, N=N,
             h=h, Bl=Bl, Be=Be, cl=cl, ce=ce, hl=bases[0][2], he=bases[0][3], in_Bl=blk["B"][0], in_Be=blk["B"][1])
    # raw records: zeros (flag), zero mantissa, short sizes, negative, rounding carries, limbs past size
    for nl, L in ((4, 4), (13, 26), (3, 8)):
        recs, n = bytearray(), 0
        for kind in range(60):
            if kind % 7 == 0:
                recs += b"\x01"; n += 1; continue
            asz = rng.randint(0, nl)
            limbs = [rng.getrandbits(64) for _ in range(nl)]
            if kind % 11 == 0:
                limbs[:asz] = [(1 << 64) - 1] * asz                     # rounding carries through
            size = -asz if rng.random() < 0.5 else asz
            exp = rng.randint(-40, 40)
            recs += b"\x00" + struct.pack("<iq", size, exp) + struct.pack(f"<{nl}Q", *limbs)
            n += 1
        buf = np.frombuffer(bytes(recs), np.uint8)
        lim = np.empty((n, L), np.int32)
        ex = np.empty(n, np.int64)
        lib = sdp_io._lib()
        q = lib.decode_bigfloats(buf.ctypes.data, len(buf), 0, n, nl, L, lim.ctypes.data, ex.ctypes.data, mpf.EZ)
        enc = sdp_io._encode(lim, ex, nl, L)
        save(f"bigfloat_records_nl{nl}_L{L}", raw=buf, n=n, nl=nl, L=L, limbs=lim, exps=ex, end=q,
             enc=np.frombuffer(enc, np.uint8))


def case_basecase():
    # sdpvibe/basecase.py:268-293 on single 32x32 tiles (equilibrated, fixed point)
    rng = random.Random(23)
    for L in (4, 8):
        FX = 32 * L - 40
        n = 32
        G = [[rng.randint(-100, 100) for _ in range(n)] for _ in range(n)]
        A = [[sum(G[i][k] * G[j][k] for k in range(n)) + (n * 50 if i == j else 0) for j in range(n)] for i in range(n)]
        sh = [(A[i][i].bit_length()) // 2 + 1 for i in range(n)]
        Aint = [[(A[i][j] << FX) >> (sh[i] + sh[j]) for j in range(n)] for i in range(n)]
        Am = mpmat.from_ints(Aint, -FX, L)
        Lg, Xg = basecase.chol_inv_tile(Am)
        save(f"basecase_L{L}", A=Am.limbs, L=Lg.limbs, Le=Lg.exp, X=Xg.limbs, Xe=Xg.exp)


def _equilibrated_spd(rng, n, spread, L):
    """tests/test_linalg.py:30-48 construction: A = V diag(2^-e_k) V^T (exact integers, e_k spread over
    `spread` bits), equilibrated by powers of two, fixed point with exponent fx_exp(L) (diagonal < 1)."""
    FX = -linalg.fx_exp(L)
    V = [[rng.randint(-8, 8) for _ in range(n)] for _ in range(n)]
    ek = [int(round(k * spread / (n - 1))) for k in range(n)]
    emax = max(ek)
    A = [[sum(V[i][k] * V[j][k] << (emax - ek[k]) for k in range(n)) for j in range(n)] for i in range(n)]
    sh = [(A[i][i].bit_length() - 1) // 2 for i in range(n)]
    out = []
    for i in range(n):
        row = []
        for j in range(n):
            s = FX - sh[i] - sh[j] - 1
            v = A[i][j]
            row.append(v << s if s >= 0 else (v + (1 << (-s - 1))) >> (-s))
        out.append(row)
    return mpmat.from_ints(out, -FX, L)


def case_linalg():
    # sdpvibe/linalg.py on one matrix: chol (substitution and tile-inverse panels, refinement), trsm_left
    # (gemm and substitution leaves), chol_inv + trsm, and basecase.trsv_tile
    rng = random.Random(29)
    L, n, m = 8, 96, 5
    A = _equilibrated_spd(rng, n, 60, L)
    Bv = [[rng.randrange(-(1 << 200), 1 << 200) for _ in range(m)] for _ in range(n)]
    B = mpmat.from_ints(Bv, -200, L)
    B = mpmat.MP(B.limbs, torch.tensor([rng.randint(-6, 6) for _ in range(m)], dtype=torch.int64) - 200)
    out = dict(Am=A.limbs, Ae=A.uniform_exp(), Bm=B.limbs, Be=B.exp)
    Ls, ts = linalg.chol(A, tile_inverses=True, panel_leaf="subst")
    out.update(Ls=Ls.limbs, Ls_e=Ls.uniform_exp())
    Lg, tg = linalg.chol(A, tile_inverses=True, panel_leaf="gemm", refine=1)
    out.update(Lg=Lg.limbs, Lg_e=Lg.uniform_exp())
    for leaf in ("gemm", "subst"):
        P = linalg.trsm_left(Ls, B, ts, leaf=leaf)
        out.update({f"P_{leaf}_m": P.limbs, f"P_{leaf}_e": P.exp})
    Lc, Xc = linalg.chol_inv(A)
    out.update(Lc=Lc.limbs, Lc_e=Lc.uniform_exp(), Xc=Xc.limbs, Xc_e=Xc.uniform_exp())
    P2 = linalg.trsm(Xc, B)
    out.update(P2_m=P2.limbs, P2_e=P2.exp)
    Vt = mpmat.from_ints([[rng.randrange(-(1 << 180), 1 << 180) for _ in range(32)] for _ in range(7)], 0, L)
    ve = torch.tensor([rng.randint(-10, 10) for _ in range(7)], dtype=torch.int64)
    Y, ye = basecase.trsv_tile(ts[0], Vt.limbs, ve)
    Yf, yfe = basecase.trsv_tile(ts[0], Vt.limbs, ve, out_exp=-(32 * L - 40))
    out.update(Vm=Vt.limbs, ve=ve, Ym=Y, ye=ye, Yfm=Yf, yfe=yfe,
               t0_Lw=ts[0].Lw, t0_RINV=ts[0].RINV)
    save("linalg_n96", **out)


CASES = {k[5:]: v for k, v in globals().items() if k.startswith("case_")}

if __name__ == "__main__":
    names = sys.argv[1:] or list(CASES)
    for name in names:
        t = time.time()
        print(f"{name} ...", flush=True)
        CASES[name]()
        print(f"  {time.time() - t:.1f}s", flush=True)
