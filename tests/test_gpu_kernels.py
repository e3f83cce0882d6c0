"""Parity of the CUDA path (libsdpv_b200 through the C ABI) with the reference's golden vectors and
with the CPU oracle.  Every comparison is bit-exact."""
import random

import numpy as np
import pytest
import torch

import oracle as O
from oracle import mp as OM
from conftest import golden, golden_names

pytestmark = pytest.mark.gpu


def cu(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def np_(t):
    return t.detach().cpu().numpy()


@pytest.fixture(scope="module")
def sb():
    import sdpvibe_b200 as sb
    from sdpvibe_b200 import limbops, rns, mpmat, mpf  # noqa: F401
    assert torch.cuda.is_available()
    return sb


def rand_limbs(rng, L, n):
    return rng.integers(-(1 << 31), 1 << 31, size=(L, n), dtype=np.int64).astype(np.int32)


# ------------------------------------------------------------------ limb bookkeeping
def test_bitlen_golden(sb):
    from sdpvibe_b200.limbops import bitlen_words
    g = golden("bitlen")
    assert np.array_equal(np_(bitlen_words(cu(g["X"]))), g["out"])


@pytest.mark.parametrize("name", golden_names("shift_round_"))
def test_shift_round_golden(sb, name):
    from sdpvibe_b200 import _lib
    g = golden(name)
    X, s = cu(g["X"]), cu(g["s"])
    Lout = g["out"].shape[0]
    out = torch.empty((Lout, X.shape[1]), dtype=torch.int32, device="cuda")
    flag = torch.empty((X.shape[1],), dtype=torch.int32, device="cuda")
    _lib.call("sdpv_shift_round", _lib.ptr(X), X.shape[0], X.shape[1], _lib.ptr(s), Lout, _lib.ptr(out),
              _lib.ptr(flag), _lib.stream())
    assert np.array_equal(np_(out), g["out"])
    assert np.array_equal(np_(flag), g["flag"])


def test_shift_round_random_large(sb):
    from sdpvibe_b200.limbops import shift_round
    rng = np.random.default_rng(1)
    for Lin, Lout in ((26, 27), (27, 24), (5, 9)):
        X = rand_limbs(rng, Lin, 200_003)
        s = rng.integers(-70, 32 * Lin + 40, size=X.shape[1])
        ref, _ = O.shift_round(X, s, Lout)
        assert np.array_equal(np_(shift_round(cu(X), cu(s), Lout)), ref)


def test_overflow_flag_device_word(sb):
    from sdpvibe_b200 import _lib
    from sdpvibe_b200.limbops import shift_round, check_errors
    _lib.device_error_flags()                            # clear flags left by earlier overflowing shifts
    check_errors()
    X = cu(O.to_limbs([(1 << 60) + 5, 3], 3))
    shift_round(X, cu(np.array([-10, 0])), 2)            # 2^70 does not fit two limbs
    with pytest.raises(OverflowError):
        check_errors()
    check_errors()                                       # cleared by the previous read


@pytest.mark.parametrize("name", golden_names("add_same_"))
def test_add_same_golden(sb, name):
    from sdpvibe_b200.limbops import add_same
    g = golden(name)
    assert np.array_equal(np_(add_same(cu(g["A"]), cu(g["B"]), 1)), g["plus"])
    assert np.array_equal(np_(add_same(cu(g["A"]), cu(g["B"]), -1)), g["minus"])


@pytest.mark.parametrize("name", golden_names("badd_"))
def test_badd_golden(sb, name):
    from sdpvibe_b200 import _lib
    g = golden(name)
    L = g["A"].shape[0]
    nb, rows, cols = 2, 3, 5
    EA = cu(np.broadcast_to(g["ea"].reshape(nb, cols), (nb, cols)).copy())
    EB = cu(np.broadcast_to(g["eb"].reshape(nb, cols), (nb, cols)).copy())
    A, B = cu(g["A"]), cu(g["B"])
    for sgn in (1, -1):
        out = torch.empty_like(A)
        eo = torch.empty((nb, cols), dtype=torch.int64, device="cuda")
        _lib.call("sdpv_badd_align", _lib.ptr(A), _lib.ptr(B), _lib.ptr(EA), _lib.ptr(EB), L, nb, rows, cols, sgn,
                  _lib.ptr(out), _lib.ptr(eo), _lib.stream())
        assert np.array_equal(np_(out).reshape(g[f"C_{sgn}"].shape), g[f"C_{sgn}"])
        assert np.array_equal(np_(eo), np.broadcast_to(g[f"e_{sgn}"], (nb, cols)))


# ------------------------------------------------------------------ MPF elementwise
@pytest.mark.parametrize("name", golden_names("mpf_elem_"))
def test_mpf_elementwise_golden(sb, name):
    from sdpvibe_b200.mpf import MPF, mul, add, normalize
    g = golden(name)
    L = g["am"].shape[0]
    A = MPF(cu(g["am"]), cu(g["ae"]))
    B0 = MPF(cu(g["b0m"]), cu(g["b0e"]))
    B2 = MPF(cu(g["bm"]), cu(g["be"]))
    S = MPF(cu(g["scm"]), cu(g["sce"]))
    for got, key in ((mul(A, B0), "mul"), (mul(A, S), "muls"), (add(A, B2, 1), "add"), (add(A, B2, -1), "sub"),
                     (normalize(cu(g["wide"]), cu(g["ein"]), L), "nrm")):
        assert np.array_equal(np_(got.m), g[f"{key}_m"]), key
        assert np.array_equal(np_(got.e), g[f"{key}_e"]), key


def test_mpf_elementwise_random_large(sb):
    from sdpvibe_b200.mpf import MPF, mul, add
    rng = np.random.default_rng(7)
    for L in (24, 26, 27):
        n = 100_000
        am, bm = rand_limbs(rng, L, n), rand_limbs(rng, L, n)
        ae, be = rng.integers(-500, 500, n), rng.integers(-500, 500, n)
        A, B = MPF(cu(am), cu(ae)), MPF(cu(bm), cu(be))
        m, e = O.mpf_mul(am, ae, bm, be)
        C = mul(A, B)
        assert np.array_equal(np_(C.m), m) and np.array_equal(np_(C.e), e)
        m, e = O.mpf_add(am, ae, bm, be, -1)
        C = add(A, B, -1)
        assert np.array_equal(np_(C.m), m) and np.array_equal(np_(C.e), e)


# ------------------------------------------------------------------ residues (a)
@pytest.mark.parametrize("name", golden_names("residues_"))
def test_residues_golden(sb, name):
    from sdpvibe_b200.mpmat import ctx
    g = golden(name)
    L = g["X"].shape[0]
    R = ctx(L)
    assert R.n == int(g["n"])
    for g0, G in ((0, R.n), (R.n - 16, 16)):
        hi, lo = R.residues(cu(g["X"]), int(g["k0"]), int(g["kc"]), g0, G)
        assert np.array_equal(np_(hi), g[f"hi_{g0}"])
        assert np.array_equal(np_(lo), g[f"lo_{g0}"])


@pytest.mark.parametrize("L,rows,K,k0,kc", [(24, 37, 700, 5, 651), (27, 274, 300, 0, 300), (26, 3, 4097, 1, 4096),
                                             (50, 9, 130, 2, 120), (64, 5, 64, 0, 64), (1, 11, 33, 0, 33)])
def test_residues_random(sb, L, rows, K, k0, kc):
    from sdpvibe_b200.mpmat import ctx
    rng = np.random.default_rng(L * 1000 + K)
    X = rng.integers(-(1 << 31), 1 << 31, size=(L, rows, K), dtype=np.int64).astype(np.int32)
    X[:, 0, :8] = 0
    X[-1, 0, 1] = -(1 << 31)
    T = O.tables(L)
    R = ctx(L)
    hi, lo = R.residues(cu(X), k0, kc)
    rh, rl = O.residues(T, X, k0, kc)
    assert np.array_equal(np_(hi), rh) and np.array_equal(np_(lo), rl)


# ------------------------------------------------------------------ residue GEMM (b), syrk (d)
@pytest.mark.parametrize("name", golden_names("accumulate_"))
def test_accumulate_golden(sb, name):
    from sdpvibe_b200.mpmat import ctx
    g = golden(name)
    R = ctx(int(name.split("L")[1]))
    acc = cu(g["acc0"]).clone()
    R.accumulate(cu(g["Ahi"]), cu(g["Alo"]), cu(g["Bhi"]), cu(g["Blo"]), acc, 0)
    assert np.array_equal(np_(acc), g["acc"])


def _rand_residues(rng, T, G, rows, K):
    m = T.m32[:G].astype(np.int64)[:, None, None]
    r = rng.integers(0, 1 << 30, size=(G, rows, K)) % m
    r = np.where(r > m // 2, r - m, r)
    lo = ((r + 64) & 127) - 64
    return ((r - lo) >> 7).astype(np.int8), lo.astype(np.int8)


@pytest.mark.parametrize("L,nb,M,N,K,syrk", [(24, 1, 256, 256, 256, False), (26, 1, 300, 129, 1024, False),
                                              (27, 1, 274, 274, 2000, True), (24, 3, 70, 45, 48, False),
                                              (10, 5, 33, 33, 16, True), (26, 2, 130, 7, 4096, False),
                                              # small blocks packed several to a tile
                                              (26, 7, 21, 5, 48, False), (26, 5, 64, 64, 128, False),
                                              (24, 9, 33, 60, 32, False), (34, 4, 32, 42, 48, False),
                                              (26, 13, 1, 9, 16, False),
                                              # syrk with a short last row block (tail items), and without
                                              (27, 2, 150, 150, 64, True), (26, 1, 160, 160, 128, True),
                                              (26, 1, 161, 161, 32, True), (27, 1, 290, 290, 48, True),
                                              # narrow items: one side <= 64 rows, the other longer
                                              (26, 3, 32, 300, 32, False), (26, 4, 64, 1000, 64, False),
                                              (24, 2, 17, 130, 208, False), (34, 2, 50, 90, 48, False),
                                              (26, 1, 64, 129, 4096, False), (26, 1, 1, 300, 16, False),
                                              (27, 3, 129, 33, 160, False), (26, 2, 300, 64, 16, False)])
def test_rns_gemm_random(sb, L, nb, M, N, K, syrk):
    from sdpvibe_b200.mpmat import ctx
    rng = np.random.default_rng(M * N + K)
    T = O.tables(L)
    R = ctx(L)
    Ah, Al = _rand_residues(rng, T, T.n, nb * M, K)
    Bh, Bl = (Ah, Al) if syrk else _rand_residues(rng, T, T.n, nb * (N if not syrk else M), K)
    m = T.m32.astype(np.int64)[:, None, None]
    acc0 = (rng.integers(0, 1 << 30, size=(T.n, nb * M, N)) % m).astype(np.int16)
    acc = cu(acc0).clone()
    R.accumulate(cu(Ah), cu(Al), cu(Bh), cu(Bl), acc, 0, nb=nb, syrk=syrk)
    got = np_(acc)
    for b in range(nb):
        sl = slice(b * M, (b + 1) * M)
        ref = O.accumulate(T, Ah[:, sl], Al[:, sl], Bh[:, b * N:(b + 1) * N] if not syrk else Ah[:, sl],
                           Bl[:, b * N:(b + 1) * N] if not syrk else Al[:, sl], acc0[:, sl], 0, lower=syrk)
        assert np.array_equal(got[:, sl], ref)


@pytest.mark.parametrize("nb,M,K,fresh,unsigned", [(1, 129, 16, False, False), (1, 274, 1008, True, True),
                                                   (2, 150, 48, True, False), (3, 288, 80, False, True),
                                                   (1, 400, 32, False, False), (2, 257, 400, True, True)])
def test_rns_gemm_syrk_fused_tail(sb, nb, M, K, fresh, unsigned):
    """syrk whose last row block has 1..32 rows: the tail rows against each full row block come out of the
    diagonal items (fused), the tail against itself out of the corner launch; fresh (no old residues read)
    and unsigned digits (mode bits 2 and 4) included"""
    from sdpvibe_b200.mpmat import ctx
    L = 26
    rng = np.random.default_rng(M + K + nb)
    T = O.tables(L)
    R = ctx(L)
    m = T.m32.astype(np.int64)[:, None, None]
    if unsigned:
        r = rng.integers(0, 1 << 30, size=(T.n, nb * M, K)) % m
        Ah, Al = (r >> 7).astype(np.uint8), (r & 127).astype(np.uint8)
    else:
        Ah, Al = _rand_residues(rng, T, T.n, nb * M, K)
    acc0 = (rng.integers(0, 1 << 30, size=(T.n, nb * M, M)) % m).astype(np.int16)
    acc = cu(acc0).clone()
    R.accumulate(cu(Ah), cu(Al), cu(Ah), cu(Al), acc, 0, nb=nb, syrk=True, fresh=fresh, unsigned=unsigned)
    got = np_(acc)
    low = np.tril(np.ones((M, M), dtype=bool))
    for b in range(nb):
        sl = slice(b * M, (b + 1) * M)
        base = np.zeros_like(acc0[:, sl]) if fresh else acc0[:, sl]
        ref = O.accumulate(T, Ah[:, sl].astype(np.int64), Al[:, sl].astype(np.int64), Ah[:, sl].astype(np.int64),
                           Al[:, sl].astype(np.int64), base, 0, lower=True)
        assert np.array_equal(got[:, sl][:, low], ref[:, low])
        assert np.array_equal(got[:, sl][:, ~low], acc0[:, sl][:, ~low])     # upper triangle untouched


@pytest.mark.parametrize("L,R,C", [(26, 300, 37), (26, 130, 5), (50, 200, 9), (26, 33000, 3), (26, 7, 1)])
def test_operand_rows_alignment_and_residues(sb, L, R, C):
    """GramAcc's operand rows: the bytes of the planar aligned limbs, the sign byte, zero padding rows; their
    residues equal the planar path's (unsigned digits), for both 128-entry K ranges of a 33000-row chunk"""
    from sdpvibe_b200.mpf import MPF, aligned, aligned_rows, top_max, NBITS, EZ
    from sdpvibe_b200.mpmat import ctx
    rng = np.random.default_rng(L + R + C)
    m = rand_limbs(rng, L, R * C).reshape(L, R, C)
    e = rng.integers(-8, 9, size=(R, C))
    m[:, 0, :] = 0
    e[0, :] = EZ                                                 # a zero row
    m[:, 1 % R, 0] = 0
    m[0, 1 % R, 0] = 5                                           # a short mantissa
    P = MPF(cu(m), cu(e))
    tp = top_max(P, over_rows=True)[0]
    target = (torch.where(tp > EZ // 2, tp, torch.zeros_like(tp)) - NBITS(L))[None, :]
    Lo = L + 1
    X = aligned(P, target, per_col=True, transpose=True, Lout=Lo).view(Lo, C, R)
    Rp = -(-R // 128) * 128
    Xr = aligned_rows(P, target, per_col=True, Lout=Lo, Rp=Rp)
    rb = Xr.shape[-1]
    assert rb == (128 if Lo <= 31 else 256)
    xr = np_(Xr).reshape(C, Rp, rb)
    xp = np_(X)                                                  # (Lo, C, R) int32
    limb_bytes = np.ascontiguousarray(np.moveaxis(xp, 0, -1)).view(np.uint8).reshape(C, R, 4 * Lo)
    assert np.array_equal(xr[:, :R, :4 * Lo], limb_bytes)
    assert np.array_equal(xr[:, :R, 4 * Lo], (xp[Lo - 1] < 0).astype(np.uint8))
    assert not xr[:, :R, 4 * Lo + 1:].any() and not xr[:, R:].any()
    Rc = ctx(Lo)
    for k0 in range(0, R, 32768):
        kc = min(32768, R - k0)
        gh, gl = Rc.residues_rows(Xr, C, Rp, k0, kc)
        wh, wl = Rc.residues(X, k0, kc, spread=True, unsigned=True)
        assert np.array_equal(np_(gh), np_(wh)) and np.array_equal(np_(gl), np_(wl)), k0


# ------------------------------------------------------------------ CRT (c)
@pytest.mark.parametrize("name", golden_names("crt_block_"))
def test_crt_block_golden(sb, name):
    from sdpvibe_b200.mpmat import ctx
    g = golden(name)
    R = ctx(int(name.split("L")[1]))
    acc = cu(g["acc"])
    for width in (1, 5, 11):
        W, bl, cnt = R.crt_block(acc, acc.shape[2], int(g["start"]), width, acc.shape[1])
        assert np.array_equal(np_(W), g[f"W_{width}"])
        assert np.array_equal(np_(bl), g[f"bl_{width}"])


@pytest.mark.parametrize("L", [24, 27, 34, 50])
def test_crt_norm_random(sb, L):
    from sdpvibe_b200.mpmat import ctx
    rng = random.Random(L)
    T = O.tables(L)
    R = ctx(L)
    rows, N = 37, 53
    lim = T.M // 4
    vals = [rng.randrange(-lim + 1, lim) >> rng.randrange(0, T.M.bit_length() - 3) for _ in range(rows * N)]
    vals[:6] = [0, 1, -1, lim - 1, -lim + 1, 1 << 77]
    acc = np.array([[v % p for v in vals] for p in T.mods], np.int16).reshape(T.n, rows, N)
    rowexp = np.array([rng.randrange(-900, 900) for _ in range(rows)], np.int64)
    colexp = np.array([rng.randrange(-900, 900) for _ in range(N)], np.int64)
    Wd, bl = O.crt_block(T, acc, N, 3, 41, rows)
    ein = (rowexp[:, None] + colexp[None, 3:44]).reshape(-1)
    rm, re_ = O.mpf_norm(Wd, ein, L)
    m, e = R.crt_norm(cu(acc), N, 3, 41, rows, cu(rowexp), cu(colexp), L)
    assert np.array_equal(np_(m), rm) and np.array_equal(np_(e), re_)
    W2, bl2, _ = R.crt_block(cu(acc), N, 3, 41, rows)
    assert np.array_equal(np_(W2), Wd) and np.array_equal(np_(bl2), bl)


# ------------------------------------------------------------------ composed paths
@pytest.mark.parametrize("name", golden_names("gemm_nt_L"))
def test_gemm_nt_golden(sb, name):
    from sdpvibe_b200.mpmat import MP, gemm_nt
    g = golden(name)
    mode = str(g["mode"])
    mode = int(mode) if mode.lstrip("-").isdigit() else mode
    C = gemm_nt(MP(cu(g["A"]), int(g["eA"])), MP(cu(g["B"]), int(g["eB"])), out_exp=mode)
    assert np.array_equal(np_(C.limbs), g["C"])
    assert np.array_equal(np.broadcast_to(np_(C.exp), g["Ce"].shape), g["Ce"])


@pytest.mark.parametrize("name", golden_names("gemm_nt_rowexp_"))
def test_gemm_nt_rowexp_golden(sb, name):
    from sdpvibe_b200.mpmat import MP, gemm_nt
    g = golden(name)
    C = gemm_nt(MP(cu(g["A"]), int(g["eA"])), MP(cu(g["B"]), 0), out_exp="col", bt_rowexp=cu(g["rowexp"]))
    assert np.array_equal(np_(C.limbs), g["C"]) and np.array_equal(np_(C.exp), g["Ce"])


@pytest.mark.parametrize("name", golden_names("mpf_gemm_"))
def test_mpf_gemm_golden(sb, name):
    from sdpvibe_b200.mpf import MPF, gemm
    g = golden(name)
    C = gemm(MPF(cu(g["Am"]), cu(g["Ae"])), MPF(cu(g["Bm"]), cu(g["Be"])), bool(g["tA"]), bool(g["tB"]))
    assert np.array_equal(np_(C.m), g["Cm"]) and np.array_equal(np_(C.e), g["Ce"])


def _lower(m, e):
    N = e.shape[-1]
    low = np.tril(np.ones((N, N), bool))
    return np.where(low, m, 0), np.where(low, e, 0)


@pytest.mark.parametrize("name", golden_names("gramacc_"))
def test_gramacc_golden(sb, name):
    from sdpvibe_b200.mpf import MPF, GramAcc
    g = golden(name)
    chunks = [MPF(cu(g[f"P{i}m"]), cu(g[f"P{i}e"])) for i in range(3) if f"P{i}m" in g]
    N, L = chunks[0].shape[1], chunks[0].L
    acc = GramAcc(N, L, E_ref=cu(g["Eref"]) if name == "gramacc_eref" else None)
    for c in chunks:
        acc.add(c)
    Q = acc.result()
    gm, ge = _lower(g["Qm"], g["Qe"])
    om, oe = _lower(np_(Q.m), np_(Q.e))
    assert np.array_equal(om, gm) and np.array_equal(oe, ge)
    assert acc.flushes == int(g["flushes"])


# ------------------------------------------------------------------ operand alignment
def _rand_mpf_np(rng, L, shape, lo=-40, hi=40, zero_frac=0.1):
    n = int(np.prod(shape))
    m = rng.integers(-(1 << 31), 1 << 31, size=(L, n), dtype=np.int64).astype(np.int32)
    e = rng.integers(lo, hi + 1, size=n).astype(np.int64)
    z = rng.random(n) < zero_frac
    m[:, z] = 0
    e[z] = O.EZ
    m, e = O.mpf_norm(m, e, L)
    e = np.where(z, O.EZ, e)
    return m.reshape((L,) + shape), e.reshape(shape)


@pytest.mark.parametrize("L,shape", [(26, (1, 300, 274)), (24, (3, 37, 50)), (27, (2, 16, 33))])
def test_top_max_and_align(sb, L, shape):
    from sdpvibe_b200.mpf import MPF, top_max, aligned
    rng = np.random.default_rng(L + shape[1])
    m, e = _rand_mpf_np(rng, L, shape)
    A = MPF(cu(m), cu(e))
    tp = OM.top(m, e)                                               # (nb, R, C)
    for over_rows in (True, False):
        ref = tp.max(axis=1 if over_rows else 2)
        assert np.array_equal(np_(top_max(A, over_rows)), ref)
    nb, R, C = shape
    for per_col in (False, True):
        target = rng.integers(-900, 900, size=(nb, C if per_col else R)).astype(np.int64)
        tgt_full = target[:, None, :] if per_col else target[:, :, None]
        s = np.where(e == O.EZ, 1 << 30, tgt_full - e).reshape(-1)
        for Lout in (L, L + 1):
            ref, _ = O.shift_round(m.reshape(L, -1), s, Lout)
            ref = ref.reshape((Lout,) + shape)
            for transpose in (False, True):
                got = np_(aligned(A, cu(target), per_col, transpose, Lout))
                want = np.swapaxes(ref, 2, 3) if transpose else ref
                assert np.array_equal(got, want), (per_col, transpose, Lout)


# ------------------------------------------------------------------ full-size configurations
def _normal_mpf_np(rng, L, shape, lo, hi):
    n = int(np.prod(shape))
    m = rng.integers(0, 1 << 32, size=(L, n), dtype=np.uint64).astype(np.uint32)
    m[L - 1] = (m[L - 1] & np.uint32((1 << 29) - 1)) | np.uint32(1 << 29)
    neg = rng.random(n) < 0.5
    m = m.view(np.int32).copy()
    val, _ = O.mpf_norm(m, np.zeros(n, np.int64), L)                    # normalised positive mantissas
    negm = O.add_same(np.zeros_like(val), val, -1)
    m = np.where(neg[None, :], negm, val)
    e = rng.integers(lo, hi + 1, size=n).astype(np.int64)
    return m.reshape((L,) + shape), e.reshape(shape)


def test_mpf_gemm_256_cube_L24(sb):
    """The mp-GEMM configuration: 256 x 256 x 256 at 768 bits, exponents U[-4, 4], bit-exact."""
    from sdpvibe_b200.mpf import MPF, gemm
    rng = np.random.default_rng(0)
    am, ae = _normal_mpf_np(rng, 24, (256, 256), -4, 4)
    bm, be = _normal_mpf_np(rng, 24, (256, 256), -4, 4)
    cm, ce = OM.mpf_gemm(am, ae, bm, be)
    C = gemm(MPF(cu(am), cu(ae)), MPF(cu(bm), cu(be)))
    assert np.array_equal(np_(C.m), cm) and np.array_equal(np_(C.e), ce)


def test_gramacc_chunking_invariance_full_size(sb):
    """The Gram configuration at full size (400 blocks, 274 columns, L = 26): with fixed reference
    exponents the residue accumulation is exact, so 4 chunks, 2 chunks and 1 chunk give identical Q."""
    from sdpvibe_b200.mpf import MPF, GramAcc, top_max
    rng = np.random.default_rng(0)
    rows = rng.integers(20, 121, size=400)
    R = int(rows.sum())
    m = torch.randint(-(1 << 31), (1 << 31) - 1, (26, R, 274), dtype=torch.int32, device="cuda")
    m[-1] = (m[-1] & ((1 << 29) - 1)) | (1 << 29)
    e = torch.randint(-8, 9, (R, 274), dtype=torch.int64, device="cuda")
    P = MPF(m, e)
    Eref = top_max(P, over_rows=True)[0] + 4
    cuts = np.cumsum(rows)
    results = []
    for nch in (4, 2, 1):
        bounds = [0] + [int(cuts[len(rows) * (c + 1) // nch - 1]) for c in range(nch)]
        acc = GramAcc(274, 26, E_ref=Eref)
        for a, b in zip(bounds[:-1], bounds[1:]):
            acc.add(MPF(m[:, a:b].contiguous(), e[a:b].contiguous()))
        Q = acc.result()
        assert acc.flushes == 0
        low = torch.tril(torch.ones(274, 274, dtype=torch.bool, device="cuda"))
        results.append((torch.where(low, Q.m, 0), torch.where(low, Q.e, 0)))
    for r in results[1:]:
        assert torch.equal(r[0], results[0][0]) and torch.equal(r[1], results[0][1])


# ------------------------------------------------------------------ Cholesky / trsm (e)
@pytest.mark.parametrize("name", golden_names("basecase_"))
def test_basecase_tile_golden(sb, name):
    from sdpvibe_b200.mpmat import MP
    from sdpvibe_b200.basecase import chol_inv_tile
    g = golden(name)
    L = g["A"].shape[0]
    Lg, Xg = chol_inv_tile(MP(cu(g["A"]), -(32 * L - 40)))
    assert np.array_equal(np_(Lg.limbs), g["L"])
    assert np.array_equal(np_(Xg.limbs), g["X"])
    assert np.array_equal(np.broadcast_to(np_(Xg.exp), g["Xe"].shape), g["Xe"])


@pytest.mark.parametrize("name", golden_names("chol_"))
def test_chol_and_solves_golden(sb, name):
    from sdpvibe_b200.mpf import MPF, Chol
    g = golden(name)
    ch = Chol(MPF(cu(g["Am"]), cu(g["Ae"])))
    assert np.array_equal(np_(ch.k), g["k"])
    assert np.array_equal(np_(ch.Lt.limbs), g["Lt"])
    for i, t in enumerate(ch.tiles):
        assert np.array_equal(np_(t.X.limbs), g[f"X{i}m"]) and np.array_equal(np_(t.X.exp), g[f"X{i}e"])
    B = MPF(cu(g["Bm"]), cu(g["Be"]))
    for key, fn in (("lo", ch.solve_lower), ("up", ch.solve_upper), ("x", ch.solve)):
        R = fn(B)
        assert np.array_equal(np_(R.m), g[f"{key}_m"]), key
        assert np.array_equal(np_(R.e), g[f"{key}_e"]), key


@pytest.mark.parametrize("L,nb,n,nr", [(24, 5, 96, 8), (26, 3, 160, 8), (24, 7, 17, 3)])
def test_chol_random_vs_oracle(sb, L, nb, n, nr):
    """Batched Cholesky + both solves on SPD blocks G G^T + n I (scaled rows), against the oracle."""
    from sdpvibe_b200.mpf import MPF, Chol
    rng = np.random.default_rng(n + nb)
    vals, exps = [], []
    for b in range(nb):
        G = rng.integers(-40, 41, size=(n, n)).astype(object)
        d = rng.integers(-20, 21, size=n)
        A = G.dot(G.T) + np.eye(n, dtype=object) * (50 * n)
        for i in range(n):
            for j in range(n):
                vals.append(int(A[i, j]))
                exps.append(int(d[i] + d[j]))
    m, e = O.mpf_norm(O.to_limbs(vals, L), np.array(exps, np.int64), L)
    Am, Ae = m.reshape(L, nb, n, n), e.reshape(nb, n, n)
    Bm, Be = _normal_mpf_np(rng, L, (nb, n, nr), -20, 20)
    ref = OM.Chol(Am, Ae)
    ch = Chol(MPF(cu(Am), cu(Ae)))
    assert np.array_equal(np_(ch.Lt.limbs), ref.Lt)
    B = MPF(cu(Bm), cu(Be))
    for (rm, re_), got in ((ref.solve_lower(Bm, Be), ch.solve_lower(B)), (ref.solve(Bm, Be), ch.solve(B))):
        assert np.array_equal(np_(got.m), rm) and np.array_equal(np_(got.e), re_)


def test_from_float_matches_oracle(sb):
    from sdpvibe_b200.mpf import from_float
    rs = np.random.default_rng(7)
    V = rs.standard_normal((3, 5, 5)) * 2.0 ** np.random.default_rng(8).integers(-900, 900, (3, 5, 5))
    V[0, 0, 0] = 0
    V[1, 0, :] = [5e-324, -2.5e-310, -0.0, 1.7976931348623157e308, -1.0]      # subnormals, -0, extremes
    for L in (2, 26, 40):
        got = from_float(V, L)
        rm, re_ = OM.mpf_from_float(V, L)
        assert np.array_equal(np_(got.m), rm) and np.array_equal(np_(got.e), re_)


def test_cholsolve_buckets_vs_oracle(sb):
    """The batched Cholesky + solve workload (SPD blocks of uneven size grouped by padded size, identity
    padding) on a few blocks, bit-exact against the oracle per bucket."""
    from sdpvibe_b200 import mpf
    from sdpvibe_b200.kernel_bench import cholsolve_inputs, cholsolve_buckets
    cases = cholsolve_inputs(6, 8, 70, 8, seed=3)
    for npad, idx, A, B in cholsolve_buckets(cases, 26):
        X = mpf.Chol(A).solve(B)
        ref = OM.Chol(np_(A.m), np_(A.e))
        rm, re_ = ref.solve(np_(B.m), np_(B.e))
        assert np.array_equal(np_(X.m), rm) and np.array_equal(np_(X.e), re_), npad
        # the solution solves the float64 system to double accuracy
        for q, i in enumerate(idx):
            n, Ai, Bi = cases[i]
            xf = mpf.MPF(X.m[:, q, :n], X.e[q, :n]).to_float()
            assert np.allclose(Ai @ xf, Bi, rtol=0, atol=1e-9)


def test_chol_solve_many_matches_sequential(sb):
    """the buckets' systems on concurrent streams give the bits of the same calls one after the other"""
    from sdpvibe_b200 import mpf
    from sdpvibe_b200.kernel_bench import cholsolve_inputs, cholsolve_buckets
    buckets = cholsolve_buckets(cholsolve_inputs(40, 8, 160, 8, seed=4), 26)
    seq = [mpf.Chol(A).solve(B) for _, _, A, B in buckets]
    for _ in range(2):                                          # eager, then graph replays
        got = mpf.chol_solve_many([(A, B) for _, _, A, B in buckets])
        for X, Y in zip(got, seq):
            assert torch.equal(X.m, Y.m) and torch.equal(X.e, Y.e)


def _spd_tiles(rng, nb, L, ill):
    """nb random 32 x 32 SPD tiles in wide fixed point (WL = L + 24 words, F = 32 L fraction bits),
    entry-major (nb, 32, 32, WL) uint32; diagonal below 1.  ill: columns of the generator scaled by
    2^-e, e up to 8 L bits, so pivots get tiny and the pivot reciprocals and the inverse get large."""
    WL, F = L + 24, 32 * L
    out = np.zeros((nb, 32, 32, WL), np.uint32)
    for b in range(nb):
        G = [[int(v) for v in row] for row in rng.integers(-(1 << 20), 1 << 20, size=(32, 32))]
        ex = [int(v) for v in rng.integers(0, 8 * L if ill else 4, size=32)]
        emax = 2 * max(ex)
        A = [[sum(G[i][k] * G[j][k] << (emax - 2 * ex[k]) for k in range(32)) for j in range(32)] for i in range(32)]
        if not ill:
            for i in range(32):
                A[i][i] += 1 << (emax + 30)
        s = max(A[i][i] for i in range(32)).bit_length() + 1
        for i in range(32):
            for j in range(32):
                v = A[i][j]
                v = (v << (F - s)) if F >= s else (v >> (s - F))
                u = v % (1 << (32 * WL))
                out[b, i, j] = [(u >> (32 * w)) & 0xffffffff for w in range(WL)]
    return out


@pytest.mark.parametrize("L", [8, 26, 40, 44])
@pytest.mark.parametrize("ill", [False, True])
def test_tile_kernels_vs_oracle(sb, L, ill):
    """sdpv_chol_tiles / sdpv_trinv_tiles on random SPD tiles against the oracle, bit for bit: the
    shared-memory kernels (WL <= 64) and the global-memory kernels (WL > 64), well and ill conditioned."""
    from sdpvibe_b200 import _lib
    rng = np.random.default_rng(L * 7 + ill)
    nb, WL, LF = 3, L + 24, L
    W = _spd_tiles(rng, nb, L, ill)
    RA, RR = O.chol_tiles(W, 32, WL, LF)
    A = cu(W.view(np.int32))
    RINV = torch.zeros((nb, 32, WL), dtype=torch.int32, device="cuda")
    _lib.call("sdpv_chol_tiles", _lib.ptr(A), _lib.ptr(RINV), nb, 32, WL, LF, _lib.stream())
    got = np_(A).view(np.uint32)
    tri = np.tril(np.ones((32, 32), bool))
    assert np.array_equal(got[:, tri], RA[:, tri])
    assert np.array_equal(np_(RINV).view(np.uint32), RR)
    Lw = np.where(tri[None, :, :, None], RA, 0).astype(np.uint32)
    RX = O.trinv_tiles(Lw, RR, 32, WL, LF)
    X = torch.empty_like(A)
    S = torch.empty_like(A)
    _lib.call("sdpv_trinv_tiles", _lib.ptr(cu(Lw.view(np.int32))), _lib.ptr(RINV), _lib.ptr(X), _lib.ptr(S), nb, 32,
              WL, LF, _lib.stream())
    assert np.array_equal(np_(X).view(np.uint32), RX)


def test_chol_graph_replay_matches_eager(sb):
    """Chol + solves replayed from CUDA graphs (same shapes, new data each call) give the eager bits,
    and a result stays valid while the same graph runs again."""
    from sdpvibe_b200 import graphs
    from sdpvibe_b200.mpf import MPF, Chol
    rng = np.random.default_rng(77)
    L, nb, n, nr = 26, 3, 70, 5

    def case():
        vals, exps = [], []
        for b in range(nb):
            G = rng.integers(-40, 41, size=(n, n)).astype(object)
            A = G.dot(G.T) + np.eye(n, dtype=object) * (50 * n)
            vals += [int(v) for v in A.reshape(-1)]
            exps += [int(x) for x in rng.integers(-5, 6, size=n * n)]
        m, e = O.mpf_norm(O.to_limbs(vals, L), np.array(exps, np.int64), L)
        Bm, Be = _normal_mpf_np(rng, L, (nb, n, nr), -20, 20)
        return MPF(cu(m.reshape(L, nb, n, n)), cu(e.reshape(nb, n, n))), MPF(cu(Bm), cu(Be))
    cases = [case() for _ in range(3)]
    graphs.clear()
    graphs.ENABLED = False
    try:
        eager = []
        for A, B in cases:
            ch = Chol(A)
            eager.append((np_(ch.Lt.limbs), ch.solve_lower(B), ch.solve(B)))
    finally:
        graphs.ENABLED = True
    kept = []
    for (A, B), (lt, lo, x) in zip(cases, eager):
        ch = Chol(A)
        got_lo, got_x = ch.solve_lower(B), ch.solve(B)
        assert np.array_equal(np_(ch.Lt.limbs), lt)
        for got, ref in ((got_lo, lo), (got_x, x)):
            assert np.array_equal(np_(got.m), np_(ref.m)) and np.array_equal(np_(got.e), np_(ref.e))
        kept.append((got_x, x))
    for got, ref in kept:                           # earlier results untouched by later replays
        assert np.array_equal(np_(got.m), np_(ref.m)) and np.array_equal(np_(got.e), np_(ref.e))
    assert len(graphs._cache) >= 3
    graphs.clear()


def test_trsv_tiles_vs_oracle(sb):
    """sdpv_trsv_tiles (substitution with one factored tile, one warp per vector) against the oracle, both
    words-per-lane instantiations."""
    from sdpvibe_b200 import _lib
    rng = np.random.default_rng(5)
    for L in (8, 26, 40, 44):                       # WL 68 > 64: three words per lane
        WL, LF = L + 24, L
        W = _spd_tiles(rng, 1, L, False)
        RA, RR = O.chol_tiles(W, 32, WL, LF)
        tri = np.tril(np.ones((32, 32), bool))
        Lw = np.where(tri[None, :, :, None], RA, 0).astype(np.uint32)[0]
        V = rng.integers(0, 1 << 32, size=(9, 32, WL), dtype=np.uint64).astype(np.uint32)
        V[..., LF + 1:] = np.where(V[..., LF:LF + 1] >> 31, np.uint32(0xffffffff), np.uint32(0))   # |v| < 2^32
        ref = O.trsv_tiles(Lw, RR[0], V, 32, WL, LF)
        Vd = cu(V.view(np.int32))
        _lib.call("sdpv_trsv_tiles", _lib.ptr(cu(Lw.view(np.int32))), _lib.ptr(cu(RR[0].view(np.int32))),
                  _lib.ptr(Vd), V.shape[0], 32, WL, LF, _lib.stream())
        assert np.array_equal(np_(Vd).view(np.uint32), ref)


@pytest.mark.skipif("linalg_n96" not in golden_names("linalg"), reason="fixture not generated")
def test_linalg_golden(sb):
    """linalg.chol (both panel leaves, refinement), trsm_left (both leaves), chol_inv + trsm and
    basecase.trsv_tile bit-exact against the reference's own linalg run (tests/golden: linalg_n96)."""
    from sdpvibe_b200 import linalg, basecase
    from sdpvibe_b200.mpmat import MP
    g = golden("linalg_n96")
    A = MP(cu(g["Am"]), int(g["Ae"]))
    B = MP(cu(g["Bm"]), cu(g["Be"]))
    Ls, ts = linalg.chol(A, tile_inverses=True, panel_leaf="subst")
    assert np.array_equal(np_(Ls.limbs), g["Ls"]) and Ls.uniform_exp() == int(g["Ls_e"])
    Lg, _ = linalg.chol(A, tile_inverses=True, panel_leaf="gemm", refine=1)
    assert np.array_equal(np_(Lg.limbs), g["Lg"]) and Lg.uniform_exp() == int(g["Lg_e"])
    for leaf in ("gemm", "subst"):
        P = linalg.trsm_left(Ls, B, ts, leaf=leaf)
        assert np.array_equal(np_(P.limbs), g[f"P_{leaf}_m"]) and np.array_equal(np_(P.exp), g[f"P_{leaf}_e"]), leaf
    Lc, Xc = linalg.chol_inv(A)
    assert np.array_equal(np_(Lc.limbs), g["Lc"]) and Lc.uniform_exp() == int(g["Lc_e"])
    assert np.array_equal(np_(Xc.limbs), g["Xc"]) and Xc.uniform_exp() == int(g["Xc_e"])
    P2 = linalg.trsm(Xc, B)
    assert np.array_equal(np_(P2.limbs), g["P2_m"]) and np.array_equal(np_(P2.exp), g["P2_e"])
    assert np.array_equal(np_(ts[0].Lw).view(np.uint32), g["t0_Lw"].view(np.uint32))
    Y, ye = basecase.trsv_tile(ts[0], cu(g["Vm"]), cu(g["ve"]))
    assert np.array_equal(np_(Y), g["Ym"]) and np.array_equal(np_(ye), g["ye"])
    Yf, yfe = basecase.trsv_tile(ts[0], cu(g["Vm"]), cu(g["ve"]), out_exp=-(32 * 8 - 40))
    assert np.array_equal(np_(Yf), g["Yfm"]) and np.array_equal(np_(yfe), g["yfe"])


@pytest.mark.parametrize("nb,M,N,K", [(1, 200, 130, 64), (6, 32, 42, 32), (3, 100, 7, 48), (5, 32, 1000, 32),
                                      (2, 48, 200, 96)])
def test_rns_gemm_fresh_overwrites(sb, nb, M, N, K):
    """fresh mode: the accumulator's previous content is ignored (overwritten with the product residues)."""
    from sdpvibe_b200.mpmat import ctx
    rng = np.random.default_rng(nb + M + N)
    L = 26
    T = O.tables(L)
    R = ctx(L)
    Ah, Al = _rand_residues(rng, T, T.n, nb * M, K)
    Bh, Bl = _rand_residues(rng, T, T.n, nb * N, K)
    acc = cu((rng.integers(0, 30000, size=(T.n, nb * M, N))).astype(np.int16))      # garbage
    R.accumulate(cu(Ah), cu(Al), cu(Bh), cu(Bl), acc, 0, nb=nb, fresh=True)
    got = np_(acc)
    zero = np.zeros((T.n, M, N), np.int16)
    for b in range(nb):
        sl = slice(b * M, (b + 1) * M)
        ref = O.accumulate(T, Ah[:, sl], Al[:, sl], Bh[:, b * N:(b + 1) * N], Bl[:, b * N:(b + 1) * N], zero, 0)
        assert np.array_equal(got[:, sl], ref)


def test_tuning_knobs_do_not_change_results(sb):
    """every value of the launch-shape knobs gives the same bits: narrow items on or off, packing on or
    off, CRT CTAs per SM"""
    from sdpvibe_b200.autotune import set_knob, get_knob
    from sdpvibe_b200.mpmat import ctx
    L = 26
    rng = np.random.default_rng(12)
    T = O.tables(L)
    R = ctx(L)
    saved = {k: get_knob(k) for k in ("crt_ctas", "narrow_max", "pack_max")}
    try:
        for nb, M, N, K in ((4, 32, 300, 32), (6, 32, 40, 48)):
            Ah, Al = _rand_residues(rng, T, T.n, nb * M, K)
            Bh, Bl = _rand_residues(rng, T, T.n, nb * N, K)
            outs = []
            for nm, pm in ((64, 64), (0, 0), (32, 32)):
                set_knob("narrow_max", nm)
                set_knob("pack_max", pm)
                acc = torch.zeros((T.n, nb * M, N), dtype=torch.int16, device="cuda")
                R.accumulate(cu(Ah), cu(Al), cu(Bh), cu(Bl), acc, nb=nb, fresh=True)
                outs.append(np_(acc))
            assert all(np.array_equal(outs[0], o) for o in outs[1:])
        m = T.m32.astype(np.int64)[:, None, None]
        acc = cu((rng.integers(0, 1 << 30, size=(T.n, 70, 90)) % m).astype(np.int16))
        got = []
        for c in (1, 2, 3, 4):
            set_knob("crt_ctas", c)
            W, bl, _ = R.crt_block(acc, 90, 0, 90, 70)
            got.append((np_(W), np_(bl)))
        assert all(np.array_equal(got[0][0], g[0]) and np.array_equal(got[0][1], g[1]) for g in got[1:])
    finally:
        for k, v in saved.items():
            set_knob(k, v)


@pytest.mark.parametrize("L,rows,K", [(27, 274, 1000), (50, 9, 132), (26, 3, 4097), (50, 17, 4000), (27, 5, 2048)])
def test_decomposition_reducer_warps(sb, L, rows, K):
    """8 and 16 reducer warps of the decomposition kernel give the oracle's residues (API digits) and its
    canonical residues (unsigned digits)"""
    from sdpvibe_b200.autotune import set_knob, get_knob
    from sdpvibe_b200.mpmat import ctx
    rng = np.random.default_rng(L + rows + K)
    T = O.tables(L)
    R = ctx(L)
    X = rand_limbs(rng, L, rows * K).reshape(L, rows, K)
    X[:, 0, :5] = 0
    X[-1, 0, 5] = -(1 << 31)
    X[:, 0, 6] = -1
    rh, rl = O.residues(T, X, 1, K - 1)
    rh0, rl0 = O.residues(T, X, 0, K)
    m = T.m32.astype(np.int64)[:, None, None]
    rc = (128 * rh.astype(np.int64) + rl) % m
    # the same entries as operand rows (limb bytes, sign byte, zero rows up to a multiple of 128)
    Rp = -(-(K - 1) // 128) * 128
    Xr = np.zeros((rows, Rp, 128 if L <= 31 else 256), np.uint8)
    xs = X[:, :, 1:]
    Xr[:, :K - 1, :4 * L] = np.ascontiguousarray(np.moveaxis(xs, 0, -1)).view(np.uint8).reshape(rows, K - 1, 4 * L)
    Xr[:, :K - 1, 4 * L] = (xs[L - 1] < 0)
    saved = get_knob("res_warps")
    try:
        for w in (8, 16):
            set_knob("res_warps", w)
            hi, lo = R.residues(cu(X), 1, K - 1)
            assert np.array_equal(np_(hi), rh) and np.array_equal(np_(lo), rl), w
            uh, ul = R.residues(cu(X), 1, K - 1, spread=True, unsigned=True)
            kk = rc.shape[2]
            assert np.array_equal(np_(uh)[:, :, :kk], (rc >> 7).astype(np.uint8)), w
            assert np.array_equal(np_(ul)[:, :, :kk], (rc & 127).astype(np.uint8)), w
            vh, vl = R.residues_rows(cu(Xr), rows, Rp, 0, K - 1)
            assert np.array_equal(np_(vh), np_(uh)) and np.array_equal(np_(vl), np_(ul)), w
            # k0 = 0 and 16-byte aligned rows: the limb planes come in by TMA
            hi0, lo0 = R.residues(cu(X), 0, K)
            assert np.array_equal(np_(hi0), rh0) and np.array_equal(np_(lo0), rl0), w
    finally:
        set_knob("res_warps", saved)



@pytest.mark.parametrize("L,rows,K", [(27, 274, 300), (24, 37, 700), (26, 5, 4096)])
def test_unsigned_digit_residues_and_gemm(sb, L, rows, K):
    """the GEMM's internal digit format: canonical residues r in [0, m) as hi = r >> 7, lo = r & 127 equal the
    oracle's residues; their products (mode bit 2) equal the oracle's, also as syrk"""
    from sdpvibe_b200.mpmat import ctx
    rng = np.random.default_rng(L + rows)
    T = O.tables(L)
    R = ctx(L)
    X = rand_limbs(rng, L, rows * K).reshape(L, rows, K)
    rh, rl = O.residues(T, X, 0, K)                                  # centred (API) digits
    m = T.m32.astype(np.int64)[:, None, None]
    rc = ((128 * rh.astype(np.int64) + rl) % m)[:, :, :K]
    Uh, Ul = R.residues(cu(X), 0, K, spread=True, unsigned=True)
    assert np.array_equal(np_(Uh)[:, :, :K], (rc >> 7).astype(np.uint8))
    assert np.array_equal(np_(Ul)[:, :, :K], (rc & 127).astype(np.uint8))
    M = min(rows, 60)
    acc0 = (rng.integers(0, 1 << 30, size=(T.n, M, M)) % m).astype(np.int16)
    for syrk in (False, True):
        acc = cu(acc0).clone()
        A_h, A_l = Uh[:, :M].contiguous(), Ul[:, :M].contiguous()
        R.accumulate(A_h, A_l, A_h, A_l, acc, syrk=syrk, unsigned=True)
        ref = O.accumulate(T, np_(A_h), np_(A_l), np_(A_h), np_(A_l), acc0, 0, lower=syrk)
        assert np.array_equal(np_(acc), ref), syrk
