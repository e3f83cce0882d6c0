"""The decomposition kernel's integer arithmetic, restated in numpy on the CPU (no GPU): the bound that keeps
its u8 x u8 table product below 2^31, the exact Barrett quotient it uses for the canonical residue, and the
byte-permute split of four residues into unsigned digits.  The kernel's results are checked against the
oracle on the GPU (test_gpu_kernels.py); these tests pin the arithmetic argument those results rely on."""
import numpy as np
import pytest

import oracle as O


def _byte_perm_6420(a, b):
    """__byte_perm(a, b, 0x6420): bytes 0 and 2 of a, then bytes 0 and 2 of b"""
    return (a & 0xFF) | (((a >> 16) & 0xFF) << 8) | ((b & 0xFF) << 16) | (((b >> 16) & 0xFF) << 24)


@pytest.mark.parametrize("L", [1, 24, 26, 27, 31, 50, 63])
def test_unsigned_table_product_fits_31_bits(L):
    """v = 128 D_hi + D_lo over 4L limb bytes and one sign byte, every byte and digit at its maximum, stays
    below 2^31 (the kernel's Barrett range) for every L the warp-specialised kernel serves (L <= 63)"""
    mods = O.tables(L).m32.astype(np.int64)
    assert mods.min() > (1 << 14) and mods.max() < (1 << 15)
    t = mods - 1                                          # largest canonical table entry
    v_max = (4 * L + 1) * 255 * (128 * (t >> 7) + (t & 127))
    assert v_max.max() < (1 << 31)


@pytest.mark.parametrize("L", [26, 27, 50])
def test_barrett_quotient_is_exact(L):
    """floor(v ceil(2^46/m) / 2^46) = floor(v/m) for 0 <= v < 2^31 and every modulus of the context: random v,
    the multiples of m and their neighbours, and the top of the range"""
    rng = np.random.default_rng(L)
    for m in O.tables(L).m32.astype(np.int64):
        bm = ((1 << 46) + m - 1) // m
        assert bm < (1 << 32)
        k = rng.integers(0, (1 << 31) // m, size=200)
        v = np.concatenate([rng.integers(0, 1 << 31, size=2000), k * m, k * m - 1, k * m + m - 1,
                            np.array([0, 1, m - 1, m, (1 << 31) - 1])])
        v = v[(v >= 0) & (v < (1 << 31))].astype(object)      # Python integers: no 64-bit overflow
        q = [((int(x) * int(bm)) >> 32) >> 14 for x in v]
        assert q == [int(x) // int(m) for x in v]


def test_digit_split_by_byte_permutes():
    """four residues r < 2^15 packed as two 16-bit pairs: hi = r >> 7 from bytes 0 / 2 of (pair >> 7), lo =
    r & 127 from bytes 0 / 2 of the pair masked to 7 bits"""
    rng = np.random.default_rng(0)
    r = rng.integers(0, 1 << 15, size=(100_000, 4)).astype(np.uint64)
    r[:4] = [[0, 0, 0, 0], [32766, 32767, 1, 127], [128, 255, 256, 16383], [16384, 32512, 127, 128]]
    p01, p23 = r[:, 0] + (r[:, 1] << 16), r[:, 2] + (r[:, 3] << 16)
    hi = _byte_perm_6420(p01 >> 7, p23 >> 7)
    lo = _byte_perm_6420(p01, p23) & 0x7F7F7F7F
    for u in range(4):
        assert np.array_equal((hi >> (8 * u)) & 0xFF, r[:, u] >> 7)
        assert np.array_equal((lo >> (8 * u)) & 0xFF, r[:, u] & 127)


@pytest.mark.parametrize("L", [26, 50])
def test_unsigned_table_reproduces_the_residue(L):
    """the unsigned formulation, restated: sum_j u_j (256^j mod m) + neg ((-2^(32L)) mod m) = x (mod m) for
    two's-complement limbs, and it agrees with the oracle's residues"""
    rng = np.random.default_rng(L + 1)
    T = O.tables(L)
    n = 300
    X = rng.integers(-(1 << 31), 1 << 31, size=(L, 1, n), dtype=np.int64).astype(np.int32)
    X[:, 0, 0] = -1
    X[:, 0, 1] = 0
    X[-1, 0, 2] = -(1 << 31)
    rh, rl = O.residues(T, X, 0, n)
    ref = (128 * rh.astype(np.int64) + rl)[:, 0, :n]
    by = np.ascontiguousarray(X[:, 0, :].T).view(np.uint8).reshape(n, 4 * L).astype(object)
    neg = (X[-1, 0, :] < 0)
    for g in range(0, T.n, 17):
        m = int(T.m32[g])
        tab = [pow(256, j, m) for j in range(4 * L)]
        sgn = (m - pow(2, 32 * L, m)) % m
        v = [sum(int(b) * t for b, t in zip(row, tab)) + (sgn if ng else 0) for row, ng in zip(by, neg)]
        assert [x % m for x in v] == [int(x) % m for x in ref[g]]


def _magic_quotient(v, minv_f32):
    """the residue GEMM's rounded quotient: __float_as_int(fmaf((float)v, minv, 12582912.0f)) - 0x4B400000,
    i.e. (float)v (round to nearest even) times the float 1/m, plus 1.5 2^23 with one rounding to a float
    whose unit is 1 -- computed here exactly with fractions and rounded half to even"""
    from fractions import Fraction
    fv = Fraction(float(np.float32(v)))
    s = fv * Fraction(float(minv_f32))                       # the fma's exact product; the magic adds 1.5 2^23
    q = s.numerator // s.denominator                         # floor, then round half to even
    rem = s - q
    if rem > Fraction(1, 2) or (rem == Fraction(1, 2) and q % 2):
        q += 1
    return q


@pytest.mark.parametrize("L", [26, 27])
def test_float_rounded_quotient_needs_one_correction(L):
    """The narrow residue-GEMM epilogue reduces v (|v| < 2^31) by q = round(v / m) taken from the float
    estimate above and applies a single correction (add m when negative).  That is exact when v - q m lies in
    (-m, m/2 + m/64]: checked for every modulus of the context on random v over the whole range, on the
    multiples of m and their half-way neighbours, and at the range's ends"""
    rng = np.random.default_rng(L)
    for m in O.tables(L).m32.astype(np.int64)[::3]:
        minv = np.float32(1.0 / float(m))
        k = rng.integers(-((1 << 31) // m), (1 << 31) // m, size=40)
        v = np.concatenate([rng.integers(-(1 << 31) + 1, 1 << 31, size=120), k * m, k * m + m // 2,
                            k * m + (m + 1) // 2, k * m - m // 2,
                            np.array([0, 1, -1, m // 2, -(m // 2), (1 << 31) - 1, -(1 << 31) + 1])])
        v = v[(v > -(1 << 31)) & (v < (1 << 31))]
        for x in v.tolist():
            r = x - _magic_quotient(x, minv) * int(m)
            assert -int(m) < r <= int(m) // 2 + int(m) // 64
            r += int(m) if r < 0 else 0
            assert r == x % int(m)
