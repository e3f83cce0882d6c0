// Magnitude helpers shared by the MPF kernels (limbops.cu) and the fused CRT epilogue (crt.cu).
#pragma once
#include "common.cuh"

namespace sdpv {
__device__ __forceinline__ void neg_words(u32* a, int n) {
  u32 c = 1;
  for (int k = 0; k < n; k++) {
    u32 t = ~a[k] + c;
    c = (c && t == 0) ? 1u : 0u;
    a[k] = t;
  }
}
__device__ __forceinline__ int bitlen_mag(const u32* a, int n) {
  for (int k = n - 1; k >= 0; k--)
    if (a[k]) return 32 * k + 32 - __clz(a[k]);
  return 0;
}
// Magnitude shift: round half up (s > 0, carry kept in nd words) or exact left shift: mpf.py:36-56.
__device__ __forceinline__ void mag_shift(const u32* src, int ns, int s, u32* dst, int nd) {
  if (s > 0) {
    int q = s >> 5, r = s & 31;
    for (int k = 0; k < nd; k++) {
      u64 lo = (q + k < ns) ? src[q + k] : 0u, hi = (q + k + 1 < ns) ? src[q + k + 1] : 0u;
      dst[k] = (u32)(((hi << 32) | lo) >> r);
    }
    int qb = (s - 1) >> 5, rb = (s - 1) & 31;
    u32 c = (qb < ns) ? ((src[qb] >> rb) & 1u) : 0u;
    for (int k = 0; k < nd && c; k++) {
      u32 t = dst[k] + c;
      c = (t == 0) ? 1u : 0u;
      dst[k] = t;
    }
  } else {
    int t = -s, q = t >> 5, r = t & 31;
    for (int k = 0; k < nd; k++) {
      int i0 = k - q, i1 = k - q - 1;
      u64 lo = (i0 >= 0 && i0 < ns) ? src[i0] : 0u, lo2 = (i1 >= 0 && i1 < ns) ? src[i1] : 0u;
      dst[k] = (u32)((((lo << 32) | lo2) << r) >> 32);
    }
  }
}

// MPF product r = a b of two's-complement L-word mantissas with exponents (magnitude rounded half up to
// NB = 32L-2 bits; zero -> EZ): the arithmetic of mpf_mul (mpf.py:58-89) on registers / local arrays.
template <int LMAX>
__device__ __forceinline__ void mpf_mul_dev(const u32* ain, i64 ea, const u32* bin, i64 eb, int L, u32* r,
                                            i64& er) {
  u32 a[LMAX], b[LMAX], p[2 * LMAX];
  for (int k = 0; k < L; k++) {
    a[k] = ain[k];
    b[k] = bin[k];
  }
  const bool na = a[L - 1] >> 31, nb = b[L - 1] >> 31;
  if (na) neg_words(a, L);
  if (nb) neg_words(b, L);
  if (!bitlen_mag(a, L) || !bitlen_mag(b, L)) {
    for (int k = 0; k < L; k++) r[k] = 0;
    er = SDPV_EZ;
    return;
  }
  u64 carry = 0, hprev = 0;                          // product by output columns, one carry pass
  for (int k = 0; k < 2 * L - 1; k++) {
    u64 slo = 0, shi = 0;
    int x0 = k - L + 1 > 0 ? k - L + 1 : 0, x1 = k < L - 1 ? k : L - 1;
    for (int x = x0; x <= x1; x++) {
      u64 pr = (u64)a[x] * b[k - x];
      slo += (u32)pr;
      shi += pr >> 32;
    }
    u64 sum = slo + hprev + carry;
    p[k] = (u32)sum;
    carry = sum >> 32;
    hprev = shi;
  }
  p[2 * L - 1] = (u32)(hprev + carry);
  const int s = bitlen_mag(p, 2 * L) - (32 * L - 2);
  mag_shift(p, 2 * L, s, r, L);
  if (na != nb) neg_words(r, L);
  er = ea + eb + s;
}

// MPF sum r = a + sgn b (operands aligned at max exponent - 32 in L+2 words, then renormalised with the
// magnitude rounded half up): the arithmetic of mpf_add (mpf.py:92-124).  r may alias a or b.
template <int LMAX>
__device__ __forceinline__ void mpf_add_dev(const u32* ain, i64 ea, const u32* bin, i64 eb, int sgn, int L, u32* r,
                                            i64& er) {
  u32 a[LMAX], b[LMAX], wa[LMAX + 2], wb[LMAX + 2];
  for (int k = 0; k < L; k++) {
    a[k] = ain[k];
    b[k] = bin[k];
  }
  const bool na = a[L - 1] >> 31;
  const bool nbs = (b[L - 1] >> 31) ^ (sgn < 0);
  if (a[L - 1] >> 31) neg_words(a, L);
  if (b[L - 1] >> 31) neg_words(b, L);
  if (!bitlen_mag(a, L)) ea = SDPV_EZ;
  if (!bitlen_mag(b, L)) eb = SDPV_EZ;
  if (ea == SDPV_EZ && eb == SDPV_EZ) {
    for (int k = 0; k < L; k++) r[k] = 0;
    er = SDPV_EZ;
    return;
  }
  const int far = 32 * (L + 3);
  const i64 t = (ea > eb ? ea : eb) - 32;
  const i64 da = ea - t, db = eb - t;
  const int sa = (da < -(i64)far) ? far : (int)(-da);
  const int sb = (db < -(i64)far) ? far : (int)(-db);
  if (ea == SDPV_EZ) {
    for (int k = 0; k < L + 2; k++) wa[k] = 0;
  } else {
    mag_shift(a, L, sa, wa, L + 2);
  }
  if (eb == SDPV_EZ) {
    for (int k = 0; k < L + 2; k++) wb[k] = 0;
  } else {
    mag_shift(b, L, sb, wb, L + 2);
  }
  if (na) neg_words(wa, L + 2);
  if (nbs) neg_words(wb, L + 2);
  u64 c = 0;
  for (int k = 0; k < L + 2; k++) {
    u64 v = (u64)wa[k] + wb[k] + c;
    wa[k] = (u32)v;
    c = v >> 32;
  }
  const bool ns = wa[L + 1] >> 31;
  if (ns) neg_words(wa, L + 2);
  const int bl = bitlen_mag(wa, L + 2);
  if (!bl) {
    for (int k = 0; k < L; k++) r[k] = 0;
    er = SDPV_EZ;
    return;
  }
  const int s = bl - (32 * L - 2);
  mag_shift(wa, L + 2, s, r, L);
  if (ns) neg_words(r, L);
  er = t + s;
}

}  // namespace sdpv
