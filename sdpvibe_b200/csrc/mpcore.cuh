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

}  // namespace sdpv
