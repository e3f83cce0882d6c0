// SDPB's binary number records (boost-serialised El::BigFloat over GMP mpf_t limbs) to and from MPF limb
// planes (sdpvibe/_bigfloat.c:1-111).
//
// Record: byte is_zero; unless zero, int32 size, int64 exp and nl little-endian 64-bit limbs; value =
// sign(size) M 2^(64 (exp - |size|)), M = the first |size| limbs.  Records have two lengths (1 or 13 + 8 nl
// bytes), so their offsets come from one sequential pass over the zero flags on the host
// (sdpv_bigfloat_index); the bit work is one GPU thread per record:
//   sdpv_bigfloat_unpack: records -> planar (L, n) limbs, M rounded half up to at most 32 L - 2 bits
//                         (shift s), exponent 64 (exp - |size|) + s, zeros -> 0 / EZ
//   sdpv_bigfloat_pack:   planar limbs -> records at given offsets (the exponent's residue mod 64 moved
//                         into the mantissa, |size| = the 64-bit limbs used); a mantissa needing more than
//                         nl limbs sets the overflow bit and is written as a zero record
#include <cstring>

#include "common.cuh"

namespace {
using namespace sdpv;

constexpr int kThreads = 128;
constexpr int kMaxW = 2 * 64 + 2;          // 32-bit words of a record mantissa (nl <= 64)
constexpr int kMaxL = 64;

__device__ __forceinline__ u64 ld64(const uint8_t* p) {      // unaligned little-endian load
  u64 v = 0;
  for (int k = 7; k >= 0; k--) v = (v << 8) | p[k];
  return v;
}
__device__ __forceinline__ void st64(uint8_t* p, u64 v) {
  for (int k = 0; k < 8; k++) p[k] = (uint8_t)(v >> (8 * k));
}

__global__ void __launch_bounds__(kThreads) unpack_kernel(const uint8_t* __restrict__ buf, const i64* __restrict__ offs,
                                                          i64 n, int nl, int L, int32_t* __restrict__ out,
                                                          i64* __restrict__ exps) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint8_t* p = buf + offs[i];
  u32 r[kMaxL + 1];
  for (int k = 0; k <= L; k++) r[k] = 0;
  i64 ex = SDPV_EZ;
  if (!p[0]) {
    const int size = (int)(u32)ld64(p + 1);                   // low 4 bytes: int32 size
    const i64 exp = (i64)ld64(p + 5);
    const int asz = min(size < 0 ? -size : size, nl);       // |size| <= nl (checked by the index pass)
    u32 w[kMaxW];
    for (int k = 0; k < 2 * asz; k += 2) {
      const u64 d = ld64(p + 13 + 4 * k);
      w[k] = (u32)d;
      w[k + 1] = (u32)(d >> 32);
    }
    int top = 2 * asz - 1;
    while (top >= 0 && w[top] == 0) top--;
    if (top >= 0) {
      const int bl = 32 * top + 32 - __clz(w[top]);
      const int T = 32 * L - 2;
      const int s = bl > T ? bl - T : 0;
      const int q = s >> 5, b = s & 31;
      for (int k = 0; k <= L; k++) {                          // M >> s, then + the bit below (half up)
        const u32 lo = q + k <= top ? w[q + k] : 0u, hi = q + k + 1 <= top ? w[q + k + 1] : 0u;
        r[k] = b ? (lo >> b) | (hi << (32 - b)) : lo;
      }
      if (s > 0 && ((w[(s - 1) >> 5] >> ((s - 1) & 31)) & 1u))
        for (int k = 0; k <= L; k++)
          if (++r[k] != 0) break;
      if (size < 0) {
        u32 c = 1;
        for (int k = 0; k < L; k++) {
          const u32 t = ~r[k] + c;
          c = (c && t == 0) ? 1u : 0u;
          r[k] = t;
        }
      }
      ex = 64 * (exp - asz) + s;
    }
  }
  for (int k = 0; k < L; k++) out[(i64)k * n + i] = (int32_t)r[k];
  exps[i] = ex;
}

__global__ void __launch_bounds__(kThreads) pack_kernel(const int32_t* __restrict__ m, const i64* __restrict__ e, i64 n,
                                                        int L, int nl, const i64* __restrict__ offs,
                                                        uint8_t* __restrict__ out, unsigned* __restrict__ err) {
  const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint8_t* p = out + offs[i];
  u32 a[kMaxL + 2];
  for (int k = 0; k < L; k++) a[k] = (u32)m[(i64)k * n + i];
  a[L] = a[L + 1] = 0;
  const bool neg = (int32_t)a[L - 1] < 0;
  if (neg) {
    u32 c = 1;
    for (int k = 0; k < L; k++) {
      const u32 t = ~a[k] + c;
      c = (c && t == 0) ? 1u : 0u;
      a[k] = t;
    }
  }
  int top = L - 1;
  while (top >= 0 && a[top] == 0) top--;
  const i64 ev = e[i];
  if (top < 0 || ev == SDPV_EZ) {
    p[0] = 1;
    return;
  }
  const int rr = (int)(((ev % 64) + 64) % 64);               // value = (|M| << rr) 2^(64 base)
  const i64 base = (ev - rr) / 64;
  const int q = rr >> 5, b = rr & 31;
  u32 d[kMaxW];
  for (int k = 0; k < 2 * nl + 2; k++) d[k] = 0;
  for (int k = 0; k <= top + 1; k++) {                       // words of |M| << rr
    const u32 lo = a[k], prev = k > 0 ? a[k - 1] : 0u;
    if (k + q < 2 * nl + 2) d[k + q] = b ? (lo << b) | (prev >> (32 - b)) : lo;
  }
  int dtop = 2 * nl + 1;
  while (dtop >= 0 && d[dtop] == 0) dtop--;
  const int size = dtop / 2 + 1;                              // 64-bit limbs used
  if (size > nl || top + 1 + q >= 2 * nl + 2) {
    atomicOr(err, SDPV_ERRBIT_OVERFLOW);
    p[0] = 1;
    return;
  }
  p[0] = 0;
  const u32 ssize = (u32)(neg ? -size : size);
  for (int k = 0; k < 4; k++) p[1 + k] = (uint8_t)(ssize >> (8 * k));
  st64(p + 5, (u64)(base + size));
  for (int k = 0; k < nl; k++) st64(p + 13 + 8 * k, (u64)d[2 * k] | ((u64)d[2 * k + 1] << 32));
}

}  // namespace

extern "C" int sdpv_bigfloat_index(const uint8_t* buf, int64_t len, int64_t pos, int64_t n, int nl, int64_t* offsets,
                                   int64_t* end) {
  if (!buf || !offsets || !end || pos < 0 || n < 0 || nl < 1 || nl > 64) return SDPV_EINVAL;
  const i64 rec = 13 + 8 * (i64)nl;
  for (i64 i = 0; i < n; i++) {
    if (pos >= len) return SDPV_EINVAL;                       // truncated
    offsets[i] = pos;
    if (buf[pos]) {
      pos += 1;
      continue;
    }
    if (pos + rec > len) return SDPV_EINVAL;
    int32_t size;
    memcpy(&size, buf + pos + 1, 4);
    if (size > nl || size < -nl) return SDPV_EINVAL;          // corrupt
    pos += rec;
  }
  *end = pos;
  return SDPV_OK;
}

extern "C" int sdpv_bigfloat_unpack(const uint8_t* buf, const int64_t* offsets, int64_t n, int nl, int L, int32_t* out,
                                    int64_t* exps, void* stream) {
  if (n < 0 || nl < 1 || nl > 64 || L < 1 || L > kMaxL) return SDPV_EINVAL;
  if (n == 0) return SDPV_OK;
  unpack_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, sdpv::as_stream(stream)>>>(
      buf, offsets, n, nl, L, out, exps);
  return sdpv::launch_status();
}

extern "C" int sdpv_bigfloat_pack(const int32_t* m, const int64_t* e, int64_t n, int L, int nl, const int64_t* offsets,
                                  uint8_t* out, void* stream) {
  if (n < 0 || nl < 1 || nl > 64 || L < 1 || L > kMaxL) return SDPV_EINVAL;
  if (n == 0) return SDPV_OK;
  pack_kernel<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, sdpv::as_stream(stream)>>>(
      m, e, n, L, nl, offsets, out, sdpv::device_error_word());
  return sdpv::launch_status();
}
