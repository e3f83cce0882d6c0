// Cholesky base case on CUDA cores: 32 x 32 tiles in wide fixed point.
//
// A tile entry is WL 32-bit words (two's complement) with F = 32*LF fraction bits; tiles are entry-major
// (tiles, 32, 32, WL), the layout of sdpvibe/basecase.py.  The arithmetic is the reference's, so results
// are bit-identical (sdpvibe/basecase.py:31-226):
//   * fx product: |a| * |b| summed by product columns from column max(LF-2, la+lb) upward (columns below
//     are never formed), exact carries, words >= LF kept (truncation), sign applied last; t > 0 keeps only
//     the top t words of each operand;
//   * d^-1/2: double seed 1/sqrt(d) converted exactly, then r += r (1 - d r^2) / 2 with products truncated
//     to the top 100, 200, 400, ... bits until full width;
//   * Cholesky by columns (pivot, column scaled by the pivot reciprocal, trailing update of the lower
//     triangle); inverse X = L^-1 row by row with the pivot reciprocals.
// One CTA (256 threads) per tile.  The Newton steps run warp-cooperatively (each lane forms product
// columns, lane 0 carries); column scaling and the trailing update give one product to each thread.
#include <cmath>
#include <mutex>

#include "common.cuh"

namespace {

constexpr int BT = 32;
constexpr int kThreads = 256;
constexpr int WMAX = 96;                  // WL <= 96 (L <= 72)

__device__ __forceinline__ int top_word(const u32* a, int WL) {
  for (int i = WL - 1; i > 0; i--)
    if (a[i]) return i;
  return 0;
}

__device__ __forceinline__ void negate_words(u32* a, int n) {
  u32 c = 1;
  for (int k = 0; k < n; k++) {
    u32 t = ~a[k] + c;
    c = (c && t == 0) ? 1u : 0u;
    a[k] = t;
  }
}

// Column sums of x * y restricted to i in [la, ta], j in [lb, tb], from column kmin; carried into r
// (words LF .. LF+WL-1).  Pure function of the magnitudes, shared by the thread and warp versions.
__device__ __forceinline__ void column_sum(const u32* x, const u32* y, int k, int la, int ta, int lb, int tb,
                                           u64& lo, u64& hi) {
  lo = 0;
  hi = 0;
  int i0 = max(la, k - tb), i1 = min(ta, k - lb);
  for (int i = i0; i <= i1; i++) {
    u64 p = (u64)x[i] * y[k - i];
    lo += (u32)p;
    hi += p >> 32;
  }
}

// r = (a * b) >> F truncated (thread-serial); r may alias a or b.
__device__ void fx_mul(u32* r, const u32* a, const u32* b, int t, int WL, int LF) {
  u32 x[WMAX], y[WMAX];
  for (int i = 0; i < WL; i++) {
    x[i] = a[i];
    y[i] = b[i];
  }
  const bool sa = x[WL - 1] >> 31, sb = y[WL - 1] >> 31;
  if (sa) negate_words(x, WL);
  if (sb) negate_words(y, WL);
  const int ta = top_word(x, WL), tb = top_word(y, WL);
  const int la = t ? max(0, ta - t + 1) : 0, lb = t ? max(0, tb - t + 1) : 0;
  const int kmin = max(LF - 2, la + lb), kmax = ta + tb;
  for (int i = 0; i < WL; i++) r[i] = 0;
  u64 carry = 0, hprev = 0;
  for (int k = kmin; k <= kmax + 2 && k < LF + WL; k++) {
    u64 lo = 0, hi = 0;
    if (k <= kmax) column_sum(x, y, k, la, ta, lb, tb, lo, hi);
    u64 s = lo + hprev + carry;
    if (k >= LF) r[k - LF] = (u32)s;
    carry = s >> 32;
    hprev = hi;
  }
  if (sa ^ sb) negate_words(r, WL);
}

// Warp-cooperative version: operands and result in shared memory (r must not alias a or b);
// sx, sy: WL words of scratch, col: 2*(2*WL+4) u64.
__device__ void fx_mul_warp(u32* r, const u32* a, const u32* b, int t, int WL, int LF, u32* sx, u32* sy, u64* col) {
  const int lane = threadIdx.x & 31;
  for (int i = lane; i < WL; i += 32) {
    sx[i] = a[i];
    sy[i] = b[i];
  }
  __syncwarp();
  const bool sa = sx[WL - 1] >> 31, sb = sy[WL - 1] >> 31;
  __syncwarp();
  if (lane == 0) {
    if (sa) negate_words(sx, WL);
    if (sb) negate_words(sy, WL);
  }
  __syncwarp();
  const int ta = top_word(sx, WL), tb = top_word(sy, WL);
  const int la = t ? max(0, ta - t + 1) : 0, lb = t ? max(0, tb - t + 1) : 0;
  const int kmin = max(LF - 2, la + lb), kmax = ta + tb;
  for (int k = kmin + lane; k <= kmax; k += 32) {
    u64 lo, hi;
    column_sum(sx, sy, k, la, ta, lb, tb, lo, hi);
    col[2 * (k - kmin)] = lo;
    col[2 * (k - kmin) + 1] = hi;
  }
  for (int i = lane; i < WL; i += 32) r[i] = 0;
  __syncwarp();
  if (lane == 0) {
    u64 carry = 0, hprev = 0;
    for (int k = kmin; k <= kmax + 2 && k < LF + WL; k++) {
      u64 lo = 0, hi = 0;
      if (k <= kmax) {
        lo = col[2 * (k - kmin)];
        hi = col[2 * (k - kmin) + 1];
      }
      u64 s = lo + hprev + carry;
      if (k >= LF) r[k - LF] = (u32)s;
      carry = s >> 32;
      hprev = hi;
    }
    if (sa ^ sb) negate_words(r, WL);
  }
  __syncwarp();
}

__device__ double fx_to_double(const u32* a, int WL, int LF) {
  u32 x[WMAX];
  for (int i = 0; i < WL; i++) x[i] = a[i];
  const bool s = x[WL - 1] >> 31;
  if (s) negate_words(x, WL);
  const int t = top_word(x, WL);
  double v = (double)x[t];
  if (t >= 1) v = v * 4294967296.0 + (double)x[t - 1];
  if (t >= 2) v = v * 4294967296.0 + (double)x[t - 2];
  v = ldexp(v, 32 * max(t - 2, 0) - 32 * LF);
  return s ? -v : v;
}

__device__ void fx_from_double(u32* r, double v, int WL, int LF) {   // v > 0
  for (int i = 0; i < WL; i++) r[i] = 0;
  int e;
  const double m = frexp(v, &e);
  u64 mi = (u64)ldexp(m, 53);
  int pos = e - 53 + 32 * LF;
  if (pos < 0) {
    mi = (-pos < 64) ? (mi >> (-pos)) : 0ull;
    pos = 0;
  }
  const int li = pos / 32, sh = pos % 32;
  u64 lo = mi << sh, hi = sh ? (mi >> (64 - sh)) : 0ull;       // 96-bit window mi << sh
  u32 w[4] = {(u32)lo, (u32)(lo >> 32), (u32)hi, (u32)(hi >> 32)};
  for (int k = 0; k < 4 && li + k < WL; k++) r[li + k] = w[k];
}

// ---- batched Cholesky of 32 x 32 tiles, in place (lower), plus the pivot reciprocals
__global__ void __launch_bounds__(kThreads) chol_tiles_kernel(u32* __restrict__ A, u32* __restrict__ RINV, int WL,
                                                              int LF, unsigned* __restrict__ err) {
  __shared__ u32 sd[WMAX], sr[WMAX], st1[WMAX], st2[WMAX], sone[WMAX], sx[WMAX], sy[WMAX];
  __shared__ u64 scol[2 * (2 * WMAX + 4)];
  u32* T = A + (size_t)blockIdx.x * BT * BT * WL;
  u32* RI = RINV + (size_t)blockIdx.x * BT * WL;
  const int tid = threadIdx.x, lane = tid & 31;
#define AT(i, j) (T + ((size_t)(i) * BT + (j)) * WL)
  for (int k = 0; k < BT; k++) {
    if (tid < 32) {
      for (int i = lane; i < WL; i += 32) sd[i] = AT(k, k)[i];
      __syncwarp();
      if (lane == 0) {
        if ((sd[WL - 1] >> 31) || top_word(sd, WL) == 0 && sd[0] == 0) atomicOr(err, SDPV_ERRBIT_NOTSPD);
        fx_from_double(sr, 1.0 / sqrt(fx_to_double(sd, WL, LF)), WL, LF);
        for (int i = 0; i < WL; i++) sone[i] = 0;
        sone[LF] = 1;
      }
      __syncwarp();
      for (int bits = 100;; bits *= 2) {                 // r <- r + r (1 - d r^2) / 2
        int t = bits / 32 + 2;
        if (t >= WL) t = 0;
        fx_mul_warp(st1, sr, sr, t, WL, LF, sx, sy, scol);
        fx_mul_warp(st2, st1, sd, t, WL, LF, sx, sy, scol);
        if (lane == 0) {
          i64 br = 0;                                     // st1 = 1 - st2
          for (int i = 0; i < WL; i++) {
            i64 v = (i64)sone[i] - (i64)st2[i] + br;
            st1[i] = (u32)v;
            br = v >> 32;
          }
        }
        __syncwarp();
        fx_mul_warp(st2, sr, st1, t, WL, LF, sx, sy, scol);
        if (lane == 0) {
          for (int i = 0; i < WL - 1; i++) st2[i] = (st2[i] >> 1) | (st2[i + 1] << 31);
          st2[WL - 1] = (u32)(((int32_t)st2[WL - 1]) >> 1);
          u64 c = 0;
          for (int i = 0; i < WL; i++) {
            u64 v = (u64)sr[i] + st2[i] + c;
            sr[i] = (u32)v;
            c = v >> 32;
          }
        }
        __syncwarp();
        if (t == 0) break;
      }
      fx_mul_warp(st1, sd, sr, 0, WL, LF, sx, sy, scol);  // l_kk = d * d^-1/2
      for (int i = lane; i < WL; i += 32) {
        AT(k, k)[i] = st1[i];
        RI[(size_t)k * WL + i] = sr[i];
      }
    }
    __syncthreads();
    const u32* rk = RI + (size_t)k * WL;
    for (int i = k + 1 + tid; i < BT; i += kThreads) fx_mul(AT(i, k), AT(i, k), rk, 0, WL, LF);
    __syncthreads();
    const int m = BT - k - 1, npairs = m * (m + 1) / 2;
    for (int p = tid; p < npairs; p += kThreads) {
      int ii = (int)((sqrtf(8.f * p + 1.f) - 1.f) * 0.5f);
      while ((ii + 1) * (ii + 2) / 2 <= p) ii++;
      while (ii * (ii + 1) / 2 > p) ii--;
      const int i = k + 1 + ii, j = k + 1 + (p - ii * (ii + 1) / 2);
      u32 v[WMAX];
      fx_mul(v, AT(i, k), AT(j, k), 0, WL, LF);
      u32* aij = AT(i, j);
      i64 br = 0;
      for (int w = 0; w < WL; w++) {
        i64 d = (i64)aij[w] - (i64)v[w] + br;
        aij[w] = (u32)d;
        br = d >> 32;
      }
    }
    __syncthreads();
  }
#undef AT
}

// ---- batched inverse X = L^-1 of lower tiles (upper part of Lt must be zero), row by row:
// x_ii = 1/l_ii, x_ik = -(1/l_ii) sum_{j=k}^{i-1} l_ij x_jk.  S: per-tile scratch for the products.
__global__ void __launch_bounds__(kThreads) trinv_tiles_kernel(const u32* __restrict__ Lt, const u32* __restrict__ RINV,
                                                               u32* __restrict__ X, u32* __restrict__ S, int WL, int LF) {
  const size_t tsz = (size_t)BT * BT * WL;
  const u32* T = Lt + blockIdx.x * tsz;
  const u32* RI = RINV + (size_t)blockIdx.x * BT * WL;
  u32* XT = X + blockIdx.x * tsz;
  u32* SC = S + blockIdx.x * tsz;                        // SC[k][j] = l_ij x_jk for the current row i
  const int tid = threadIdx.x;
  for (size_t w = tid; w < tsz; w += kThreads) XT[w] = 0;
  __syncthreads();
  for (int i = 0; i < BT; i++) {
    const int np = i * (i + 1) / 2;                      // pairs k <= j < i
    for (int p = tid; p < np; p += kThreads) {
      int j = (int)((sqrtf(8.f * p + 1.f) - 1.f) * 0.5f);
      while ((j + 1) * (j + 2) / 2 <= p) j++;
      while (j * (j + 1) / 2 > p) j--;
      const int k = p - j * (j + 1) / 2;
      fx_mul(SC + ((size_t)k * BT + j) * WL, T + ((size_t)i * BT + j) * WL, XT + ((size_t)j * BT + k) * WL, 0, WL,
             LF);
    }
    __syncthreads();
    for (int k = tid; k <= i; k += kThreads) {
      u32* xik = XT + ((size_t)i * BT + k) * WL;
      if (k == i) {
        for (int w = 0; w < WL; w++) xik[w] = RI[(size_t)i * WL + w];
        continue;
      }
      u32 acc[WMAX];
      for (int w = 0; w < WL; w++) acc[w] = 0;
      for (int j = k; j < i; j++) {
        const u32* s = SC + ((size_t)k * BT + j) * WL;
        u64 c = 0;
        for (int w = 0; w < WL; w++) {
          u64 v = (u64)acc[w] + s[w] + c;
          acc[w] = (u32)v;
          c = v >> 32;
        }
      }
      fx_mul(acc, acc, RI + (size_t)i * WL, 0, WL, LF);
      negate_words(acc, WL);
      for (int w = 0; w < WL; w++) xik[w] = acc[w];
    }
    __syncthreads();
  }
}


// ================================================================ shared-memory tile kernels (WL <= 64)
// The same arithmetic as the kernels above, organised for latency: the tile lives in shared memory,
// serial products (Newton, pivot-column scaling, the row sums of the inverse) run warp-cooperatively with
// one product column per lane and carries resolved by warp ballots, and the bulk products (trailing update,
// inverse row products) run one per thread on 96-bit column accumulators (mad.cc carry chains) straight
// from shared-memory magnitudes.  Every product is the same truncated product (same columns, same kept
// words), and sums of products are exact in WL words, so the results are bit-identical to the kernels above.
constexpr int FW = 64;                    // fast path: WL <= FW
constexpr int kThreadsS = 512;            // shared-memory kernels: 16 warps per tile
constexpr int kWarpsS = kThreadsS / 32;
constexpr unsigned kFull = 0xffffffffu;

struct WarpScratch {                      // per-warp product scratch
  u32 xa[FW], xb[FW], acc[FW];
};

// c += d (96-bit)
__device__ __forceinline__ void add96(u32& c0, u32& c1, u32& c2, u32 d0, u32 d1, u32 d2) {
  asm("add.cc.u32 %0, %0, %3;\n\t"
      "addc.cc.u32 %1, %1, %4;\n\t"
      "addc.u32 %2, %2, %5;"
      : "+r"(c0), "+r"(c1), "+r"(c2)
      : "r"(d0), "r"(d1), "r"(d2));
}

// Exact 96-bit sum of x[i] y[k - i] over i0 <= i <= i1, added to (c0, c1, c2): two interleaved
// accumulators (independent carry chains) and the loads of four terms issued ahead of their products.
__device__ __forceinline__ void column96(u32& c0, u32& c1, u32& c2, const u32* x, const u32* y, int k, int i0,
                                         int i1);

__device__ __forceinline__ void mac96(u32& c0, u32& c1, u32& c2, u32 x, u32 y) {
  asm("mad.lo.cc.u32 %0, %3, %4, %0;\n\t"
      "madc.hi.cc.u32 %1, %3, %4, %1;\n\t"
      "addc.u32 %2, %2, 0;"
      : "+r"(c0), "+r"(c1), "+r"(c2)
      : "r"(x), "r"(y));
}

__device__ __forceinline__ void column96(u32& c0, u32& c1, u32& c2, const u32* x, const u32* y, int k, int i0,
                                         int i1) {
  // four independent carry chains (the sum is exact whatever the grouping), loads of eight terms ahead
  u32 d0 = 0, d1 = 0, d2 = 0, e0 = 0, e1 = 0, e2 = 0, f0 = 0, f1 = 0, f2 = 0;
  int i = i0;
  for (; i + 7 <= i1; i += 8) {
    u32 a[8], b[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      a[u] = x[i + u];
      b[u] = y[k - i - u];
    }
    mac96(c0, c1, c2, a[0], b[0]);
    mac96(d0, d1, d2, a[1], b[1]);
    mac96(e0, e1, e2, a[2], b[2]);
    mac96(f0, f1, f2, a[3], b[3]);
    mac96(c0, c1, c2, a[4], b[4]);
    mac96(d0, d1, d2, a[5], b[5]);
    mac96(e0, e1, e2, a[6], b[6]);
    mac96(f0, f1, f2, a[7], b[7]);
  }
  if (i + 3 <= i1) {
    const u32 a0 = x[i], a1 = x[i + 1], a2 = x[i + 2], a3 = x[i + 3];
    const u32 b0 = y[k - i], b1 = y[k - i - 1], b2 = y[k - i - 2], b3 = y[k - i - 3];
    mac96(c0, c1, c2, a0, b0);
    mac96(d0, d1, d2, a1, b1);
    mac96(e0, e1, e2, a2, b2);
    mac96(f0, f1, f2, a3, b3);
    i += 4;
  }
  for (; i <= i1; i++) mac96(c0, c1, c2, x[i], y[k - i]);
  add96(d0, d1, d2, f0, f1, f2);
  add96(c0, c1, c2, e0, e1, e2);
  add96(c0, c1, c2, d0, d1, d2);
}


// Carry into this lane of a 32-lane digit chain: g = this lane's digit overflowed (carry out whatever
// comes in), p = this lane's digit is all ones (passes a carry on).  cin: carry into lane 0; cout: carry
// out of lane 31.  g and p are never both set.  With X = G|P and Y = G as 32-bit numbers, the internal
// carries of X + Y + cin are exactly the chain's carries.
__device__ __forceinline__ u32 chain_carry(bool g, bool p, u32 cin, u32& cout) {
  const unsigned G = __ballot_sync(kFull, g), P = __ballot_sync(kFull, p);
  const unsigned X = G | P;
  const u64 sum = (u64)X + G + cin;
  cout = (u32)(sum >> 32);
  return (((u32)sum ^ X ^ G) >> (threadIdx.x & 31)) & 1u;
}

// Words lane and lane+32 of a two's-complement WL-word number negated (mod 2^(32 WL)): ~x plus a carry that
// enters word w when every lower word is zero.
__device__ __forceinline__ void warp_negate(u32& v0, u32& v1, int WL) {
  const int lane = threadIdx.x & 31;
  const unsigned lower = (1u << lane) - 1u;
  const unsigned nz0 = __ballot_sync(kFull, lane < WL && v0 != 0);
  const unsigned nz1 = __ballot_sync(kFull, lane + 32 < WL && v1 != 0);
  v0 = ~v0 + (((nz0 & lower) == 0) ? 1u : 0u);
  v1 = ~v1 + ((nz0 == 0 && (nz1 & lower) == 0) ? 1u : 0u);
}

__device__ __forceinline__ int warp_top(u32 v0, u32 v1, int WL) {
  const int lane = threadIdx.x & 31;
  const unsigned b0 = __ballot_sync(kFull, lane < WL && v0 != 0);
  const unsigned b1 = __ballot_sync(kFull, lane + 32 < WL && v1 != 0);
  return b1 ? 63 - __clz(b1) : (b0 ? 31 - __clz(b0) : 0);
}

// Magnitude of a two's-complement WL-word operand (shared or global memory) into m[0..WL); returns its sign,
// top = index of its highest nonzero word (0 for zero).  Warp-collective.
__device__ __forceinline__ int load_mag(const u32* src, u32* m, int WL, int& top) {
  const int lane = threadIdx.x & 31;
  const int sign = (int)(src[WL - 1] >> 31);
  u32 v0 = lane < WL ? src[lane] : 0u, v1 = lane + 32 < WL ? src[lane + 32] : 0u;
  if (sign) warp_negate(v0, v1, WL);
  if (lane < WL) m[lane] = v0;
  if (lane + 32 < WL) m[lane + 32] = v1;
  top = warp_top(v0, v1, WL);
  return sign;
}

// Warp-cooperative truncated product a * b >> F (top t words of each operand when t > 0): one product
// column per lane, columns kmin .. min(kmax + 2, LF + WL - 1), each a 96-bit exact sum; the column sums are
// added with their 32- and 64-bit shifts and the carries resolved by chain_carry.  Outputs (any may be
// null): out = signed result (may alias a or b), omag = magnitude, *osign / *otop (written by lane 0).
__device__ void wmul(const u32* a, const u32* b, int t, int WL, int LF, WarpScratch& s, u32* out, u32* omag,
                     uint8_t* osign, uint8_t* otop) {
  const int lane = threadIdx.x & 31;
  int ta, tb;
  const int sa = load_mag(a, s.xa, WL, ta);
  const int sb = load_mag(b, s.xb, WL, tb);
  __syncwarp();
  s.acc[lane] = 0;
  s.acc[lane + 32] = 0;
  const int la = t ? max(0, ta - t + 1) : 0, lb = t ? max(0, tb - t + 1) : 0;
  const int kmin = max(LF - 2, la + lb), kmax = ta + tb;
  const int ncol = min(kmax + 2, LF + WL - 1) - kmin + 1;
  __syncwarp();
  u32 p_c1 = 0, p_c2a = 0, p_c2b = 0, p_h = 0, cin = 0;          // carried over from the previous 32 columns
  for (int q0 = 0; q0 < ncol; q0 += 32) {
    const int q = q0 + lane, k = kmin + q;
    u32 c0 = 0, c1 = 0, c2 = 0;
    if (q < ncol && k <= kmax) column96(c0, c1, c2, s.xa, s.xb, k, max(la, k - tb), min(ta, k - lb));
    u32 c1u = __shfl_up_sync(kFull, c1, 1), c2u = __shfl_up_sync(kFull, c2, 2);
    if (lane == 0) c1u = p_c1;
    if (lane == 0) c2u = p_c2a;
    if (lane == 1) c2u = p_c2b;
    const u32 n_c1 = __shfl_sync(kFull, c1, 31), n_c2a = __shfl_sync(kFull, c2, 30), n_c2b = __shfl_sync(kFull, c2, 31);
    const u64 v = (u64)c0 + c1u + c2u;                                 // < 3 * 2^32
    const u32 lo = (u32)v, h = (u32)(v >> 32);
    u32 hu = __shfl_up_sync(kFull, h, 1);
    if (lane == 0) hu = p_h;
    const u32 n_h = __shfl_sync(kFull, h, 31);
    const u32 e = lo + hu;
    u32 cout;
    const u32 cj = chain_carry(e < lo, e == kFull, cin, cout);
    const int w = k - LF;
    if (q < ncol && w >= 0 && w < WL) s.acc[w] = e + cj;
    p_c1 = n_c1;
    p_c2a = n_c2a;
    p_c2b = n_c2b;
    p_h = n_h;
    cin = cout;
  }
  __syncwarp();
  u32 m0 = lane < WL ? s.acc[lane] : 0u, m1 = lane + 32 < WL ? s.acc[lane + 32] : 0u;
  const int sg = sa ^ sb;
  if (omag) {
    if (lane < WL) omag[lane] = m0;
    if (lane + 32 < WL) omag[lane + 32] = m1;
  }
  if (otop) {
    const int tp = warp_top(m0, m1, WL);
    if (lane == 0) *otop = (uint8_t)tp;
  }
  if (osign && lane == 0) *osign = (uint8_t)sg;
  if (out) {
    if (sg) warp_negate(m0, m1, WL);
    if (lane < WL) out[lane] = m0;
    if (lane + 32 < WL) out[lane + 32] = m1;
  }
  __syncwarp();
}

// dst (two's complement, WL words) += trunc(|x| |y|) if add, else -= ; x, y magnitudes with tops tx, ty.
// Columns from LF - 2 (t = 0 products), product scanning on a 96-bit accumulator; the kept words are
// added into dst as they come out, then the carry (borrow) runs up until it dies.  One thread.
__device__ void fx_rmw(u32* dst, const u32* x, int tx, const u32* y, int ty, bool add, int WL, int LF) {
  const int kmin = LF - 2, kmax = tx + ty;
  u32 c0 = 0, c1 = 0, c2 = 0, cy = 0;
  int w = 0;
  auto emit = [&](u32 d) {
    if (w < WL) {
      const u32 o = dst[w];
      if (add) {
        const u64 r = (u64)o + d + cy;
        dst[w] = (u32)r;
        cy = (u32)(r >> 32);
      } else {
        const u64 r = (u64)o - d - cy;
        dst[w] = (u32)r;
        cy = (u32)(r >> 63);
      }
      w++;
    }
  };
  for (int k = kmin; k <= kmax; k++) {
    column96(c0, c1, c2, x, y, k, max(0, k - ty), min(tx, k));
    if (k >= LF) emit(c0);
    c0 = c1;
    c1 = c2;
    c2 = 0;
  }
  for (int k = max(kmax + 1, kmin); k <= kmax + 2; k++) {
    if (k >= LF) emit(c0);
    c0 = c1;
    c1 = 0;
  }
  while (cy && w < WL) emit(0);
}


// fx_rmw for operands of at most LFT + 1 words (top <= LFT: fixed-point magnitudes <= 2^(F+32), as the
// Cholesky columns |l_ik| <= 1 are): both operands are loaded into registers once and every column sum runs
// from registers (fx_rmw reads two shared-memory words per multiply-add).  The same columns LF - 2 ..
// (zero beyond the tops), the same carries and kept words, so the same result.
template <int LFT>
__device__ __forceinline__ void fx_rmw_reg(u32* dst, const u32* x, const u32* y, bool add, int WL) {
  constexpr int NW = LFT + 1;
  u32 xr[NW], yr[NW];
#pragma unroll
  for (int i = 0; i < NW; i++) {
    xr[i] = x[i];
    yr[i] = y[i];
  }
  u32 c0 = 0, c1 = 0, c2 = 0, cy = 0;
  int w = 0;
  auto emit = [&](u32 d) {
    if (w < WL) {
      const u32 o = dst[w];
      if (add) {
        const u64 r = (u64)o + d + cy;
        dst[w] = (u32)r;
        cy = (u32)(r >> 32);
      } else {
        const u64 r = (u64)o - d - cy;
        dst[w] = (u32)r;
        cy = (u32)(r >> 63);
      }
      w++;
    }
  };
#pragma unroll
  for (int k = LFT - 2; k <= 2 * LFT; k++) {
    constexpr int dummy = 0;
    (void)dummy;
    u32 d0 = 0, d1 = 0, d2 = 0;                         // a second carry chain (odd terms)
    const int i0 = k - LFT > 0 ? k - LFT : 0, i1 = k < LFT ? k : LFT;
#pragma unroll
    for (int i = i0; i <= i1; i += 2) {
      mac96(c0, c1, c2, xr[i], yr[k - i]);
      if (i + 1 <= i1) mac96(d0, d1, d2, xr[i + 1], yr[k - i - 1]);
    }
    add96(c0, c1, c2, d0, d1, d2);
    if (k >= LFT) emit(c0);
    c0 = c1;
    c1 = c2;
    c2 = 0;
  }
  emit(c0);                                              // columns 2 LFT + 1, 2 LFT + 2: no new terms
  emit(c1);
  while (cy && w < WL) emit(0);
}

// fx_rmw with only the first operand bounded (top <= LFT, kept in registers) and the second read from shared
// memory (one load per multiply-add instead of two): the triangular inverse's products |l_ij| |x_jk|.
template <int LFT>
__device__ __forceinline__ void fx_rmw_lreg(u32* dst, const u32* x, const u32* y, int ty, bool add, int WL) {
  constexpr int NW = LFT + 1;
  u32 xr[NW];
#pragma unroll
  for (int i = 0; i < NW; i++) xr[i] = x[i];
  u32 c0 = 0, c1 = 0, c2 = 0, cy = 0;
  int w = 0;
  auto emit = [&](u32 d) {
    if (w < WL) {
      const u32 o = dst[w];
      if (add) {
        const u64 r = (u64)o + d + cy;
        dst[w] = (u32)r;
        cy = (u32)(r >> 32);
      } else {
        const u64 r = (u64)o - d - cy;
        dst[w] = (u32)r;
        cy = (u32)(r >> 63);
      }
      w++;
    }
  };
  const int kmax = LFT + ty;
  for (int k = LFT - 2; k <= kmax; k++) {
    u32 d0 = 0, d1 = 0, d2 = 0;
#pragma unroll
    for (int i = 0; i < NW; i++) {
      const int jj = k - i;
      if (jj >= 0 && jj <= ty) {
        if (i & 1)
          mac96(d0, d1, d2, xr[i], y[jj]);
        else
          mac96(c0, c1, c2, xr[i], y[jj]);
      }
    }
    add96(c0, c1, c2, d0, d1, d2);
    if (k >= LFT) emit(c0);
    c0 = c1;
    c1 = c2;
    c2 = 0;
  }
  emit(c0);
  emit(c1);
  while (cy && w < WL) emit(0);
}

// Warp-parallel WL-word arithmetic for the Newton steps (words lane and lane + 32 of each operand).
__device__ __forceinline__ void warp_addsub(u32* r, const u32* a, const u32* b, bool sub, int WL) {
  const int lane = threadIdx.x & 31;
  u32 carry = sub ? 1u : 0u;                                  // a - b = a + ~b + 1
  for (int c = 0; c < 2; c++) {
    const int w = lane + 32 * c;
    const u32 av = w < WL ? a[w] : 0u, bv = w < WL ? (sub ? ~b[w] : b[w]) : 0u;
    const u64 v = (u64)av + bv;
    const u32 e = (u32)v;
    u32 cout;
    const u32 cj = chain_carry((v >> 32) != 0, e == kFull, carry, cout);
    __syncwarp();
    if (w < WL) r[w] = e + cj;
    carry = cout;
  }
  __syncwarp();
}

__device__ __forceinline__ void warp_shr1(u32* x, int WL) {              // arithmetic shift right by one bit
  const int lane = threadIdx.x & 31;
  u32 n[2];
  for (int c = 0; c < 2; c++) {
    const int w = lane + 32 * c;
    n[c] = 0;
    if (w < WL - 1) n[c] = (x[w] >> 1) | (x[w + 1] << 31);
    else if (w == WL - 1) n[c] = (u32)(((int32_t)x[w]) >> 1);
  }
  __syncwarp();
  for (int c = 0; c < 2; c++)
    if (lane + 32 * c < WL) x[lane + 32 * c] = n[c];
  __syncwarp();
}

// Entries sit in shared memory at an odd pitch of WP = WL | 1 words: the thread products read one operand
// word per lane from different entries, and an odd pitch puts those words in distinct banks.
__host__ __device__ constexpr int pitch(int WL) { return WL | 1; }
__host__ __device__ constexpr size_t chol_smem_bytes(int WL) {
  return (size_t)(528 + 32) * pitch(WL) * 4 + kWarpsS * sizeof(WarpScratch) + 5 * FW * 4 + 64;
}
__host__ __device__ constexpr size_t trinv_smem_bytes(int WL) {
  return (size_t)(528 + 32) * pitch(WL) * 4 + kWarpsS * sizeof(WarpScratch) + 2 * 528 + 64;
}

__device__ __forceinline__ int tri(int i, int j) { return i * (i + 1) / 2 + j; }

__global__ void __launch_bounds__(kThreadsS) chol_tiles_smem_kernel(u32* __restrict__ A, u32* __restrict__ RINV,
                                                                   int WL, int LF, unsigned* __restrict__ err) {
  extern __shared__ __align__(16) u32 sm[];
  u32* T = sm;                                                   // lower triangle, entry (i, j) at tri(i, j)
  const int WP = pitch(WL);
  u32* colmag = T + 528 * WP;                                    // |l_ik| of the current column
  WarpScratch* ws = reinterpret_cast<WarpScratch*>(colmag + 32 * WP);
  u32* nw = reinterpret_cast<u32*>(ws + kWarpsS);
  u32 *sd = nw, *sr = nw + FW, *st1 = nw + 2 * FW, *st2 = nw + 3 * FW, *sone = nw + 4 * FW;
  uint8_t* colsign = reinterpret_cast<uint8_t*>(nw + 5 * FW);
  uint8_t* coltop = colsign + 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  u32* G = A + (size_t)blockIdx.x * BT * BT * WL;
  u32* RI = RINV + (size_t)blockIdx.x * BT * WL;
  for (int i = 0; i < BT; i++) {
    const u32* src = G + (size_t)i * BT * WL;
    u32* dst = T + (size_t)tri(i, 0) * WP;
    for (int w = tid; w < (i + 1) * WL; w += kThreadsS) dst[(w / WL) * WP + w % WL] = src[w];
  }
  __syncthreads();
  // Pivot k (warp 0): r = d^-1/2 by the Newton schedule, l_kk = d r, r kept in sr and RINV.
  auto pivot = [&](int k) {
    u32* akk = T + (size_t)tri(k, k) * WP;
    for (int w = lane; w < WL; w += 32) sd[w] = akk[w];
    for (int w = lane; w < WL; w += 32) sone[w] = (w == LF) ? 1u : 0u;
    __syncwarp();
    if (lane == 0) {
      if ((sd[WL - 1] >> 31) || (top_word(sd, WL) == 0 && sd[0] == 0)) atomicOr(err, SDPV_ERRBIT_NOTSPD);
      fx_from_double(sr, 1.0 / sqrt(fx_to_double(sd, WL, LF)), WL, LF);
    }
    __syncwarp();
    for (int bits = 100;; bits *= 2) {                             // r <- r + r (1 - d r^2) / 2
      int t = bits / 32 + 2;
      if (t >= WL) t = 0;
      wmul(sr, sr, t, WL, LF, ws[0], st1, nullptr, nullptr, nullptr);
      wmul(st1, sd, t, WL, LF, ws[0], st2, nullptr, nullptr, nullptr);
      warp_addsub(st1, sone, st2, true, WL);
      wmul(sr, st1, t, WL, LF, ws[0], st2, nullptr, nullptr, nullptr);
      warp_shr1(st2, WL);
      warp_addsub(sr, sr, st2, false, WL);
      if (t == 0) break;
    }
    wmul(sd, sr, 0, WL, LF, ws[0], akk, nullptr, nullptr, nullptr);     // l_kk = d * d^-1/2
    for (int w = lane; w < WL; w += 32) RI[(size_t)k * WL + w] = sr[w];
  };
  if (warp == 0) pivot(0);
  __syncthreads();
  // Step k: column k scaled by r_k; then, with one pivot of look-ahead, warp 0 updates a_{k+1,k+1} and runs
  // pivot k+1's Newton chain while warps 1.. apply the rest of step k's trailing update.  Every entry gets
  // the same truncated products as without look-ahead (their exact sum is order-free).
  for (int k = 0; k < BT; k++) {
    for (int i = k + 1 + warp; i < BT; i += kWarpsS) {           // l_ik = a_ik * r_k
      u32* aik = T + (size_t)tri(i, k) * WP;
      wmul(aik, sr, 0, WL, LF, ws[warp], aik, colmag + (size_t)i * WP, colsign + i, coltop + i);
    }
    __syncthreads();
    if (k == BT - 1) break;
    if (warp == 0) {
      u32* dn = T + (size_t)tri(k + 1, k + 1) * WP;                // a_{k+1,k+1} -= l_{k+1,k}^2
      const u32* lk = colmag + (size_t)(k + 1) * WP;
      wmul(lk, lk, 0, WL, LF, ws[0], st1, nullptr, nullptr, nullptr);
      warp_addsub(dn, dn, st1, true, WL);
      pivot(k + 1);
    } else {
      const int m = BT - k - 1, npairs = m * (m + 1) / 2;
      for (int p = 1 + tid - 32; p < npairs; p += kThreadsS - 32) {   // a_ij -= l_ik l_jk, k < j <= i, but (k+1, k+1)
        int ii = (int)((sqrtf(8.f * p + 1.f) - 1.f) * 0.5f);
        while ((ii + 1) * (ii + 2) / 2 <= p) ii++;
        while (ii * (ii + 1) / 2 > p) ii--;
        const int i = k + 1 + ii, j = k + 1 + (p - ii * (ii + 1) / 2);
        u32* dst = T + (size_t)tri(i, j) * WP;
        const u32 *xi = colmag + (size_t)i * WP, *xj = colmag + (size_t)j * WP;
        const bool add = colsign[i] != colsign[j];
        if (LF == 26 && coltop[i] <= 26 && coltop[j] <= 26)
          fx_rmw_reg<26>(dst, xi, xj, add, WL);
        else if (LF == 24 && coltop[i] <= 24 && coltop[j] <= 24)
          fx_rmw_reg<24>(dst, xi, xj, add, WL);
        else
          fx_rmw(dst, xi, coltop[i], xj, coltop[j], add, WL, LF);
      }
    }
    __syncthreads();
  }
  for (int i = 0; i < BT; i++) {
    u32* dst = G + (size_t)i * BT * WL;
    const u32* src = T + (size_t)tri(i, 0) * WP;
    for (int w = tid; w < (i + 1) * WL; w += kThreadsS) dst[w] = src[(w / WL) * WP + w % WL];
  }
}

// X = L^-1 right-looking: slot (i, k) of Xm first accumulates sum_j l_ij x_jk (two's complement, exact
// modulo 2^(32 WL)) as the rows j < i are finished; row j+1 is finished as x_{j+1,k} = -(its sum) r_{j+1}.
// Step j forms all (31 - j)(j + 1) <= 256 products l_ij x_jk (i > j, k <= j) in one round of threads, so
// the critical path is one product round and one warp product per row.  The products and the final
// products are the reference's; only the order of the exact sums differs.
__global__ void __launch_bounds__(kThreadsS) trinv_tiles_smem_kernel(const u32* __restrict__ Lt,
                                                                    const u32* __restrict__ RINV,
                                                                    u32* __restrict__ X, int WL, int LF) {
  extern __shared__ __align__(16) u32 sm[];
  u32* Xm = sm;                                                  // slots tri(i, k), lower triangle
  const int WP = pitch(WL);
  u32* Lcol = Xm + 528 * WP;                                     // |l_ij| of the current column j, by row i
  WarpScratch* ws = reinterpret_cast<WarpScratch*>(Lcol + 32 * WP);
  uint8_t* xs = reinterpret_cast<uint8_t*>(ws + kWarpsS);             // signs, tops of finished x
  uint8_t* xt = xs + 528;
  uint8_t* ls = xt + 528;                                        // signs, tops of the column of L
  uint8_t* lt = ls + 32;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const u32* LG = Lt + (size_t)blockIdx.x * BT * BT * WL;
  const u32* RI = RINV + (size_t)blockIdx.x * BT * WL;
  u32* XG = X + (size_t)blockIdx.x * BT * BT * WL;
  for (int e = tid; e < 528 * WP; e += kThreadsS) Xm[e] = 0;
  __syncthreads();
  for (int i = warp; i < BT; i += kWarpsS) {                     // x_ii = r_i
    int top;
    const int sg = load_mag(RI + (size_t)i * WL, Xm + (size_t)tri(i, i) * WP, WL, top);
    if (lane == 0) {
      xs[tri(i, i)] = (uint8_t)sg;
      xt[tri(i, i)] = (uint8_t)top;
    }
  }
  for (int j = 0; j < BT - 1; j++) {
    for (int i = j + 1 + warp; i < BT; i += kWarpsS) {
      int top;
      const int sg = load_mag(LG + ((size_t)i * BT + j) * WL, Lcol + (size_t)i * WP, WL, top);
      if (lane == 0) {
        ls[i] = (uint8_t)sg;
        lt[i] = (uint8_t)top;
      }
    }
    __syncthreads();
    const int nk = j + 1, np = (BT - 1 - j) * nk;
    for (int p = tid; p < np; p += kThreadsS) {                  // slot (i, k) += l_ij x_jk
      const int i = j + 1 + p / nk, k = p % nk;
      const int e = tri(j, k);
      u32* dst = Xm + (size_t)tri(i, k) * WP;
      const u32 *xl = Lcol + (size_t)i * WP, *yx = Xm + (size_t)e * WP;
      const bool add = ls[i] == xs[e];
      if (LF == 26 && lt[i] <= 26)
        fx_rmw_lreg<26>(dst, xl, yx, xt[e], add, WL);
      else if (LF == 24 && lt[i] <= 24)
        fx_rmw_lreg<24>(dst, xl, yx, xt[e], add, WL);
      else
        fx_rmw(dst, xl, lt[i], yx, xt[e], add, WL, LF);
    }
    __syncthreads();
    for (int k = warp; k <= j; k += kWarpsS) {                   // x_{j+1,k} = -(sum) r_{j+1}
      const int ei = tri(j + 1, k);
      wmul(Xm + (size_t)ei * WP, RI + (size_t)(j + 1) * WL, 0, WL, LF, ws[warp], nullptr, Xm + (size_t)ei * WP,
           xs + ei, xt + ei);
      if (lane == 0) xs[ei] ^= 1;                                // the negation
      __syncwarp();
    }
    __syncthreads();
  }
  for (int e = warp; e < BT * BT; e += kWarpsS) {                      // two's complement out; upper part zero
    const int i = e / BT, k = e % BT;
    u32* dst = XG + (size_t)e * WL;
    if (k > i) {
      for (int w = lane; w < WL; w += 32) dst[w] = 0;
      continue;
    }
    const int ei = tri(i, k);
    u32 v0 = lane < WL ? Xm[(size_t)ei * WP + lane] : 0u, v1 = lane + 32 < WL ? Xm[(size_t)ei * WP + lane + 32] : 0u;
    if (xs[ei]) warp_negate(v0, v1, WL);
    if (lane < WL) dst[lane] = v0;
    if (lane + 32 < WL) dst[lane + 32] = v1;
  }
}


// ---- batched triangular solve L y = v with one factored tile (sdpvibe/basecase.py:228-245): one warp per
// vector, lane i owns v_i; for each j, lane j forms y_j = v_j r_j and broadcasts it, lanes i > j subtract
// l_ij y_j.  V (nvec, 32, WL) is overwritten by y.
__global__ void __launch_bounds__(kThreads) trsv_tiles_kernel(const u32* __restrict__ Lt, const u32* __restrict__ RINV,
                                                              u32* __restrict__ V, i64 nvec, int WL, int LF) {
  __shared__ u32 sp[kThreads / 32][WMAX];
  const i64 w = ((i64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31, ws = threadIdx.x >> 5;
  if (w >= nvec) return;                                         // the whole warp leaves together
  u32* vi = V + ((size_t)w * BT + lane) * WL;
  for (int j = 0; j < BT; j++) {
    if (lane == j) {
      fx_mul(vi, vi, RINV + (size_t)j * WL, 0, WL, LF);
      for (int k = 0; k < WL; k++) sp[ws][k] = vi[k];
    }
    __syncwarp();
    if (lane > j) {
      u32 t[WMAX];
      fx_mul(t, Lt + ((size_t)lane * BT + j) * WL, sp[ws], 0, WL, LF);
      i64 br = 0;
      for (int k = 0; k < WL; k++) {
        const i64 d = (i64)vi[k] - (i64)t[k] + br;
        vi[k] = (u32)d;
        br = d >> 32;
      }
    }
    __syncwarp();
  }
}
}  // namespace

namespace {
// Opt-in shared memory of the tile kernels, set once per process for the largest fast-path tile (WL = FW).
int smem_attributes() {
  static std::once_flag once;
  static cudaError_t e1 = cudaSuccess, e2 = cudaSuccess;
  std::call_once(once, [] {
    e1 = cudaFuncSetAttribute(chol_tiles_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)chol_smem_bytes(FW));
    e2 = cudaFuncSetAttribute(trinv_tiles_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)trinv_smem_bytes(FW));
  });
  if (e1 != cudaSuccess) return sdpv::set_cuda_error(e1);
  if (e2 != cudaSuccess) return sdpv::set_cuda_error(e2);
  return SDPV_OK;
}
}  // namespace

extern "C" int sdpv_chol_tiles(uint32_t* A, uint32_t* RINV, int64_t ntiles, int bt, int WL, int LF, void* stream) {
  if (bt != BT || WL < 2 || WL > WMAX || LF < 2 || LF >= WL || ntiles < 0 || ntiles > 0x7fffffff) return SDPV_EINVAL;
  if (ntiles == 0) return SDPV_OK;
  if (WL <= FW) {
    int st = smem_attributes();
    if (st != SDPV_OK) return st;
    chol_tiles_smem_kernel<<<(unsigned)ntiles, kThreadsS, chol_smem_bytes(WL), sdpv::as_stream(stream)>>>(
        A, RINV, WL, LF, sdpv::device_error_word());
    return sdpv::launch_status();
  }
  chol_tiles_kernel<<<(unsigned)ntiles, kThreads, 0, sdpv::as_stream(stream)>>>(A, RINV, WL, LF,
                                                                               sdpv::device_error_word());
  return sdpv::launch_status();
}

extern "C" int sdpv_trinv_tiles(const uint32_t* Lt, const uint32_t* RINV, uint32_t* X, uint32_t* S, int64_t ntiles,
                                int bt, int WL, int LF, void* stream) {
  if (bt != BT || WL < 2 || WL > WMAX || LF < 2 || LF >= WL || ntiles < 0 || ntiles > 0x7fffffff) return SDPV_EINVAL;
  if (ntiles == 0) return SDPV_OK;
  if (WL <= FW) {                                   // shared-memory kernel: S is not used
    int st = smem_attributes();
    if (st != SDPV_OK) return st;
    trinv_tiles_smem_kernel<<<(unsigned)ntiles, kThreadsS, trinv_smem_bytes(WL), sdpv::as_stream(stream)>>>(
        Lt, RINV, X, WL, LF);
    return sdpv::launch_status();
  }
  trinv_tiles_kernel<<<(unsigned)ntiles, kThreads, 0, sdpv::as_stream(stream)>>>(Lt, RINV, X, S, WL, LF);
  return sdpv::launch_status();
}

// ---------------------------------------------------------------- allocation-free variant of sdpv_trinv_tiles
// Some callers cannot allocate device memory when they need the inverse: their process has already handed
// all device memory to another allocator (a framework's caching pool or a fixed memory budget), or they
// call from code that must not allocate.  For WL <= FW the inverse runs in shared memory and needs no
// scratch at all.  For WL > FW this variant takes the product scratch from a fixed array that is part of
// the library image: SDPV_TRINV_NOALLOC_WORDS 32-bit words (16 MiB), held on every device that loads the
// library's tile module until the process exits.  With lazy module loading (the CUDA 12 default) the module,
// and so the array, is loaded on a device by the first call of any tile entry point there; a caller that
// will hand its device memory away makes one such call first.  A call with WL > FW needs
// ntiles * 32 * 32 * WL words of the array.
#define SDPV_TRINV_NOALLOC_WORDS (4u << 20)
static __device__ __align__(256) uint32_t g_trinv_scratch[SDPV_TRINV_NOALLOC_WORDS];

namespace {
std::mutex g_scratch_mu;
uint32_t* g_scratch_addr[64] = {};

// Device address of g_trinv_scratch on the current device, looked up once per device.  Host code must
// not pass the symbol itself to a kernel: on the host it names a stand-in, not device memory.
int trinv_scratch_address(uint32_t** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return sdpv::set_cuda_error(e);
  if (dev < 0 || dev >= 64) return SDPV_EINVAL;
  std::lock_guard<std::mutex> g(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_trinv_scratch);
    if (e != cudaSuccess) return sdpv::set_cuda_error(e);
    g_scratch_addr[dev] = (uint32_t*)p;
  }
  *out = g_scratch_addr[dev];
  return SDPV_OK;
}
}  // namespace

extern "C" int sdpv_trinv_tiles_noalloc(const uint32_t* Lt, const uint32_t* RINV, uint32_t* X, int64_t ntiles,
                                        int bt, int WL, int LF, void* stream) {
  if (bt != BT || WL < 2 || WL > WMAX || LF < 2 || LF >= WL || ntiles < 0 || ntiles > 0x7fffffff) return SDPV_EINVAL;
  if (ntiles == 0) return SDPV_OK;
  if (WL <= FW) {                                   // shared-memory kernel: no scratch, no size limit
    int st = smem_attributes();
    if (st != SDPV_OK) return st;
    trinv_tiles_smem_kernel<<<(unsigned)ntiles, kThreadsS, trinv_smem_bytes(WL), sdpv::as_stream(stream)>>>(
        Lt, RINV, X, WL, LF);
    return sdpv::launch_status();
  }
  if ((uint64_t)ntiles * BT * BT * (uint64_t)WL > SDPV_TRINV_NOALLOC_WORDS) {
    sdpv::set_message("sdpv_trinv_tiles_noalloc: ntiles * 32 * 32 * WL exceeds the fixed scratch of 4 Mi words");
    return SDPV_EINVAL;
  }
  uint32_t* scratch = nullptr;
  int st = trinv_scratch_address(&scratch);
  if (st != SDPV_OK) return st;
  trinv_tiles_kernel<<<(unsigned)ntiles, kThreads, 0, sdpv::as_stream(stream)>>>(Lt, RINV, X, scratch, WL, LF);
  return sdpv::launch_status();
}

extern "C" int sdpv_trsv_tiles(const uint32_t* Lt, const uint32_t* RINV, uint32_t* V, int64_t nvec, int bt, int WL,
                               int LF, void* stream) {
  if (bt != BT || WL < 2 || WL > WMAX || LF < 2 || LF >= WL || nvec < 0) return SDPV_EINVAL;
  if (nvec == 0) return SDPV_OK;
  const i64 blocks = (nvec * 32 + kThreads - 1) / kThreads;
  if (blocks > 0x7fffffff) return SDPV_EINVAL;
  trsv_tiles_kernel<<<(unsigned)blocks, kThreads, 0, sdpv::as_stream(stream)>>>(Lt, RINV, V, nvec, WL, LF);
  return sdpv::launch_status();
}
