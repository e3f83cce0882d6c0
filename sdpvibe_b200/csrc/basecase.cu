// Cholesky base case on CUDA cores: 32 x 32 tiles in wide fixed point.
//
// A tile entry is WL 32-bit words (two's complement) with F = 32*LF fraction bits; tiles are entry-major
// (tiles, 32, 32, WL), the layout of sdpvibe/basecase.py.  The results are the reference's bit for bit
// (sdpvibe/basecase.py:31-226), because every product is the reference's truncated product and every sum
// of products is exact:
//   * fx product: |a| * |b| summed by product columns from column max(LF-2, la+lb) upward (columns below
//     are never formed), exact carries, words >= LF kept (truncation), sign applied last; t > 0 keeps only
//     the top t words of each operand;
//   * d^-1/2: double seed 1/sqrt(d) converted exactly, then r += r (1 - d r^2) / 2 with products truncated
//     to the top 100, 200, 400, ... bits until full width;
//   * Cholesky by columns (pivot, column scaled by the pivot reciprocal, trailing update of the lower
//     triangle); inverse X = L^-1 with the pivot reciprocals.
// How they are computed is this library's own, organised for latency: one CTA of 16 warps per tile; serial
// products (Newton, pivot-column scaling, the inverse's row finishing) run warp-cooperatively with one
// product column per lane and carries resolved by warp ballots; the bulk products (trailing update, inverse
// row products) run one per thread on 96-bit column accumulators (mad.cc carry chains), the operands of the
// common limb counts held in registers.  WL <= 64: the tile lives in shared memory; 64 < WL <= 96: the same
// kernels keep it in global memory (the factor in place, the inverse's sums in a scratch), three words per
// lane.  The batched substitution L y = v reuses the warp product and a thread product of a signed operand.
#include <cmath>
#include <mutex>

#include "common.cuh"

namespace {

constexpr int BT = 32;
constexpr int kThreads = 256;
constexpr int WMAX = 96;                  // WL <= 96 (L <= 72)
constexpr int FW = 64;                    // WL <= FW: the tile in shared memory
constexpr int kThreadsS = 512;            // tile kernels: 16 warps per tile
constexpr int kWarpsS = kThreadsS / 32;
constexpr unsigned kFull = 0xffffffffu;

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

// Per-warp product scratch for WL <= 32 NPL: the operands' magnitudes and the product.
template <int NPL>
struct WarpScratchT {
  u32 xa[32 * NPL], xb[32 * NPL], acc[32 * NPL];
};

// Words lane + 32 c (c < NPL) of a two's-complement WL-word number negated (mod 2^(32 WL)): ~x plus a carry
// that enters word w when every lower word is zero.
template <int NPL>
__device__ __forceinline__ void warp_negate(u32 (&v)[NPL], int WL) {
  const int lane = threadIdx.x & 31;
  const unsigned lower = (1u << lane) - 1u;
  bool below_zero = true;                                     // every word of the lower lane groups is zero
#pragma unroll
  for (int c = 0; c < NPL; c++) {
    const unsigned nz = __ballot_sync(kFull, lane + 32 * c < WL && v[c] != 0);
    v[c] = ~v[c] + ((below_zero && (nz & lower) == 0) ? 1u : 0u);
    below_zero = below_zero && nz == 0;
  }
}

template <int NPL>
__device__ __forceinline__ int warp_top(const u32 (&v)[NPL], int WL) {
  const int lane = threadIdx.x & 31;
  int top = 0;
#pragma unroll
  for (int c = 0; c < NPL; c++) {
    const unsigned b = __ballot_sync(kFull, lane + 32 * c < WL && v[c] != 0);
    if (b) top = 32 * c + 31 - __clz(b);
  }
  return top;
}

// Magnitude of a two's-complement WL-word operand (shared or global memory) into m[0..WL); returns its sign,
// top = index of its highest nonzero word (0 for zero).  Warp-collective.
template <int NPL>
__device__ __forceinline__ int load_mag(const u32* src, u32* m, int WL, int& top) {
  const int lane = threadIdx.x & 31;
  const int sign = (int)(src[WL - 1] >> 31);
  u32 v[NPL];
#pragma unroll
  for (int c = 0; c < NPL; c++) v[c] = lane + 32 * c < WL ? src[lane + 32 * c] : 0u;
  if (sign) warp_negate<NPL>(v, WL);
#pragma unroll
  for (int c = 0; c < NPL; c++)
    if (lane + 32 * c < WL) m[lane + 32 * c] = v[c];
  top = warp_top<NPL>(v, WL);
  return sign;
}

// Warp-cooperative truncated product of magnitudes: out = trunc(x y) (top t words of each operand when t > 0;
// tops tx, ty): one product column per lane, columns kmin .. min(kmax + 2, LF + WL - 1), each a 96-bit exact
// sum; the column sums are added with their 32- and 64-bit shifts and the carries resolved by chain_carry.
// x, y: shared memory (read at words <= their tops); out: 32 NPL words of shared memory, overwritten.
// SQ: a square (y = x, ty = tx): each column sums the products x_i x_(k-i), i < k - i, doubles the sum and
// adds the middle term x_(k/2)^2 (half the multiply-adds, the same exact column sums).
template <int NPL, bool SQ = false>
__device__ void wmul_core(const u32* x, int tx, const u32* y, int ty, int t, int WL, int LF, u32* out) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int c = 0; c < NPL; c++) out[lane + 32 * c] = 0;
  const int la = t ? max(0, tx - t + 1) : 0, lb = t ? max(0, ty - t + 1) : 0;
  const int kmin = max(LF - 2, la + lb), kmax = tx + ty;
  const int ncol = min(kmax + 2, LF + WL - 1) - kmin + 1;
  __syncwarp();
  u32 p_c1 = 0, p_c2a = 0, p_c2b = 0, p_h = 0, cin = 0;          // carried over from the previous 32 columns
  for (int q0 = 0; q0 < ncol; q0 += 32) {
    const int q = q0 + lane, k = kmin + q;
    // column k = sum of x[i] y[k - i], i0 <= i <= i1: every lane runs the warp's longest column (its own
    // terms past i1 are zeros), four carry chains, so the loop neither diverges nor waits on one chain
    u32 c0 = 0, c1 = 0, c2 = 0;
    {
      const bool act = q < ncol && k <= kmax;
      const int i0 = max(la, k - ty), i1f = act ? min(tx, k - lb) : i0 - 1;
      const int i1 = SQ ? min(i1f, (k - 1) >> 1) : i1f;          // SQ: the pairs i < k - i
      const int nt = (int)__reduce_max_sync(kFull, (unsigned)max(i1 - i0 + 1, 0));
      u32 d0 = 0, d1 = 0, d2 = 0, e0 = 0, e1 = 0, e2 = 0, f0 = 0, f1 = 0, f2 = 0;
      // the next four terms' loads are issued before this four's multiply-adds (software pipelined)
      u32 a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
        const int i = i0 + u;
        a[u] = i <= i1 ? x[i] : 0u;
        b[u] = i <= i1 ? y[k - i] : 0u;
      }
      for (int j = 0; j < nt; j += 4) {
        u32 an[4], bn[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
          const int i = i0 + j + 4 + u;
          an[u] = i <= i1 ? x[i] : 0u;
          bn[u] = i <= i1 ? y[k - i] : 0u;
        }
        mac96(c0, c1, c2, a[0], b[0]);
        mac96(d0, d1, d2, a[1], b[1]);
        mac96(e0, e1, e2, a[2], b[2]);
        mac96(f0, f1, f2, a[3], b[3]);
#pragma unroll
        for (int u = 0; u < 4; u++) {
          a[u] = an[u];
          b[u] = bn[u];
        }
      }
      add96(d0, d1, d2, f0, f1, f2);
      add96(c0, c1, c2, e0, e1, e2);
      add96(c0, c1, c2, d0, d1, d2);
      if (SQ) {
        c2 = (c2 << 1) | (c1 >> 31);
        c1 = (c1 << 1) | (c0 >> 31);
        c0 <<= 1;
        const int mid = k >> 1;
        if (!(k & 1) && i0 <= mid && mid <= i1f) mac96(c0, c1, c2, x[mid], x[mid]);
      }
    }
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
    if (q < ncol && w >= 0 && w < WL) out[w] = e + cj;
    p_c1 = n_c1;
    p_c2a = n_c2a;
    p_c2b = n_c2b;
    p_h = n_h;
    cin = cout;
  }
  __syncwarp();
}

// The truncated product a * b >> F of two's-complement operands (magnitudes multiplied by wmul_core, sign
// applied last).  Outputs (any may be null): out = signed result (may alias a or b), omag = magnitude,
// *osign / *otop (written by lane 0).
template <int NPL>
__device__ void wmul(const u32* a, const u32* b, int t, int WL, int LF, WarpScratchT<NPL>& s, u32* out, u32* omag,
                     uint8_t* osign, uint8_t* otop) {
  const int lane = threadIdx.x & 31;
  int ta, tb;
  const int sa = load_mag<NPL>(a, s.xa, WL, ta);
  const int sb = load_mag<NPL>(b, s.xb, WL, tb);
  __syncwarp();
  wmul_core<NPL>(s.xa, ta, s.xb, tb, t, WL, LF, s.acc);
  u32 m[NPL];
#pragma unroll
  for (int c = 0; c < NPL; c++) m[c] = lane + 32 * c < WL ? s.acc[lane + 32 * c] : 0u;
  const int sg = sa ^ sb;
  if (omag) {
#pragma unroll
    for (int c = 0; c < NPL; c++)
      if (lane + 32 * c < WL) omag[lane + 32 * c] = m[c];
  }
  if (otop) {
    const int tp = warp_top<NPL>(m, WL);
    if (lane == 0) *otop = (uint8_t)tp;
  }
  if (osign && lane == 0) *osign = (uint8_t)sg;
  if (out) {
    if (sg) warp_negate<NPL>(m, WL);
#pragma unroll
    for (int c = 0; c < NPL; c++)
      if (lane + 32 * c < WL) out[lane + 32 * c] = m[c];
  }
  __syncwarp();
}

// ---- register-resident WL-word arithmetic of one warp (word lane + 32 c in v[c], zero at and above WL)
template <int NPL>
__device__ __forceinline__ void reg_load(const u32* src, u32 (&v)[NPL], int WL) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int c = 0; c < NPL; c++) v[c] = lane + 32 * c < WL ? src[lane + 32 * c] : 0u;
}
template <int NPL>
__device__ __forceinline__ void reg_store(u32* dst, const u32 (&v)[NPL], int WL) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int c = 0; c < NPL; c++)
    if (lane + 32 * c < WL) dst[lane + 32 * c] = v[c];
}
// word w of v, in every lane
template <int NPL>
__device__ __forceinline__ u32 reg_word(const u32 (&v)[NPL], int w) {
  u32 r = 0;
#pragma unroll
  for (int c = 0; c < NPL; c++) {
    const u32 x = __shfl_sync(kFull, v[c], w & 31);
    if (c == (w >> 5)) r = x;
  }
  return r;
}
// r = a + b or a - b (mod 2^(32 WL)); r may alias a or b
template <int NPL>
__device__ __forceinline__ void reg_addsub(u32 (&r)[NPL], const u32 (&a)[NPL], const u32 (&b)[NPL], bool sub, int WL) {
  const int lane = threadIdx.x & 31;
  u32 carry = sub ? 1u : 0u;
#pragma unroll
  for (int c = 0; c < NPL; c++) {
    const bool in = lane + 32 * c < WL;
    const u32 av = in ? a[c] : 0u, bv = in ? (sub ? ~b[c] : b[c]) : 0u;
    const u64 v = (u64)av + bv;
    const u32 e = (u32)v;
    u32 cout;
    const u32 cj = chain_carry((v >> 32) != 0, e == kFull, carry, cout);
    r[c] = in ? e + cj : 0u;
    carry = cout;
  }
}
// arithmetic shift right by one bit (floor of half)
template <int NPL>
__device__ __forceinline__ void reg_shr1(u32 (&x)[NPL], int WL) {
  const int lane = threadIdx.x & 31;
  u32 up[NPL], first[NPL];
#pragma unroll
  for (int c = 0; c < NPL; c++) {
    up[c] = __shfl_down_sync(kFull, x[c], 1);                     // word w + 1 within the chunk
    first[c] = __shfl_sync(kFull, x[c], 0);                        // word 32 c
  }
#pragma unroll
  for (int c = 0; c < NPL; c++) {
    const int w = lane + 32 * c;
    const u32 nx = lane < 31 ? up[c] : (c + 1 < NPL ? first[c + 1 < NPL ? c + 1 : c] : 0u);
    if (w < WL - 1) x[c] = (x[c] >> 1) | (nx << 31);
    else if (w == WL - 1) x[c] = (u32)(((int32_t)x[c]) >> 1);
    else x[c] = 0u;
  }
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

// fx_rmw with both operands bounded by compile-time tops (|x| top <= LX, |y| top <= LY) and LF fraction words:
// both in registers, every column sum unrolled over its exact term range (columns LF - 2 .. LX + LY, zero
// beyond the actual tops), so no multiply-add is predicated away.  The same result as fx_rmw.
template <int LF_, int LX, int LY>
__device__ __forceinline__ void fx_rmw_reg2(u32* dst, const u32* x, const u32* y, bool add, int WL) {
  u32 xr[LX + 1], yr[LY + 1];
#pragma unroll
  for (int i = 0; i <= LX; i++) xr[i] = x[i];
#pragma unroll
  for (int i = 0; i <= LY; i++) yr[i] = y[i];
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
  for (int k = LF_ - 2; k <= LX + LY; k++) {
    u32 d0 = 0, d1 = 0, d2 = 0, e0 = 0, e1 = 0, e2 = 0, f0 = 0, f1 = 0, f2 = 0;   // four carry chains
    const int i0 = k - LY > 0 ? k - LY : 0, i1 = k < LX ? k : LX;
#pragma unroll
    for (int i = i0; i <= i1; i++) {
      const int ch = (i - i0) & 3;
      if (ch == 0) mac96(c0, c1, c2, xr[i], yr[k - i]);
      else if (ch == 1) mac96(d0, d1, d2, xr[i], yr[k - i]);
      else if (ch == 2) mac96(e0, e1, e2, xr[i], yr[k - i]);
      else mac96(f0, f1, f2, xr[i], yr[k - i]);
    }
    add96(d0, d1, d2, f0, f1, f2);
    add96(c0, c1, c2, e0, e1, e2);
    add96(c0, c1, c2, d0, d1, d2);
    if (k >= LF_) emit(c0);
    c0 = c1;
    c1 = c2;
    c2 = 0;
  }
  emit(c0);                                              // columns LX + LY + 1, + 2: no new terms
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

// dst (two's complement, WL words) -= trunc(x y) for a signed two's-complement operand x (read in place,
// e.g. from global memory) and a magnitude y (top ty) with sign ysign: x's magnitude is read word by word
// (~x plus the carry that enters at its lowest nonzero word z), then the product columns from LF - 2 as in
// fx_rmw.  One thread.
__device__ void fx_rmw_signed(u32* dst, const u32* x, const u32* y, int ty, int ysign, int WL, int LF) {
  const int xs = (int)(x[WL - 1] >> 31);
  int z = 0;
  while (z < WL - 1 && x[z] == 0) z++;
  auto xw = [&](int k) -> u32 {
    const u32 v = x[k];
    return !xs ? v : (k < z ? 0u : (k == z ? 0u - v : ~v));
  };
  int tx = WL - 1;
  while (tx > 0 && xw(tx) == 0) tx--;
  const bool add = xs != ysign;                                 // dst - sign(x) sign(y) |x||y|
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
    for (int i = max(0, k - ty); i <= min(tx, k); i++) mac96(c0, c1, c2, xw(i), y[k - i]);
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

// Warp-parallel WL-word arithmetic for the Newton steps (words lane and lane + 32 of each operand).
template <int NPL>
__device__ __forceinline__ void warp_addsub(u32* r, const u32* a, const u32* b, bool sub, int WL) {
  const int lane = threadIdx.x & 31;
  u32 carry = sub ? 1u : 0u;                                  // a - b = a + ~b + 1
  for (int c = 0; c < NPL; c++) {
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

template <int NPL>
__device__ __forceinline__ void warp_shr1(u32* x, int WL) {              // arithmetic shift right by one bit
  const int lane = threadIdx.x & 31;
  u32 n[NPL];
  for (int c = 0; c < NPL; c++) {
    const int w = lane + 32 * c;
    n[c] = 0;
    if (w < WL - 1) n[c] = (x[w] >> 1) | (x[w + 1] << 31);
    else if (w == WL - 1) n[c] = (u32)(((int32_t)x[w]) >> 1);
  }
  __syncwarp();
  for (int c = 0; c < NPL; c++)
    if (lane + 32 * c < WL) x[lane + 32 * c] = n[c];
  __syncwarp();
}

// Entries sit in shared memory at an odd pitch of WP = WL | 1 words: the thread products read one operand
// word per lane from different entries, and an odd pitch puts those words in distinct banks.
__host__ __device__ constexpr int pitch(int WL) { return WL | 1; }
template <int NPL, bool GLOBAL>
__host__ __device__ constexpr size_t chol_smem_bytes(int WL) {
  return (size_t)((GLOBAL ? 0 : 528) + 32) * pitch(WL) * 4 + kWarpsS * sizeof(WarpScratchT<NPL>) + 6 * 32 * NPL * 4 + 80;
}
template <int NPL, bool GLOBAL>
__host__ __device__ constexpr size_t trinv_smem_bytes(int WL) {
  return (size_t)((GLOBAL ? 0 : 528) + 96) * pitch(WL) * 4 + kWarpsS * sizeof(WarpScratchT<NPL>) + 2 * 528 + 128 + 64;
}

__device__ __forceinline__ int tri(int i, int j) { return i * (i + 1) / 2 + j; }

// NPL words per lane (WL <= 32 NPL); GLOBAL: the working triangle is the tile itself in global memory (entry
// (i, j) at (32 i + j) WL), else a copy in shared memory (entry (i, j) at tri(i, j), odd pitch WP).
template <int NPL, bool GLOBAL>
__global__ void __launch_bounds__(kThreadsS) chol_tiles_k(u32* __restrict__ A, u32* __restrict__ RINV, int WL, int LF,
                                                          unsigned* __restrict__ err) {
  extern __shared__ __align__(16) u32 sm[];
  const int WP = pitch(WL), NWD = 32 * NPL;
  u32* G = A + (size_t)blockIdx.x * BT * BT * WL;
  u32* T = sm;                                                   // lower triangle, entry (i, j) at tri(i, j)
  auto ent = [&](int i, int j) -> u32* {
    return GLOBAL ? G + ((size_t)i * BT + j) * WL : T + tri(i, j) * WP;
  };
  u32* colmag = GLOBAL ? sm : sm + 528 * WP;                     // |l_ik| of the current column
  WarpScratchT<NPL>* ws = reinterpret_cast<WarpScratchT<NPL>*>(colmag + 32 * WP);
  u32* nw = reinterpret_cast<u32*>(ws + kWarpsS);
  // |r| of pivots of alternate parity in rbuf[k & 1]: warp 0 runs pivot k + 1 while the other warps still scale
  // column k by r_k
  u32 *sd = nw, *st1 = nw + NWD, *st2 = nw + 2 * NWD, *sone = nw + 3 * NWD, *rbuf = nw + 4 * NWD;
  uint8_t* colsign = reinterpret_cast<uint8_t*>(nw + 6 * NWD);
  uint8_t* coltop = colsign + 32;
  int* rinfo = reinterpret_cast<int*>(coltop + 32);               // top and sign of |r| per parity
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  u32* RI = RINV + (size_t)blockIdx.x * BT * WL;
  // Row i of the triangle between the tile (global, entry pitch WL) and shared memory (pitch WP), by one warp:
  // eight entries' loads issued before their stores
  auto copy_row = [&](int i, bool in) {
    u32* g = G + (size_t)i * BT * WL;
    u32* t = ent(i, 0);
    for (int j0 = 0; j0 <= i; j0 += 8) {
      u32 v[8][NPL];
#pragma unroll
      for (int u = 0; u < 8; u++)
#pragma unroll
        for (int c = 0; c < NPL; c++) {
          const int j = j0 + u, w = lane + 32 * c;
          v[u][c] = (j <= i && w < WL) ? (in ? g[(size_t)j * WL + w] : t[j * WP + w]) : 0u;
        }
#pragma unroll
      for (int u = 0; u < 8; u++)
#pragma unroll
        for (int c = 0; c < NPL; c++) {
          const int j = j0 + u, w = lane + 32 * c;
          if (j <= i && w < WL) {
            if (in) t[j * WP + w] = v[u][c];
            else g[(size_t)j * WL + w] = v[u][c];
          }
        }
    }
  };
  // Pivot k (warp 0): r = d^-1/2 by the Newton schedule; |r| in rbuf[k & 1] (top, sign in rinfo), r in RINV.
  // l_kk = d r is formed later by another warp (kkprod), off the chain of pivots.
  auto pivot = [&](int k, const u32* akk) {                      // akk: where d = a_kk is read
    u32* sr = rbuf + (k & 1) * NWD;
    u32 D[NPL];
    reg_load<NPL>(akk, D, WL);
    reg_store<NPL>(sd, D, WL);
    const bool dneg = reg_word<NPL>(D, WL - 1) >> 31;
    bool dnz = false;
#pragma unroll
    for (int c = 0; c < NPL; c++) dnz = dnz || __any_sync(kFull, D[c] != 0u);
    if (lane == 0 && (dneg || !dnz)) atomicOr(err, SDPV_ERRBIT_NOTSPD);
    if (!dneg && dnz) {
      // d > 0: the same truncated products as below, with the operands kept as magnitudes in shared memory
      // (|r| in sr, d in sd, |1 - d r^2| in ws[0].xa) and the additions, sign changes and halvings done in
      // registers; r stays positive in practice, its sign is carried all the same.  The first r is
      // fx_from_double(1 / sqrt(fx_to_double(d))), evaluated by every lane on d's top three words.
      const int td = warp_top<NPL>(D, WL);
      const u32 x0 = reg_word<NPL>(D, td), x1 = reg_word<NPL>(D, max(td - 1, 0)), x2 = reg_word<NPL>(D, max(td - 2, 0));
      double dv = (double)x0;
      if (td >= 1) dv = dv * 4294967296.0 + (double)x1;
      if (td >= 2) dv = dv * 4294967296.0 + (double)x2;
      dv = ldexp(dv, 32 * max(td - 2, 0) - 32 * LF);
      u32 R[NPL], Rt[NPL], P[NPL], S[NPL], O[NPL];
      {
        int e;
        const double mf = frexp(1.0 / sqrt(dv), &e);
        u64 mi = (u64)ldexp(mf, 53);
        int pos = e - 53 + 32 * LF;
        if (pos < 0) {
          mi = (-pos < 64) ? (mi >> (-pos)) : 0ull;
          pos = 0;
        }
        const int li = pos / 32, sh = pos % 32;
        const u64 lo = mi << sh, hi = sh ? (mi >> (64 - sh)) : 0ull;
#pragma unroll
        for (int c = 0; c < NPL; c++) {
          const int q = lane + 32 * c - li;
          const u32 wv = q == 0 ? (u32)lo : q == 1 ? (u32)(lo >> 32) : q == 2 ? (u32)hi : q == 3 ? (u32)(hi >> 32) : 0u;
          Rt[c] = (q >= 0 && lane + 32 * c < WL) ? wv : 0u;
        }
      }
#pragma unroll
      for (int c = 0; c < NPL; c++) {
        O[c] = (lane + 32 * c == LF) ? 1u : 0u;                   // fixed-point 1
        R[c] = Rt[c];
      }
      u32 sR = reg_word<NPL>(Rt, WL - 1) >> 31;
      if (sR) warp_negate<NPL>(R, WL);
      reg_store<NPL>(sr, R, WL);
      __syncwarp();
      int tr = warp_top<NPL>(R, WL);
      for (int bits = 100;; bits *= 2) {                           // r <- r + r (1 - d r^2) / 2
        int t = bits / 32 + 2;
        if (t >= WL) t = 0;
        wmul_core<NPL, true>(sr, tr, sr, tr, t, WL, LF, st1);     // r^2
        reg_load<NPL>(st1, P, WL);
        const int tp = warp_top<NPL>(P, WL);
        wmul_core<NPL>(st1, tp, sd, td, t, WL, LF, st2);          // d r^2
        reg_load<NPL>(st2, P, WL);
        reg_addsub<NPL>(S, O, P, true, WL);                        // 1 - d r^2
        const u32 sS = reg_word<NPL>(S, WL - 1) >> 31;
        if (sS) warp_negate<NPL>(S, WL);
        const int ts = warp_top<NPL>(S, WL);
        reg_store<NPL>(ws[0].xa, S, WL);
        __syncwarp();
        wmul_core<NPL>(sr, tr, ws[0].xa, ts, t, WL, LF, st2);     // |r (1 - d r^2)|
        reg_load<NPL>(st2, P, WL);
        if (sR ^ sS) warp_negate<NPL>(P, WL);
        reg_shr1<NPL>(P, WL);                                      // floor of half
        reg_addsub<NPL>(Rt, Rt, P, false, WL);
        sR = reg_word<NPL>(Rt, WL - 1) >> 31;
#pragma unroll
        for (int c = 0; c < NPL; c++) R[c] = Rt[c];
        if (sR) warp_negate<NPL>(R, WL);
        tr = warp_top<NPL>(R, WL);
        reg_store<NPL>(sr, R, WL);
        __syncwarp();
        if (t == 0) break;
      }
      reg_store<NPL>(RI + (size_t)k * WL, Rt, WL);
      if (lane == 0) {
        rinfo[k & 1] = tr;
        rinfo[2 + (k & 1)] = (int)sR;
      }
      __syncwarp();
    } else {
      for (int w = lane; w < WL; w += 32) sone[w] = (w == LF) ? 1u : 0u;
      __syncwarp();
      if (lane == 0) fx_from_double(sr, 1.0 / sqrt(fx_to_double(sd, WL, LF)), WL, LF);
      __syncwarp();
      for (int bits = 100;; bits *= 2) {                           // r <- r + r (1 - d r^2) / 2
        int t = bits / 32 + 2;
        if (t >= WL) t = 0;
        wmul<NPL>(sr, sr, t, WL, LF, ws[0], st1, nullptr, nullptr, nullptr);
        wmul<NPL>(st1, sd, t, WL, LF, ws[0], st2, nullptr, nullptr, nullptr);
        warp_addsub<NPL>(st1, sone, st2, true, WL);
        wmul<NPL>(sr, st1, t, WL, LF, ws[0], st2, nullptr, nullptr, nullptr);
        warp_shr1<NPL>(st2, WL);
        warp_addsub<NPL>(sr, sr, st2, false, WL);
        if (t == 0) break;
      }
      for (int w = lane; w < WL; w += 32) RI[(size_t)k * WL + w] = sr[w];
      int tr;
      const int sg = load_mag<NPL>(sr, st2, WL, tr);              // |r|, then back into sr
      __syncwarp();
      for (int w = lane; w < WL; w += 32) sr[w] = st2[w];
      if (lane == 0) {
        rinfo[k & 1] = tr;
        rinfo[2 + (k & 1)] = sg;
      }
      __syncwarp();
    }
  };
  // a (shared or global memory, may alias out) times r_k given as |r_k| in rbuf with its top and sign: the
  // truncated product of wmul with the second operand's magnitude already formed
  auto mul_r = [&](u32* a, int k, u32* out, u32* omag, uint8_t* osign, uint8_t* otop) {
    WarpScratchT<NPL>& s = ws[warp];
    int ta;
    const int sa = load_mag<NPL>(a, s.xa, WL, ta);
    __syncwarp();
    wmul_core<NPL>(s.xa, ta, rbuf + (k & 1) * NWD, rinfo[k & 1], 0, WL, LF, s.acc);
    u32 m[NPL];
#pragma unroll
    for (int c = 0; c < NPL; c++) m[c] = lane + 32 * c < WL ? s.acc[lane + 32 * c] : 0u;
    const int sg = sa ^ rinfo[2 + (k & 1)];
    if (omag) {
#pragma unroll
      for (int c = 0; c < NPL; c++)
        if (lane + 32 * c < WL) omag[lane + 32 * c] = m[c];
    }
    if (otop) {
      const int tp = warp_top<NPL>(m, WL);
      if (lane == 0) *otop = (uint8_t)tp;
    }
    if (osign && lane == 0) *osign = (uint8_t)sg;
    if (sg) warp_negate<NPL>(m, WL);
#pragma unroll
    for (int c = 0; c < NPL; c++)
      if (lane + 32 * c < WL) out[lane + 32 * c] = m[c];
    __syncwarp();
  };
  // pivot 0 reads a_00 from the tile itself while warps 1.. copy the triangle into shared memory
  if (warp == 0) pivot(0, GLOBAL ? ent(0, 0) : G);
  else if (!GLOBAL)
    for (int i = warp - 1; i < BT; i += kWarpsS - 1) copy_row(i, true);
  __syncthreads();
  // Step k: column k scaled by r_k; then, with one pivot of look-ahead, warp 0 updates a_{k+1,k+1} and runs
  // pivot k+1's Newton chain while warps 1.. apply the rest of step k's trailing update.  Every entry gets
  // the same truncated products as without look-ahead (their exact sum is order-free).
  for (int k = 0; k < BT; k++) {
    // l_ik = a_ik * r_k: warp 0 takes row k + 1 (its next pivot needs only that row) and goes on without
    // waiting; warps 1.. take the other rows and l_kk = d_k r_k (the last warp) and wait for the whole column
    // (barrier 1: warp 0 arrives)
    if (warp == 0) {
      if (k + 1 < BT) {
        u32* aik = ent(k + 1, k);
        mul_r(aik, k, aik, colmag + (size_t)(k + 1) * WP, colsign + k + 1, coltop + k + 1);
      }
      asm volatile("bar.arrive 1, %0;" ::"r"(kThreadsS) : "memory");
    } else {
      if (warp == kWarpsS - 1) {
        u32* akk = ent(k, k);
        mul_r(akk, k, akk, nullptr, nullptr, nullptr);
      }
      for (int i = k + 1 + warp; i < BT; i += kWarpsS - 1) {
        u32* aik = ent(i, k);
        mul_r(aik, k, aik, colmag + (size_t)i * WP, colsign + i, coltop + i);
      }
      asm volatile("bar.sync 1, %0;" ::"r"(kThreadsS) : "memory");
    }
    if (k == BT - 1) break;
    if (warp == 0) {
      u32* dn = ent(k + 1, k + 1);                // a_{k+1,k+1} -= l_{k+1,k}^2 (a square of magnitudes)
      const u32* lk = colmag + (size_t)(k + 1) * WP;
      wmul_core<NPL, true>(lk, coltop[k + 1], lk, coltop[k + 1], 0, WL, LF, st1);
      warp_addsub<NPL>(dn, dn, st1, true, WL);
      pivot(k + 1, dn);
    } else {
      const int m = BT - k - 1, npairs = m * (m + 1) / 2;
      for (int p = 1 + tid - 32; p < npairs; p += kThreadsS - 32) {   // a_ij -= l_ik l_jk, k < j <= i, but (k+1, k+1)
        int ii = (int)((sqrtf(8.f * p + 1.f) - 1.f) * 0.5f);
        while ((ii + 1) * (ii + 2) / 2 <= p) ii++;
        while (ii * (ii + 1) / 2 > p) ii--;
        const int i = k + 1 + ii, j = k + 1 + (p - ii * (ii + 1) / 2);
        u32* dst = ent(i, j);
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
  // l_kk of the last pivot was written by the last warp after warp 0 had passed its final barrier
  __syncthreads();
  for (int i = warp; i < BT && !GLOBAL; i += kWarpsS) copy_row(BT - 1 - i, false);
}

// X = L^-1 right-looking: slot (i, k) of Xm first accumulates sum_j l_ij x_jk (two's complement, exact
// modulo 2^(32 WL)) as the rows j < i are finished; row j+1 is finished as x_{j+1,k} = -(its sum) r_{j+1}.
// Step j forms all (31 - j)(j + 1) <= 256 products l_ij x_jk (i > j, k <= j) in one round of threads, so
// the critical path is one product round and one warp product per row.  The products and the final
// products are the reference's; only the order of the exact sums differs.
// NPL words per lane; GLOBAL: the slots in the scratch S (528 WP words per tile) instead of shared memory.
template <int NPL, bool GLOBAL>
__global__ void __launch_bounds__(kThreadsS) trinv_tiles_k(const u32* __restrict__ Lt, const u32* __restrict__ RINV,
                                                           u32* __restrict__ X, u32* __restrict__ S, int WL, int LF) {
  extern __shared__ __align__(16) u32 sm[];
  const int WP = pitch(WL);
  u32* Xm = GLOBAL ? S + (size_t)blockIdx.x * 528 * WP : sm;     // slots tri(i, k), lower triangle
  // |l_ij| of column j by row i in Lcol + (j & 1) 32 WP (column j + 1 is read from the tile during step j's
  // products and stored after them); the pivot reciprocals r_i in RIs
  u32* Lcol = GLOBAL ? sm : sm + 528 * WP;
  u32* RIs = Lcol + 64 * WP;
  WarpScratchT<NPL>* ws = reinterpret_cast<WarpScratchT<NPL>*>(RIs + 32 * WP);
  uint8_t* xs = reinterpret_cast<uint8_t*>(ws + kWarpsS);             // signs, tops of finished x
  uint8_t* xt = xs + 528;
  uint8_t* ls = xt + 528;                                        // signs, tops of the columns of L (2 x 32)
  uint8_t* lt = ls + 64;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const u32* LG = Lt + (size_t)blockIdx.x * BT * BT * WL;
  const u32* RI = RINV + (size_t)blockIdx.x * BT * WL;
  u32* XG = X + (size_t)blockIdx.x * BT * BT * WL;
  for (int e = tid; e < 528 * WP; e += kThreadsS) Xm[e] = 0;
  for (int i = warp; i < BT; i += kWarpsS)
    for (int w = lane; w < WL; w += 32) RIs[i * WP + w] = RI[(size_t)i * WL + w];
  __syncthreads();
  for (int i = warp; i < BT; i += kWarpsS) {                     // x_ii = r_i
    int top;
    const int sg = load_mag<NPL>(RIs + i * WP, Xm + (size_t)tri(i, i) * WP, WL, top);
    if (lane == 0) {
      xs[tri(i, i)] = (uint8_t)sg;
      xt[tri(i, i)] = (uint8_t)top;
    }
  }
  for (int i = 1 + warp; i < BT; i += kWarpsS) {                 // column 0
    int top;
    const int sg = load_mag<NPL>(LG + (size_t)i * BT * WL, Lcol + (size_t)i * WP, WL, top);
    if (lane == 0) {
      ls[i] = (uint8_t)sg;
      lt[i] = (uint8_t)top;
    }
  }
  __syncthreads();
  for (int j = 0; j < BT - 1; j++) {
    const u32* Lc = Lcol + (j & 1) * 32 * WP;
    const uint8_t *lsj = ls + (j & 1) * 32, *ltj = lt + (j & 1) * 32;
    u32 pf[2][NPL];                                              // column j + 1, rows j + 2 + warp (+ 16)
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int i = j + 2 + warp + q * kWarpsS;
#pragma unroll
      for (int c = 0; c < NPL; c++)
        pf[q][c] = (i < BT && lane + 32 * c < WL) ? LG[((size_t)i * BT + j + 1) * WL + lane + 32 * c] : 0u;
    }
    const int nk = j + 1, np = (BT - 1 - j) * nk;
    for (int p = tid; p < np; p += kThreadsS) {                  // slot (i, k) += l_ij x_jk
      const int i = j + 1 + p / nk, k = p % nk;
      const int e = tri(j, k);
      u32* dst = Xm + (size_t)tri(i, k) * WP;
      const u32 *xl = Lc + (size_t)i * WP, *yx = Xm + (size_t)e * WP;
      const bool add = lsj[i] == xs[e];
      if (LF == 26 && ltj[i] <= 26 && xt[e] <= 30)
        fx_rmw_reg2<26, 26, 30>(dst, xl, yx, add, WL);
      else if (LF == 24 && ltj[i] <= 24 && xt[e] <= 28)
        fx_rmw_reg2<24, 24, 28>(dst, xl, yx, add, WL);
      else if (LF == 26 && ltj[i] <= 26)
        fx_rmw_lreg<26>(dst, xl, yx, xt[e], add, WL);
      else if (LF == 24 && ltj[i] <= 24)
        fx_rmw_lreg<24>(dst, xl, yx, xt[e], add, WL);
      else
        fx_rmw(dst, xl, ltj[i], yx, xt[e], add, WL, LF);
    }
    __syncthreads();
    for (int k = warp; k <= j; k += kWarpsS) {                   // x_{j+1,k} = -(sum) r_{j+1}
      const int ei = tri(j + 1, k);
      wmul<NPL>(Xm + (size_t)ei * WP, RIs + (j + 1) * WP, 0, WL, LF, ws[warp], nullptr, Xm + (size_t)ei * WP,
           xs + ei, xt + ei);
      if (lane == 0) xs[ei] ^= 1;                                // the negation
      __syncwarp();
    }
    {
      u32* Ln = Lcol + ((j + 1) & 1) * 32 * WP;                  // column j + 1 as magnitudes
#pragma unroll
      for (int q = 0; q < 2; q++) {
        const int i = j + 2 + warp + q * kWarpsS;
        if (i < BT) {
          const int sg = (int)(reg_word<NPL>(pf[q], WL - 1) >> 31);
          if (sg) warp_negate<NPL>(pf[q], WL);
          const int top = warp_top<NPL>(pf[q], WL);
          reg_store<NPL>(Ln + (size_t)i * WP, pf[q], WL);
          if (lane == 0) {
            ls[((j + 1) & 1) * 32 + i] = (uint8_t)sg;
            lt[((j + 1) & 1) * 32 + i] = (uint8_t)top;
          }
        }
      }
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
    u32 v[NPL];
#pragma unroll
    for (int c = 0; c < NPL; c++) v[c] = lane + 32 * c < WL ? Xm[(size_t)ei * WP + lane + 32 * c] : 0u;
    if (xs[ei]) warp_negate<NPL>(v, WL);
#pragma unroll
    for (int c = 0; c < NPL; c++)
      if (lane + 32 * c < WL) dst[lane + 32 * c] = v[c];
  }
}


// ---- batched triangular solve L y = v with one factored tile (sdpvibe/basecase.py:228-245): one warp per
// vector; for each j the warp forms y_j = v_j r_j (warp product, written over v_j, its magnitude kept in
// shared memory), then lane i > j subtracts l_ij y_j from its v_i (thread product of the signed l_ij read in
// place).  V (nvec, 32, WL) is overwritten by y.
template <int NPL>
constexpr size_t trsv_smem_bytes() {
  return (kThreads / 32) * (sizeof(WarpScratchT<NPL>) + 32 * NPL * 4 + 16);
}
template <int NPL>
__global__ void __launch_bounds__(kThreads) trsv_tiles_k(const u32* __restrict__ Lt, const u32* __restrict__ RINV,
                                                         u32* __restrict__ V, i64 nvec, int WL, int LF) {
  extern __shared__ __align__(16) u32 sm[];
  const int lane = threadIdx.x & 31, wi = threadIdx.x >> 5;
  WarpScratchT<NPL>* ws = reinterpret_cast<WarpScratchT<NPL>*>(sm) + wi;
  u32* ymag = reinterpret_cast<u32*>(reinterpret_cast<WarpScratchT<NPL>*>(sm) + kThreads / 32) + wi * 32 * NPL;
  uint8_t* yinfo = reinterpret_cast<uint8_t*>(reinterpret_cast<u32*>(reinterpret_cast<WarpScratchT<NPL>*>(sm) +
                                                                    kThreads / 32) + (kThreads / 32) * 32 * NPL) + wi * 16;
  const i64 w = ((i64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w >= nvec) return;                                         // the whole warp leaves together
  u32* V0 = V + (size_t)w * BT * WL;
  for (int j = 0; j < BT; j++) {
    u32* vj = V0 + (size_t)j * WL;
    wmul<NPL>(vj, RINV + (size_t)j * WL, 0, WL, LF, *ws, vj, ymag, yinfo, yinfo + 1);     // y_j = v_j r_j
    if (lane > j) fx_rmw_signed(V0 + (size_t)lane * WL, Lt + ((size_t)lane * BT + j) * WL, ymag, yinfo[1], yinfo[0],
                                WL, LF);
    __syncwarp();
  }
}
}  // namespace

namespace {
// Opt-in shared memory of the tile kernels (once per process and instantiation).
template <class K>
int smem_attr(K kernel, size_t bytes) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  return e == cudaSuccess ? SDPV_OK : sdpv::set_cuda_error(e);
}
int smem_attributes() {
  static std::once_flag once;
  static int st = SDPV_OK;
  std::call_once(once, [] {
    int r[4] = {smem_attr(chol_tiles_k<2, false>, chol_smem_bytes<2, false>(FW)),
                smem_attr(trinv_tiles_k<2, false>, trinv_smem_bytes<2, false>(FW)),
                smem_attr(chol_tiles_k<3, true>, chol_smem_bytes<3, true>(WMAX)),
                smem_attr(trinv_tiles_k<3, true>, trinv_smem_bytes<3, true>(WMAX))};
    for (int q = 0; q < 4; q++)
      if (r[q] != SDPV_OK) st = r[q];
  });
  return st;
}

// The triangular inverse: shared-memory slots for WL <= FW (S unused), slots in S (ntiles * 528 * (WL | 1)
// words, within ntiles * 32 * 32 * WL) above.
int launch_trinv(const uint32_t* Lt, const uint32_t* RINV, uint32_t* X, uint32_t* S, int64_t ntiles, int WL, int LF,
                 void* stream) {
  int st = smem_attributes();
  if (st != SDPV_OK) return st;
  if (WL <= FW)
    trinv_tiles_k<2, false><<<(unsigned)ntiles, kThreadsS, trinv_smem_bytes<2, false>(WL), sdpv::as_stream(stream)>>>(
        Lt, RINV, X, nullptr, WL, LF);
  else
    trinv_tiles_k<3, true><<<(unsigned)ntiles, kThreadsS, trinv_smem_bytes<3, true>(WL), sdpv::as_stream(stream)>>>(
        Lt, RINV, X, S, WL, LF);
  return sdpv::launch_status();
}
}  // namespace

extern "C" int sdpv_chol_tiles(uint32_t* A, uint32_t* RINV, int64_t ntiles, int bt, int WL, int LF, void* stream) {
  if (bt != BT || WL < 2 || WL > WMAX || LF < 2 || LF >= WL || ntiles < 0 || ntiles > 0x7fffffff) return SDPV_EINVAL;
  if (ntiles == 0) return SDPV_OK;
  int st = smem_attributes();
  if (st != SDPV_OK) return st;
  if (WL <= FW)
    chol_tiles_k<2, false><<<(unsigned)ntiles, kThreadsS, chol_smem_bytes<2, false>(WL), sdpv::as_stream(stream)>>>(
        A, RINV, WL, LF, sdpv::device_error_word());
  else
    chol_tiles_k<3, true><<<(unsigned)ntiles, kThreadsS, chol_smem_bytes<3, true>(WL), sdpv::as_stream(stream)>>>(
        A, RINV, WL, LF, sdpv::device_error_word());
  return sdpv::launch_status();
}

extern "C" int sdpv_trinv_tiles(const uint32_t* Lt, const uint32_t* RINV, uint32_t* X, uint32_t* S, int64_t ntiles,
                                int bt, int WL, int LF, void* stream) {
  if (bt != BT || WL < 2 || WL > WMAX || LF < 2 || LF >= WL || ntiles < 0 || ntiles > 0x7fffffff) return SDPV_EINVAL;
  if (ntiles == 0) return SDPV_OK;
  if (WL > FW && !S) return SDPV_EINVAL;
  return launch_trinv(Lt, RINV, X, S, ntiles, WL, LF, stream);
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
  if (WL <= FW) return launch_trinv(Lt, RINV, X, nullptr, ntiles, WL, LF, stream);   // no scratch, no size limit
  if ((uint64_t)ntiles * BT * BT * (uint64_t)WL > SDPV_TRINV_NOALLOC_WORDS) {
    sdpv::set_message("sdpv_trinv_tiles_noalloc: ntiles * 32 * 32 * WL exceeds the fixed scratch of 4 Mi words");
    return SDPV_EINVAL;
  }
  uint32_t* scratch = nullptr;
  int st = trinv_scratch_address(&scratch);
  if (st != SDPV_OK) return st;
  return launch_trinv(Lt, RINV, X, scratch, ntiles, WL, LF, stream);
}

extern "C" int sdpv_trsv_tiles(const uint32_t* Lt, const uint32_t* RINV, uint32_t* V, int64_t nvec, int bt, int WL,
                               int LF, void* stream) {
  if (bt != BT || WL < 2 || WL > WMAX || LF < 2 || LF >= WL || nvec < 0) return SDPV_EINVAL;
  if (nvec == 0) return SDPV_OK;
  const i64 blocks = (nvec * 32 + kThreads - 1) / kThreads;
  if (blocks > 0x7fffffff) return SDPV_EINVAL;
  if (WL <= FW)
    trsv_tiles_k<2><<<(unsigned)blocks, kThreads, trsv_smem_bytes<2>(), sdpv::as_stream(stream)>>>(Lt, RINV, V, nvec, WL,
                                                                                                     LF);
  else
    trsv_tiles_k<3><<<(unsigned)blocks, kThreads, trsv_smem_bytes<3>(), sdpv::as_stream(stream)>>>(Lt, RINV, V, nvec, WL,
                                                                                                     LF);
  return sdpv::launch_status();
}
