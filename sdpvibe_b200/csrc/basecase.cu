// Cholesky base case on CUDA cores (north-star item (e)): 32 x 32 tiles in wide fixed point.
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

}  // namespace

extern "C" int sdpv_chol_tiles(uint32_t* A, uint32_t* RINV, int64_t ntiles, int bt, int WL, int LF, void* stream) {
  if (bt != BT || WL < 2 || WL > WMAX || LF < 2 || LF >= WL || ntiles < 0 || ntiles > 0x7fffffff) return SDPV_EINVAL;
  if (ntiles == 0) return SDPV_OK;
  chol_tiles_kernel<<<(unsigned)ntiles, kThreads, 0, sdpv::as_stream(stream)>>>(A, RINV, WL, LF,
                                                                               sdpv::device_error_word());
  return sdpv::launch_status();
}

extern "C" int sdpv_trinv_tiles(const uint32_t* Lt, const uint32_t* RINV, uint32_t* X, uint32_t* S, int64_t ntiles,
                                int bt, int WL, int LF, void* stream) {
  if (bt != BT || WL < 2 || WL > WMAX || LF < 2 || LF >= WL || ntiles < 0 || ntiles > 0x7fffffff) return SDPV_EINVAL;
  if (ntiles == 0) return SDPV_OK;
  trinv_tiles_kernel<<<(unsigned)ntiles, kThreads, 0, sdpv::as_stream(stream)>>>(Lt, RINV, X, S, WL, LF);
  return sdpv::launch_status();
}

// ---------------------------------------------------------------- allocation-free variant of sdpv_trinv_tiles
// Some callers cannot allocate device memory when they need the inverse: their process has already handed
// all device memory to another allocator (a framework's caching pool or a fixed memory budget), or they
// call from code that must not allocate.  This variant takes its product scratch from a fixed array that is
// part of the library image: SDPV_TRINV_NOALLOC_WORDS 32-bit words (16 MiB), reserved on every device that
// loads the library until the process exits.  A call needs ntiles * 32 * 32 * WL words of it.
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
