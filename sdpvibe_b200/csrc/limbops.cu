// Limb-plane bookkeeping and per-entry MPF arithmetic on CUDA cores.
//
// All of these are HBM-bound streams over limb planes X[k*B + e]: one thread per entry, limb k of
// consecutive entries adjacent in memory, so every load/store of a warp is one coalesced 128-byte
// transaction.  Semantics follow sdpvibe/limbops.py and the CUDA strings of sdpvibe/mpf.py exactly.
#include "common.cuh"
#include "mpcore.cuh"

namespace {
using namespace sdpv;

constexpr int kThreads = 256;

__device__ __forceinline__ u64 word_at(const int32_t* __restrict__ X, int L, i64 B, i64 e, i64 i, u64 ext) {
  if (i < 0) return 0;
  if (i >= L) return ext;
  return (u64)(u32)__ldg(X + i * B + e);
}

// round_half_up(X / 2^s): limbops.py:31-62.  The 64-bit window slides one word per output limb.
__global__ void shift_round_kernel(const int32_t* __restrict__ X, int Lin, i64 B, const i64* __restrict__ S,
                                   int Lout, int32_t* __restrict__ out, int32_t* __restrict__ flag,
                                   unsigned* __restrict__ err) {
  i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= B) return;
  i64 s = S[e];
  i64 q = s >> 5;
  int r = (int)(s - 32 * q);
  u64 ext = (__ldg(X + (i64)(Lin - 1) * B + e) < 0) ? 0xffffffffull : 0ull;
  i64 sb = s - 1, qb = sb >> 5;
  int rb = (int)(sb - 32 * qb);
  u64 carry = (sb >= 0) ? ((word_at(X, Lin, B, e, qb, ext) >> rb) & 1ull) : 0ull;
  u64 lo = word_at(X, Lin, B, e, q, ext);
  u64 prev = 0;
  for (int k = 0; k <= Lout; k++) {
    u64 hi = word_at(X, Lin, B, e, q + k + 1, ext);
    u64 v = (((hi << 32) | lo) >> r & 0xffffffffull) + carry;
    lo = hi;
    carry = v >> 32;
    v &= 0xffffffffull;
    if (k < Lout) {
      out[(i64)k * B + e] = (int32_t)(u32)v;
      prev = v;
    } else {
      u64 want = (prev >> 31) ? 0xffffffffull : 0ull;
      int bad = v != want;
      if (flag) flag[e] = bad;
      else if (bad) atomicOr(err, SDPV_ERRBIT_OVERFLOW);
    }
  }
}

// A + sgn*B mod 2^(32L): limbops.py:65-81.
__global__ void add_same_kernel(const int32_t* __restrict__ A, const int32_t* __restrict__ Bm, int L, i64 B, int sgn,
                                int32_t* __restrict__ out) {
  i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= B) return;
  i64 carry = 0;
  for (int k = 0; k < L; k++) {
    i64 a = (k == L - 1) ? (i64)A[(i64)k * B + e] : (i64)(u32)A[(i64)k * B + e];
    i64 b = (k == L - 1) ? (i64)Bm[(i64)k * B + e] : (i64)(u32)Bm[(i64)k * B + e];
    i64 v = a + sgn * b + carry;
    carry = v >> 32;
    out[(i64)k * B + e] = (int32_t)(u32)v;
  }
}

// Bit length of v or ~v, scanning from the top limb down (one limb for normalised data):
// limbops.py:196-210.
__global__ void bitlen_kernel(const int32_t* __restrict__ X, int L, i64 B, i64* __restrict__ out) {
  i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= B) return;
  u32 ext = (X[(i64)(L - 1) * B + e] < 0) ? 0xffffffffu : 0u;
  i64 bl = 0;
  for (int k = L - 1; k >= 0; k--) {
    u32 x = (u32)X[(i64)k * B + e] ^ ext;
    if (x) {
      bl = 32 * (i64)k + 32 - __clz(x);
      break;
    }
  }
  out[e] = bl;
}

// Two independently rounded right shifts to max(ea,eb)+1, then add: batched.py:55-79.
__global__ void badd_align_kernel(const int32_t* __restrict__ A, const int32_t* __restrict__ Bm,
                                  const i64* __restrict__ EA, const i64* __restrict__ EB, int L, i64 n, i64 rows,
                                  i64 cols, int sign, int32_t* __restrict__ out, i64* __restrict__ EO) {
  i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  i64 col = (e / (rows * cols)) * cols + e % cols;
  i64 ea = EA[col], eb = EB[col];
  i64 ex = (ea > eb ? ea : eb) + 1;
  i64 sa = ex - ea, sb = ex - eb;
  u64 ax = (A[(i64)(L - 1) * n + e] < 0) ? 0xffffffffull : 0ull;
  u64 bx = (Bm[(i64)(L - 1) * n + e] < 0) ? 0xffffffffull : 0ull;
  i64 qa = sa >> 5, qb = sb >> 5;
  int ra = (int)(sa & 31), rb = (int)(sb & 31);
  i64 qa1 = (sa - 1) >> 5, qb1 = (sb - 1) >> 5;
  u64 ca = (word_at(A, L, n, e, qa1, ax) >> ((sa - 1) & 31)) & 1ull;
  u64 cb = (word_at(Bm, L, n, e, qb1, bx) >> ((sb - 1) & 31)) & 1ull;
  u64 alo = word_at(A, L, n, e, qa, ax), blo = word_at(Bm, L, n, e, qb, bx);
  i64 carry = 0;
  for (int k = 0; k < L; k++) {
    u64 ahi = word_at(A, L, n, e, qa + k + 1, ax), bhi = word_at(Bm, L, n, e, qb + k + 1, bx);
    u64 a = ((((ahi << 32) | alo) >> ra) & 0xffffffffull) + ca;
    u64 b = ((((bhi << 32) | blo) >> rb) & 0xffffffffull) + cb;
    alo = ahi;
    blo = bhi;
    ca = a >> 32;
    cb = b >> 32;
    i64 t = (i64)(a & 0xffffffffull) + sign * (i64)(b & 0xffffffffull) + carry;
    carry = t >> 32;
    out[(i64)k * n + e] = (int32_t)(u32)t;
  }
  if ((e / cols) % rows == 0) EO[col] = ex;
}

// ------------------------------------------------------------------ MPF (one exponent per entry)
template <int LMAX>
__global__ void mpf_mul_kernel(int L, i64 n, const int32_t* __restrict__ A, const i64* __restrict__ eA,
                               const int32_t* __restrict__ Bm, const i64* __restrict__ eB, int bscalar,
                               int32_t* __restrict__ O, i64* __restrict__ eO) {
  i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  i64 ib = bscalar ? 0 : i, nbn = bscalar ? 1 : n;
  u32 a[LMAX], b[LMAX], r[LMAX];
  for (int k = 0; k < L; k++) {
    a[k] = (u32)A[(i64)k * n + i];
    b[k] = (u32)Bm[(i64)k * nbn + ib];
  }
  i64 er;
  mpf_mul_dev<LMAX>(a, eA[i], b, eB[ib], L, r, er);
  for (int k = 0; k < L; k++) O[(i64)k * n + i] = (int32_t)r[k];
  eO[i] = er;
}

template <int LMAX>
__global__ void mpf_add_kernel(int L, i64 n, const int32_t* A, const i64* eA,
                               const int32_t* __restrict__ Bm, const i64* __restrict__ eB, int sgn,
                               int32_t* O, i64* eO, const int32_t* __restrict__ pred) {
  i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (pred && *pred == 0) return;                      // predicated launch: O / eO untouched
  u32 a[LMAX], b[LMAX], r[LMAX];
  for (int k = 0; k < L; k++) {
    a[k] = (u32)A[(i64)k * n + i];
    b[k] = (u32)Bm[(i64)k * n + i];
  }
  i64 er;
  mpf_add_dev<LMAX>(a, eA[i], b, eB[i], sgn, L, r, er);
  for (int k = 0; k < L; k++) O[(i64)k * n + i] = (int32_t)r[k];
  eO[i] = er;
}

template <int LMAX>
__global__ void mpf_norm_kernel(int L, int LI, i64 n, const int32_t* __restrict__ X, const i64* __restrict__ eI,
                                int32_t* __restrict__ O, i64* __restrict__ eO) {
  i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  u32 w[160], r[LMAX];
  for (int k = 0; k < LI; k++) w[k] = (u32)X[(i64)k * n + i];
  bool ng = w[LI - 1] >> 31;
  if (ng) neg_words(w, LI);
  int bl = bitlen_mag(w, LI);
  if (!bl) {
    for (int k = 0; k < L; k++) O[(i64)k * n + i] = 0;
    eO[i] = SDPV_EZ;
    return;
  }
  int s = bl - (32 * L - 2);
  mag_shift(w, LI, s, r, L);
  if (ng) neg_words(r, L);
  for (int k = 0; k < L; k++) O[(i64)k * n + i] = (int32_t)r[k];
  eO[i] = eI[i] + s;
}

// float64 -> normalised MPF, exactly: the 53-bit significand (subnormals included) shifted to NB = 32L-2 bits
// (NB >= 62 for L >= 2, so no rounding).  The normalised form is unique, so this equals normalising the
// two-limb integer of frexp (sdpvibe/solver.py:1012-1018).  Zeros (either sign) -> m = 0, e = EZ; a
// non-finite input -> zero and the overflow bit in the device error word.
__global__ void from_f64_kernel(int L, i64 n, const double* __restrict__ V, int32_t* __restrict__ O,
                                i64* __restrict__ eO, unsigned* __restrict__ err) {
  i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const u64 bits = (u64)__double_as_longlong(__ldg(V + i));
  const bool ng = bits >> 63;
  const int bexp = (int)((bits >> 52) & 0x7ff);
  u64 mant = bits & ((1ull << 52) - 1);
  i64 ex = -1074;
  if (bexp == 0x7ff) {
    atomicOr(err, SDPV_ERRBIT_OVERFLOW);
    mant = 0;
  } else if (bexp) {
    mant |= 1ull << 52;
    ex = bexp - 1075;
  }
  if (!mant) {
    for (int k = 0; k < L; k++) O[(i64)k * n + i] = 0;
    eO[i] = SDPV_EZ;
    return;
  }
  const int bl = 64 - __clzll((long long)mant);
  const int sh = 32 * L - 2 - bl;                     // >= 9
  const int q = sh >> 5;
  const unsigned __int128 t = (unsigned __int128)mant << (sh & 31);
  u32 carry = 1;
  for (int k = 0; k < L; k++) {
    const int j = k - q;
    u32 w = (j >= 0 && j < 3) ? (u32)(t >> (32 * j)) : 0u;
    if (ng) {
      w = ~w + carry;
      carry = carry && w == 0;
    }
    O[(i64)k * n + i] = (int32_t)w;
  }
  eO[i] = ex - sh;
}

inline unsigned blocks(i64 n) { return (unsigned)((n + kThreads - 1) / kThreads); }

#define SDPV_LMAX_DISPATCH(L, KERNEL, ...)                                     \
  do {                                                                         \
    if ((L) <= 8) KERNEL<8><<<blocks(n), kThreads, 0, st>>>(__VA_ARGS__);      \
    else if ((L) <= 16) KERNEL<16><<<blocks(n), kThreads, 0, st>>>(__VA_ARGS__); \
    else if ((L) <= 32) KERNEL<32><<<blocks(n), kThreads, 0, st>>>(__VA_ARGS__); \
    else if ((L) <= 64) KERNEL<64><<<blocks(n), kThreads, 0, st>>>(__VA_ARGS__); \
    else KERNEL<160><<<blocks(n), kThreads, 0, st>>>(__VA_ARGS__);             \
  } while (0)

}  // namespace

extern "C" int sdpv_shift_round(const int32_t* X, int Lin, int64_t B, const int64_t* s, int Lout, int32_t* out,
                                int32_t* flag, void* stream) {
  if (Lin < 1 || Lout < 1 || B < 0) return SDPV_EINVAL;
  if (B == 0) return SDPV_OK;
  unsigned* err = sdpv::device_error_word();
  shift_round_kernel<<<blocks(B), kThreads, 0, sdpv::as_stream(stream)>>>(X, Lin, B, s, Lout, out, flag, err);
  return sdpv::launch_status();
}

extern "C" int sdpv_add_same(const int32_t* A, const int32_t* Bm, int L, int64_t B, int sgn, int32_t* out,
                             void* stream) {
  if (L < 1 || B < 0 || (sgn != 1 && sgn != -1)) return SDPV_EINVAL;
  if (B == 0) return SDPV_OK;
  add_same_kernel<<<blocks(B), kThreads, 0, sdpv::as_stream(stream)>>>(A, Bm, L, B, sgn, out);
  return sdpv::launch_status();
}

extern "C" int sdpv_bitlen(const int32_t* X, int L, int64_t B, int64_t* out, void* stream) {
  if (L < 1 || B < 0) return SDPV_EINVAL;
  if (B == 0) return SDPV_OK;
  bitlen_kernel<<<blocks(B), kThreads, 0, sdpv::as_stream(stream)>>>(X, L, B, out);
  return sdpv::launch_status();
}

extern "C" int sdpv_badd_align(const int32_t* A, const int32_t* Bm, const int64_t* EA, const int64_t* EB, int L,
                               int64_t nb, int64_t rows, int64_t cols, int sign, int32_t* out, int64_t* EO,
                               void* stream) {
  if (L < 1 || nb < 0 || rows < 0 || cols < 0 || (sign != 1 && sign != -1)) return SDPV_EINVAL;
  i64 n = nb * rows * cols;
  if (n == 0) return SDPV_OK;
  badd_align_kernel<<<blocks(n), kThreads, 0, sdpv::as_stream(stream)>>>(A, Bm, EA, EB, L, n, rows, cols, sign, out,
                                                                         EO);
  return sdpv::launch_status();
}

extern "C" int sdpv_mpf_mul(int L, int64_t n, const int32_t* A, const int64_t* eA, const int32_t* Bm,
                            const int64_t* eB, int bscalar, int32_t* O, int64_t* eO, void* stream) {
  if (L < 1 || L > 160 || n < 0) return SDPV_EINVAL;
  if (n == 0) return SDPV_OK;
  cudaStream_t st = sdpv::as_stream(stream);
  SDPV_LMAX_DISPATCH(L, mpf_mul_kernel, L, n, A, eA, Bm, eB, bscalar, O, eO);
  return sdpv::launch_status();
}

extern "C" int sdpv_mpf_add(int L, int64_t n, const int32_t* A, const int64_t* eA, const int32_t* Bm,
                            const int64_t* eB, int sgn, int32_t* O, int64_t* eO, void* stream) {
  if (L < 1 || L > 160 || n < 0) return SDPV_EINVAL;
  if (n == 0) return SDPV_OK;
  cudaStream_t st = sdpv::as_stream(stream);
  SDPV_LMAX_DISPATCH(L, mpf_add_kernel, L, n, A, eA, Bm, eB, sgn, O, eO, (const int32_t*)nullptr);
  return sdpv::launch_status();
}

extern "C" int sdpv_mpf_add_if(int L, int64_t n, const int32_t* A, const int64_t* eA, const int32_t* Bm,
                               const int64_t* eB, int sgn, int32_t* O, int64_t* eO, const int32_t* pred,
                               void* stream) {
  if (L < 1 || L > 160 || n < 0 || !pred) return SDPV_EINVAL;
  if (n == 0) return SDPV_OK;
  cudaStream_t st = sdpv::as_stream(stream);
  SDPV_LMAX_DISPATCH(L, mpf_add_kernel, L, n, A, eA, Bm, eB, sgn, O, eO, pred);
  return sdpv::launch_status();
}

extern "C" int sdpv_mpf_from_f64(int L, int64_t n, const double* V, int32_t* O, int64_t* eO, void* stream) {
  if (L < 2 || L > 160 || n < 0) return SDPV_EINVAL;
  if (n == 0) return SDPV_OK;
  from_f64_kernel<<<blocks(n), kThreads, 0, sdpv::as_stream(stream)>>>(L, n, V, O, eO, sdpv::device_error_word());
  return sdpv::launch_status();
}

extern "C" int sdpv_mpf_norm(int L, int LI, int64_t n, const int32_t* X, const int64_t* eI, int32_t* O,
                             int64_t* eO, void* stream) {
  if (L < 1 || L > 160 || LI < 1 || LI > 160 || n < 0) return SDPV_EINVAL;
  if (n == 0) return SDPV_OK;
  cudaStream_t st = sdpv::as_stream(stream);
  SDPV_LMAX_DISPATCH(L, mpf_norm_kernel, L, LI, n, X, eI, O, eO);
  return sdpv::launch_status();
}
