// Alignment of MPF operands to per-row / per-column reference exponents (the set-up of every exact GEMM).
//
// top(e) = e + bitlen(m) (EZ for zero entries, sdpvibe/mpf.py:348-351); the reference takes the max of
// top over each row of op(A) / column of op(B) (mpf.py:390-398) or over each column of a Gram chunk
// (mpf.py:563), and re-rounds every entry to that reference exponent with limbops.shift_round
// (ties toward +infinity), after a transposing copy.  Here:
//   sdpv_top_max: the reduction in one launch (rows: one warp per row; columns: column strips with a
//                 64-bit atomic max), reading only the top limbs of normalised data;
//   sdpv_align:   the rounding shift fused with the transpose: a 16 x 32 tile of entries is staged in
//                 shared memory with all its limbs (coalesced along columns), then each thread rounds
//                 its entries and writes the output limb planes coalesced along the new fast axis.
#include "common.cuh"

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ i64 entry_top(const int32_t* __restrict__ m, i64 plane, i64 idx, int L, i64 e) {
  if (e == SDPV_EZ) return SDPV_EZ;
  u32 ext = (m[(i64)(L - 1) * plane + idx] < 0) ? 0xffffffffu : 0u;
  for (int k = L - 1; k >= 0; k--) {
    u32 x = (u32)m[(i64)k * plane + idx] ^ ext;
    if (x) return e + 32 * (i64)k + 32 - __clz(x);
  }
  return e;
}

// Max over the contiguous axis: one warp per (b, r).
__global__ void top_max_rows_kernel(const int32_t* __restrict__ m, const i64* __restrict__ e, int L, i64 nrows, i64 C,
                                    i64* __restrict__ out) {
  i64 row = ((i64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (row >= nrows) return;
  const i64 plane = nrows * C;
  i64 best = SDPV_EZ;
  for (i64 c = lane; c < C; c += 32) {
    i64 idx = row * C + c;
    i64 t = entry_top(m, plane, idx, L, e[idx]);
    best = t > best ? t : best;
  }
  for (int o = 16; o > 0; o >>= 1) {
    i64 v = __shfl_xor_sync(0xffffffffu, best, o);
    best = v > best ? v : best;
  }
  if (lane == 0) out[row] = best;
}

__global__ void fill_kernel(i64* __restrict__ out, i64 n, i64 v) {
  i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = v;
}

// Max over the strided axis: blocks of 32 columns x 8 row groups; each thread takes 16 rows with all
// loads issued before any is used, then a shared-memory reduction and one 64-bit atomic max per column.
constexpr int kColRows = 16;
__global__ void __launch_bounds__(kThreads) top_max_cols_kernel(const int32_t* __restrict__ m,
                                                                const i64* __restrict__ e, int L, i64 nb, i64 R,
                                                                i64 C, i64* __restrict__ out) {
  __shared__ i64 red[8][32];
  const int cx = threadIdx.x & 31, ry = threadIdx.x >> 5;
  const i64 c = (i64)blockIdx.x * 32 + cx;
  const i64 b = blockIdx.z;
  const i64 r0 = ((i64)blockIdx.y * 8 + ry) * kColRows;
  const i64 plane = nb * R * C;
  i64 best = SDPV_EZ;
  if (c < C) {
    i64 ev[kColRows];
    int32_t tw[kColRows];
#pragma unroll
    for (int t = 0; t < kColRows; t++) {
      i64 r = r0 + t;
      i64 idx = (b * R + r) * C + c;
      ev[t] = (r < R) ? e[idx] : SDPV_EZ;
      tw[t] = (r < R) ? m[(i64)(L - 1) * plane + idx] : 0;
    }
#pragma unroll
    for (int t = 0; t < kColRows; t++) {
      if (ev[t] == SDPV_EZ) continue;
      i64 top;
      u32 x = (u32)tw[t] ^ (tw[t] < 0 ? 0xffffffffu : 0u);
      if (x) top = ev[t] + 32 * (i64)(L - 1) + 32 - __clz(x);           // normalised data: top limb decides
      else top = entry_top(m, plane, (b * R + r0 + t) * C + c, L, ev[t]);
      best = top > best ? top : best;
    }
  }
  red[ry][cx] = best;
  __syncthreads();
  if (ry == 0 && c < C) {
#pragma unroll
    for (int y = 1; y < 8; y++) best = red[y][cx] > best ? red[y][cx] : best;
    if (best > SDPV_EZ) atomicMax((long long*)&out[b * C + c], (long long)best);
  }
}

// Round-half-up shift of one entry whose limbs are read through `word(i)` (i in [0, L)).
template <class Word>
__device__ __forceinline__ void shift_entry(Word word, int L, i64 s, int Lout, int32_t* __restrict__ out, i64 ostride,
                                            unsigned* err) {
  i64 q = s >> 5;
  int r = (int)(s - 32 * q);
  u64 ext = ((int32_t)word(L - 1) < 0) ? 0xffffffffull : 0ull;
  auto w = [&](i64 i) -> u64 { return i < 0 ? 0ull : (i >= L ? ext : (u64)word((int)i)); };
  i64 sb = s - 1, qb = sb >> 5;
  int rb = (int)(sb - 32 * qb);
  u64 carry = (sb >= 0) ? ((w(qb) >> rb) & 1ull) : 0ull;
  u64 lo = w(q), prev = 0;
  for (int k = 0; k <= Lout; k++) {
    u64 hi = w(q + k + 1);
    u64 v = ((((hi << 32) | lo) >> r) & 0xffffffffull) + carry;
    lo = hi;
    carry = v >> 32;
    v &= 0xffffffffull;
    if (k < Lout) {
      out[(i64)k * ostride] = (int32_t)(u32)v;
      prev = v;
    } else if (v != ((prev >> 31) ? 0xffffffffull : 0ull)) {
      atomicOr(err, SDPV_ERRBIT_OVERFLOW);
    }
  }
}

// The same for s >= 0 (the alignment case: target >= exponent) in 32-bit arithmetic: one funnel shift and
// one add with carry per output word.  s beyond 32 (L + 1) gives the same words as 32 (L + 1) (every word
// read is the sign extension), so it is clamped.  s < 0 takes the general path.
template <class Word>
__device__ __forceinline__ void shift_entry32(Word word, int L, i64 s, int Lout, int32_t* __restrict__ out,
                                              i64 ostride, unsigned* err) {
  if (s < 0) {
    shift_entry(word, L, s, Lout, out, ostride, err);
    return;
  }
  const u32 ext = ((int32_t)word(L - 1) < 0) ? 0xffffffffu : 0u;
  const int si = (int)(s > 32 * (i64)(L + 1) ? 32 * (i64)(L + 1) : s);
  const int q = si >> 5, r = si & 31;
  auto w = [&](int i) -> u32 { return i < L ? (u32)word(i) : ext; };
  u32 carry = si > 0 ? (w((si - 1) >> 5) >> ((si - 1) & 31)) & 1u : 0u;
  u32 lo = w(q), prev = 0;
  for (int k = 0; k <= Lout; k++) {
    const u32 hi = w(q + k + 1);
    const u32 f = __funnelshift_r(lo, hi, r);
    const u32 v = f + carry;
    carry = v < f ? 1u : 0u;
    lo = hi;
    if (k < Lout) {
      out[(i64)k * ostride] = (int32_t)v;
      prev = v;
    } else if (v != ((prev >> 31) ? 0xffffffffu : 0u)) {
      atomicOr(err, SDPV_ERRBIT_OVERFLOW);
    }
  }
}

// No transpose: thread per entry (b, r, c); reference exponent per row (per_col = 0) or column.
__global__ void align_kernel(const int32_t* __restrict__ m, const i64* __restrict__ e, int L, i64 nb, i64 R, i64 C,
                             const i64* __restrict__ target, int per_col, int Lout, int32_t* __restrict__ out,
                             unsigned* err) {
  i64 idx = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  const i64 n = nb * R * C;
  if (idx >= n) return;
  i64 b = idx / (R * C), rc = idx - b * R * C, r = rc / C, c = rc - r * C;
  i64 ev = e[idx];
  i64 s = (ev == SDPV_EZ) ? (1ll << 30) : target[per_col ? b * C + c : b * R + r] - ev;
  shift_entry32([&](int i) { return (u32)__ldg(m + (i64)i * n + idx); }, L, s, Lout, out + idx, n, err);
}

// Transpose: tiles of ATR = 8 rows x 32 columns staged with all limbs (about 30 KB at 26 limbs, so seven CTAs
// share an SM and hide each other's loads); out is (Lout, nb, C, R), written in 32-byte runs (8 rows) per
// column and limb.  The tiles of one row band run next to each other (column tile fastest in the 1-D grid),
// so the 32-byte sectors that two column tiles share are read from DRAM once; staged rows are ATP = 36 words
// apart, which puts the 8 rows x 4 columns that a warp's lanes read at once in distinct banks.
constexpr int TR = 16, TC = 32;
constexpr int ATR = 8, ATP = 36;
__global__ void __launch_bounds__(kThreads) align_t_kernel(const int32_t* __restrict__ m, const i64* __restrict__ e,
                                                           int L, i64 nb, i64 R, i64 C, const i64* __restrict__ target,
                                                           int per_col, int Lout, i64 Rld, int32_t* __restrict__ out,
                                                           unsigned* err) {
  extern __shared__ u32 sm[];                       // [L][ATR][ATP] limbs, then [ATR][TC + 1] exponents
  i64* se = reinterpret_cast<i64*>(sm + (size_t)L * ATR * ATP);
  const i64 n = nb * R * C, no = nb * C * Rld;      // input / output plane sizes
  const i64 b = blockIdx.z;
  const i64 nct = (C + TC - 1) / TC;
  const i64 r0 = (i64)(blockIdx.x / nct) * ATR, c0 = (i64)(blockIdx.x % nct) * TC;
  const int tid = threadIdx.x;
  for (int pos = tid; pos < ATR * TC; pos += kThreads) {     // all copies in flight at once
    const int rr = pos / TC, cc = pos % TC;
    const i64 r = r0 + rr, c = c0 + cc;
    const bool in = r < R && c < C;
    const int32_t* src = m + (in ? (b * R + r) * C + c : 0);
    u32* dst = &sm[rr * ATP + cc];
    const u32 nb4 = in ? 4u : 0u;
    for (int l = 0; l < L; l++, src += n, dst += ATR * ATP) cp_async4(dst, src, nb4);
  }
  cp_async_commit();
  for (int t = tid; t < ATR * TC; t += kThreads) {
    int rr = t / TC, cc = t % TC;
    i64 r = r0 + rr, c = c0 + cc;
    se[rr * (TC + 1) + cc] = (r < R && c < C) ? e[(b * R + r) * C + c] : SDPV_EZ;
  }
  cp_async_wait<0>();
  __syncthreads();
  // thread -> (cc, rr) with rr fastest, so output stores (fast axis = r) are coalesced
  for (int t = tid; t < ATR * TC; t += kThreads) {
    int rr = t % ATR, cc = t / ATR;
    i64 r = r0 + rr, c = c0 + cc;
    if (r >= R || c >= C) continue;
    i64 ev = se[rr * (TC + 1) + cc];
    i64 s = (ev == SDPV_EZ) ? (1ll << 30) : target[per_col ? b * C + c : b * R + r] - ev;
    const u32* base = sm + rr * ATP + cc;
    shift_entry32([&](int i) { return base[i * ATR * ATP]; }, L, s, Lout, out + (b * C + c) * Rld + r, no, err);
  }
}

// shift_entry / shift_entry32 with the Lout output words in registers (o[k], k < Lout < RW; loops unrolled to
// RW so that every index is static); returns the sign bit of the result.
template <int RW, class Word>
__device__ __forceinline__ u32 shift_entry_regs(Word word, int L, i64 s, int Lout, u32 (&o)[RW], unsigned* err) {
  u32 prev = 0;
  if (s >= 0) {
    const u32 ext = ((int32_t)word(L - 1) < 0) ? 0xffffffffu : 0u;
    const int si = (int)(s > 32 * (i64)(L + 1) ? 32 * (i64)(L + 1) : s);
    const int q = si >> 5, r = si & 31;
    auto w = [&](int i) -> u32 { return i < L ? (u32)word(i) : ext; };
    u32 carry = si > 0 ? (w((si - 1) >> 5) >> ((si - 1) & 31)) & 1u : 0u;
    u32 lo = w(q);
#pragma unroll
    for (int k = 0; k < RW; k++) {                  // words past Lout are computed and dropped
      const u32 hi = w(q + k + 1);
      const u32 f = __funnelshift_r(lo, hi, r);
      const u32 v = f + carry;
      carry = v < f ? 1u : 0u;
      lo = hi;
      if (k < Lout) {
        o[k] = v;
        prev = v;
      } else if (k == Lout && v != ((prev >> 31) ? 0xffffffffu : 0u)) {
        atomicOr(err, SDPV_ERRBIT_OVERFLOW);
      }
    }
    return prev >> 31;
  }
  i64 q = s >> 5;
  int r = (int)(s - 32 * q);
  u64 ext = ((int32_t)word(L - 1) < 0) ? 0xffffffffull : 0ull;
  auto w = [&](i64 i) -> u64 { return i < 0 ? 0ull : (i >= L ? ext : (u64)word((int)i)); };
  i64 sb = s - 1, qb = sb >> 5;
  int rb = (int)(sb - 32 * qb);
  u64 carry = (sb >= 0) ? ((w(qb) >> rb) & 1ull) : 0ull;
  u64 lo = w(q);
#pragma unroll
  for (int k = 0; k < RW; k++) {
    u64 hi = w(q + k + 1);
    u64 v = ((((hi << 32) | lo) >> r) & 0xffffffffull) + carry;
    lo = hi;
    carry = v >> 32;
    v &= 0xffffffffull;
    if (k < Lout) {
      o[k] = (u32)v;
      prev = (u32)v;
    } else if (k == Lout && (u32)v != ((prev >> 31) ? 0xffffffffu : 0u)) {
      atomicOr(err, SDPV_ERRBIT_OVERFLOW);
    }
  }
  return prev >> 31;
}

// Byte offset of the per-warp output staging of align_rows_kernel in its dynamic shared memory.
__host__ __device__ inline size_t align_rows_stage_offset(int L) {
  return ((size_t)L * TR * (TC + 1) * 4 + 8 + TR * TC * 8 + 15) / 16 * 16;
}

// Transposed alignment into operand rows of 4 RW bytes per entry, entry (b, c, r) at row (b C + c) Rp + r:
// the Lout limbs little endian, then the sign byte (1 for a negative entry) at byte 4 Lout, then zeros; rows
// R .. Rp - 1 of every column are zero rows.  Staging as in align_t_kernel; each thread writes its rows with
// 16-byte stores.
template <int RW>
__global__ void __launch_bounds__(kThreads) align_rows_kernel(const int32_t* __restrict__ m, const i64* __restrict__ e,
                                                              int L, i64 nb, i64 R, i64 C, i64 Rp,
                                                              const i64* __restrict__ target, int per_col, int Lout,
                                                              uint8_t* __restrict__ out, unsigned* err) {
  extern __shared__ u32 sm[];                       // [L][TR][TC + 1] limbs, then [TR][TC] exponents
  i64* se = reinterpret_cast<i64*>(sm + (size_t)L * TR * (TC + 1) + ((L * TR * (TC + 1)) & 1));
  const i64 n = nb * R * C;
  const i64 b = blockIdx.z;
  const i64 r0 = (i64)blockIdx.x * TR, c0 = (i64)blockIdx.y * TC;
  const int tid = threadIdx.x;
  for (int pos = tid; pos < TR * TC; pos += kThreads) {
    const int rr = pos / TC, cc = pos % TC;
    const i64 r = r0 + rr, c = c0 + cc;
    const bool in = r < R && c < C;
    const int32_t* src = m + (in ? (b * R + r) * C + c : 0);
    u32* dst = &sm[rr * (TC + 1) + cc];
    const u32 nb4 = in ? 4u : 0u;
    for (int l = 0; l < L; l++, src += n, dst += TR * (TC + 1)) cp_async4(dst, src, nb4);
  }
  cp_async_commit();
  for (int t = tid; t < TR * TC; t += kThreads) {
    int rr = t / TC, cc = t % TC;
    i64 r = r0 + rr, c = c0 + cc;
    se[t] = (r < R && c < C) ? e[(b * R + r) * C + c] : SDPV_EZ;
  }
  cp_async_wait<0>();
  __syncthreads();
  // each warp stages its 32 rows (two columns x 16 rows, 16-byte chunks swizzled by row) and copies them out
  // 512 contiguous bytes per instruction
  const int lane = tid & 31;
  u32* stg = reinterpret_cast<u32*>(reinterpret_cast<uint8_t*>(sm) + align_rows_stage_offset(L)) + (tid >> 5) * 32 * RW;
  for (int t0 = 0; t0 < TR * TC; t0 += kThreads) {
    const int t = t0 + tid;
    const int rr = t % TR, cc = t / TR;
    const i64 r = r0 + rr, c = c0 + cc;
    u32 o[RW];
#pragma unroll
    for (int k = 0; k < RW; k++) o[k] = 0u;
    u32 sgn = 0;
    if (r < R && c < C) {
      i64 ev = se[rr * TC + cc];
      i64 s = (ev == SDPV_EZ) ? (1ll << 30) : target[per_col ? b * C + c : b * R + r] - ev;
      const u32* base = sm + rr * (TC + 1) + cc;
      sgn = shift_entry_regs<RW>([&](int i) { return base[i * TR * (TC + 1)]; }, L, s, Lout, o, err);
    }
    // word k: the limb (k < Lout), the sign byte (k == Lout), zero above (a select per static k)
    auto wd = [&](int k) { return o[k] | (k == Lout ? sgn : 0u); };
#pragma unroll
    for (int q = 0; q < RW / 4; q++)
      *reinterpret_cast<uint4*>(stg + lane * RW + 4 * (q ^ (lane & 7))) = make_uint4(wd(4 * q), wd(4 * q + 1),
                                                                                     wd(4 * q + 2), wd(4 * q + 3));
    __syncwarp();
    const i64 cA = c0 + (t0 + (tid & ~31)) / TR;          // column of lanes 0-15 (lanes 16-31: the next one)
#pragma unroll
    for (int j = 0; j < RW / 4; j++) {
      const int off = j * 512 + lane * 16;
      const int sr = off / (4 * RW), q = (off % (4 * RW)) / 16;   // staged row, 16-byte chunk
      const i64 cs = cA + (sr >= 16 ? 1 : 0);
      if (cs < C) {
        const uint4 v = *reinterpret_cast<const uint4*>(stg + sr * RW + 4 * (q ^ (sr & 7)));
        *reinterpret_cast<uint4*>(out + ((b * C + cs) * Rp + r0 + (sr & 15)) * (i64)(4 * RW) + 16 * q) = v;
      }
    }
    __syncwarp();
  }
}

inline unsigned blocks(i64 n, int t = kThreads) { return (unsigned)((n + t - 1) / t); }

}  // namespace

extern "C" int sdpv_top_max(const int32_t* m, const int64_t* e, int L, int64_t nb, int64_t R, int64_t C, int axis,
                            int64_t* out, void* stream) {
  if (L < 1 || nb < 0 || R < 0 || C < 0 || (axis != 0 && axis != 1)) return SDPV_EINVAL;
  cudaStream_t st = sdpv::as_stream(stream);
  if (axis == 1) {                                  // max over columns -> (nb, R)
    i64 nrows = nb * R;
    if (nrows == 0) return SDPV_OK;
    if (C == 0) {
      fill_kernel<<<blocks(nrows), kThreads, 0, st>>>(out, nrows, SDPV_EZ);
    } else {
      top_max_rows_kernel<<<blocks(nrows * 32), kThreads, 0, st>>>(m, e, L, nrows, C, out);
    }
    return sdpv::launch_status();
  }
  i64 ncols = nb * C;                               // max over rows -> (nb, C)
  if (ncols == 0) return SDPV_OK;
  fill_kernel<<<blocks(ncols), kThreads, 0, st>>>(out, ncols, SDPV_EZ);
  if (R > 0) {
    i64 ry = (R + 8 * kColRows - 1) / (8 * kColRows);
    if (ry > 65535 || nb > 65535) return SDPV_EINVAL;
    dim3 grid((unsigned)((C + 31) / 32), (unsigned)ry, (unsigned)nb);
    top_max_cols_kernel<<<grid, kThreads, 0, st>>>(m, e, L, nb, R, C, out);
  }
  return sdpv::launch_status();
}

extern "C" int sdpv_align_rows(const int32_t* m, const int64_t* e, int L, int64_t nb, int64_t R, int64_t C,
                               const int64_t* target, int per_col, int Lout, int64_t Rp, uint8_t* out, void* stream) {
  if (L < 1 || L > 64 || Lout < 1 || Lout > 63 || nb < 0 || R < 0 || C < 0 || nb > 65535 || Rp < R || (Rp & 127))
    return SDPV_EINVAL;
  if (nb * Rp * C == 0) return SDPV_OK;
  cudaStream_t st = sdpv::as_stream(stream);
  unsigned* err = sdpv::device_error_word();
  const int wide = Lout > 31;                          // 256-byte rows
  const size_t stage = (size_t)(kThreads / 32) * 32 * (wide ? 256 : 128);
  size_t smem = align_rows_stage_offset(L) + stage;
  const size_t smax = align_rows_stage_offset(64) + (size_t)(kThreads / 32) * 32 * 256;
  dim3 grid((unsigned)((Rp + TR - 1) / TR), (unsigned)((C + TC - 1) / TC), (unsigned)nb);
  if (grid.y > 65535 || (Rp + TR - 1) / TR > 0x7fffffff) return SDPV_EINVAL;
  static bool attr[2][64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[wide][dev & 63]) {
    cudaError_t ce = cudaFuncSetAttribute(wide ? align_rows_kernel<64> : align_rows_kernel<32>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax);
    if (ce != cudaSuccess) return sdpv::set_cuda_error(ce);
    attr[wide][dev & 63] = true;
  }
  if (wide)
    align_rows_kernel<64><<<grid, kThreads, smem, st>>>(m, e, L, nb, R, C, Rp, target, per_col, Lout, out, err);
  else
    align_rows_kernel<32><<<grid, kThreads, smem, st>>>(m, e, L, nb, R, C, Rp, target, per_col, Lout, out, err);
  return sdpv::launch_status();
}

extern "C" int sdpv_align_t(const int32_t* m, const int64_t* e, int L, int64_t nb, int64_t R, int64_t C,
                            const int64_t* target, int per_col, int Lout, int64_t Rld, int32_t* out, void* stream);

extern "C" int sdpv_align(const int32_t* m, const int64_t* e, int L, int64_t nb, int64_t R, int64_t C,
                          const int64_t* target, int per_col, int transpose, int Lout, int32_t* out, void* stream) {
  if (transpose) return sdpv_align_t(m, e, L, nb, R, C, target, per_col, Lout, R, out, stream);
  if (L < 1 || L > 64 || Lout < 1 || nb < 0 || R < 0 || C < 0 || nb > 65535) return SDPV_EINVAL;
  i64 n = nb * R * C;
  if (n == 0) return SDPV_OK;
  cudaStream_t st = sdpv::as_stream(stream);
  unsigned* err = sdpv::device_error_word();
  align_kernel<<<blocks(n), kThreads, 0, st>>>(m, e, L, nb, R, C, target, per_col, Lout, out, err);
  return sdpv::launch_status();
}

extern "C" int sdpv_align_t(const int32_t* m, const int64_t* e, int L, int64_t nb, int64_t R, int64_t C,
                            const int64_t* target, int per_col, int Lout, int64_t Rld, int32_t* out, void* stream) {
  if (L < 1 || L > 64 || Lout < 1 || nb < 0 || R < 0 || C < 0 || nb > 65535 || Rld < R) return SDPV_EINVAL;
  i64 n = nb * R * C;
  if (n == 0) return SDPV_OK;
  cudaStream_t st = sdpv::as_stream(stream);
  unsigned* err = sdpv::device_error_word();
  {
    size_t smem = (size_t)L * ATR * ATP * 4 + ATR * (TC + 1) * 8;
    static bool attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!attr[dev & 63]) {
      cudaError_t ce = cudaFuncSetAttribute(align_t_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            64 * ATR * ATP * 4 + ATR * (TC + 1) * 8);
      if (ce != cudaSuccess) return sdpv::set_cuda_error(ce);
      attr[dev & 63] = true;
    }
    const i64 tiles = ((R + ATR - 1) / ATR) * ((C + TC - 1) / TC);
    if (tiles > 0x7fffffff) return SDPV_EINVAL;
    dim3 grid((unsigned)tiles, 1, (unsigned)nb);
    align_t_kernel<<<grid, kThreads, smem, st>>>(m, e, L, nb, R, C, target, per_col, Lout, Rld, out, err);
  }
  return sdpv::launch_status();
}
