// Residue GEMM on INT8 tensor cores (north-star items (b) and (d)).
//
// Per modulus m (and block b):  acc <- (acc + A B^T) mod m  with A = 128 Ahi + Alo, B = 128 Bhi + Blo,
// i.e. 2^14 Ahi Bhi^T + 2^7 (Ahi Blo^T + Alo Bhi^T) + Alo Blo^T  (sdpvibe/rns.py:106-137,
// sdpvibe/batched.py:96-162).
//
// One CTA computes a 128 x 128 output tile of one (modulus, block):
//   * warp 0 (one lane) streams 128-byte K slices of Ahi, Alo, Bhi, Blo with TMA (128-byte swizzle,
//     out-of-range rows / K zero filled) into a 3-stage shared-memory ring;
//   * warp 1 (one lane) issues per 32-byte K step two tcgen05.mma kind::i8 of M=128, N=256:
//       TMEM[0:256)   += Ahi [Bhi; Blo]^T   -> hh | hl
//       TMEM[128:384) += Alo [Bhi; Blo]^T   -> (hl + lh) | ll
//     (Bhi and Blo sit back to back in shared memory, so one descriptor covers both; the second
//     product overlaps the first by 128 columns so the two cross terms add up in TMEM -- on the
//     first K step it is issued as two N=128 products so that only the overlap accumulates);
//   * warps 2-9 (two per TMEM lane quarter, 64 columns each) read hh, hx = hl + lh and ll per entry
//     from TMEM (one row per thread, old residues prefetched while the MMAs run), form
//     (hh mod m) 2^14 + (hx mod m) 2^7 + ll + old (exact in int32 for K <= 65536) and store its
//     canonical residue back, 16 bytes at a time where the row stride allows.
// int32 accumulation is exact for K <= 65536 (|hh|, |hl + lh| <= K 2^14).
// Syrk mode (Gram): B = A, only lower-triangle tiles are scheduled and only entries i >= j written.
#include <mutex>

#include "common.cuh"

namespace {

constexpr int kStages = 3;
constexpr u32 kSlice = 128 * 128;            // one operand slice: 128 rows x 128 bytes
constexpr int kThreads = 320;                // producer, MMA issuer, 8 epilogue warps

struct GemmSmem {
  uint8_t stage[kStages][4][kSlice];        // [ah, al, bh, bl], each 1024-aligned
  u64 full[kStages], empty[kStages], acc_full;
  u32 tmem_slot;
};

__device__ __forceinline__ void tile_of(int t, int mode, int ntn, int& tm, int& tn) {
  if (mode == 0) {
    tm = t / ntn;
    tn = t - tm * ntn;
  } else {                                    // lower-triangle enumeration: t = tm(tm+1)/2 + tn
    int a = (int)((sqrtf(8.f * t + 1.f) - 1.f) * 0.5f);
    while ((a + 1) * (a + 2) / 2 <= t) a++;
    while (a * (a + 1) / 2 > t) a--;
    tm = a;
    tn = t - a * (a + 1) / 2;
  }
}

__global__ void __launch_bounds__(kThreads, 1)
    rns_gemm_kernel(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
                    const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl,
                    int16_t* __restrict__ acc, i64 ldc, const int32_t* __restrict__ mods, const float* __restrict__ minvs,
                    const int32_t* __restrict__ c14s, int g0, i64 nb, i64 M, i64 N, i64 KC, int mode, int ntn,
                    unsigned* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  GemmSmem& S = *reinterpret_cast<GemmSmem*>((uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int tm, tn;
  tile_of(blockIdx.x, mode, ntn, tm, tn);
  const int b = blockIdx.y, g = blockIdx.z;
  const int m0 = tm * 128, n0 = tn * 128;
  const int nk = (int)((KC + 127) / 128);

  if (tid == 0) {
    for (int s = 0; s < kStages; s++) {
      mbar_init(&S.full[s], 1);
      mbar_init(&S.empty[s], 1);
    }
    mbar_init(&S.acc_full, 1);
    mbar_fence_init();
  }
  if (warp == 1) {
    tmem_alloc(&S.tmem_slot, 512);
    tmem_relinquish();
  }
  __syncthreads();
  tc_fence_after();
  const u32 tmem = S.tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      for (int kb = 0; kb < nk; kb++) {
        int s = kb % kStages;
        if (kb >= kStages && !mbar_wait(&S.empty[s], ((kb / kStages) - 1) & 1, err)) break;
        mbar_expect_tx(&S.full[s], 4 * kSlice);
        int kx = kb * 128;
        tma_load_4d(S.stage[s][0], &mAh, &S.full[s], kx, m0, b, g);
        tma_load_4d(S.stage[s][1], &mAl, &S.full[s], kx, m0, b, g);
        tma_load_4d(S.stage[s][2], &mBh, &S.full[s], kx, n0, b, g);
        tma_load_4d(S.stage[s][3], &mBl, &S.full[s], kx, n0, b, g);
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const u32 idesc = idesc_i8(128, 256), idesc128 = idesc_i8(128, 128);
      bool ok = true;
      for (int kb = 0; kb < nk && ok; kb++) {
        int s = kb % kStages;
        if (!mbar_wait(&S.full[s], (kb / kStages) & 1, err)) {
          ok = false;
          break;
        }
        tc_fence_after();
        u32 ah = smem_u32(S.stage[s][0]), al = smem_u32(S.stage[s][1]), bh = smem_u32(S.stage[s][2]);
#pragma unroll
        for (int ks = 0; ks < 4; ks++) {
          u64 bd = sdesc_sw128(bh + 32 * ks);
          if ((kb | ks) == 0) {
            mma_i8(tmem + 0, sdesc_sw128(ah), bd, idesc, 0u);                         // hh | hl
            mma_i8(tmem + 256, sdesc_sw128(al), sdesc_sw128(bh + kSlice), idesc128, 0u);  // ll
            mma_i8(tmem + 128, sdesc_sw128(al), bd, idesc128, 1u);                      // hl += lh
          } else {
            mma_i8(tmem + 0, sdesc_sw128(ah + 32 * ks), bd, idesc, 1u);
            mma_i8(tmem + 128, sdesc_sw128(al + 32 * ks), bd, idesc, 1u);
          }
        }
        mma_commit(&S.empty[s]);
      }
      mma_commit(&S.acc_full);
    }
  } else {
    // Epilogue: warps 2..9 -> TMEM lane quarter (warp & 3), column half (warp - 2) / 4.
    const int q = warp & 3, ch = (warp - 2) >> 2;
    const i64 i = m0 + q * 32 + lane;                 // output row within the block
    const int gg = g0 + g;
    const int m = mods[gg], c14 = c14s[gg];
    const float minv = minvs[gg];
    int16_t* rowp = acc + ((i64)gg * nb * M + (i64)b * M + i) * ldc;
    const bool vec = ((ldc & 7) == 0) && ((((uintptr_t)acc) & 15) == 0);
    // the old residues do not depend on the products: load them before waiting for the MMAs
    int16_t olds[2][32];
#pragma unroll
    for (int c = 0; c < 2; c++) {
      const i64 nc = n0 + 64 * ch + 32 * c;
      const bool full = vec && i < M && nc + 32 <= N && (mode == 0 || nc + 31 <= i);
      if (full) {
#pragma unroll
        for (int v4 = 0; v4 < 4; v4++)
          *reinterpret_cast<uint4*>(olds[c] + 8 * v4) = reinterpret_cast<const uint4*>(rowp + nc)[v4];
      } else {
#pragma unroll
        for (int j = 0; j < 32; j++)
          olds[c][j] = (i < M && nc + j < N && (mode == 0 || nc + j <= i)) ? rowp[nc + j] : (int16_t)0;
      }
    }
    const bool ok = mbar_wait(&S.acc_full, 0, err);
    tc_fence_after();
#pragma unroll
    for (int c = 0; c < 2; c++) {
      u32 hh[32], hx[32], ll[32];
      u32 base = tmem + ((u32)(q * 32) << 16) + 64 * ch + 32 * c;
      tmem_ld32(base, hh);
      tmem_ld32(base + 128, hx);
      tmem_ld32(base + 256, ll);
      tmem_ld_wait();
      if (!ok || i >= M) continue;
      const i64 nc = n0 + 64 * ch + 32 * c;
      if (nc >= N) continue;
      const bool full = vec && nc + 32 <= N && (mode == 0 || nc + 31 <= i);
      int16_t* old = olds[c];
#pragma unroll
      for (int j = 0; j < 32; j++) {
        // (hh mod m) and (hx mod m) as |r| <= m/2 + m/300 representatives, then the canonical residue
        int a = (int)hh[j], x = (int)hx[j];
        int ra = a - (__float_as_int(fmaf((float)a, minv, 12582912.0f)) - 0x4B400000) * m;
        int rx = x - (__float_as_int(fmaf((float)x, minv, 12582912.0f)) - 0x4B400000) * m;
        int v = ra * c14 + rx * 128 + (int)ll[j] + (int)old[j];
        int r = v - (__float_as_int(fmaf((float)v, minv, 12582912.0f)) - 0x4B400000) * m;
        r += (r < 0) ? m : 0;
        r -= (r >= m) ? m : 0;
        old[j] = (int16_t)r;
      }
      if (full) {
#pragma unroll
        for (int v4 = 0; v4 < 4; v4++)
          reinterpret_cast<uint4*>(rowp + nc)[v4] = *reinterpret_cast<const uint4*>(old + 8 * v4);
      } else {
        for (int j = 0; j < 32; j++)
          if (nc + j < N && (mode == 0 || nc + j <= i)) rowp[nc + j] = old[j];
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) tmem_dealloc(tmem, 512);
}

// 4-D int8 map over (K, rows, nb, G) with 128 x 128 boxes and 128-byte swizzle; gstride = bytes between
// the planes of consecutive moduli (>= K*rows*nb).
bool make_map(CUtensorMap* map, const void* base, i64 K, i64 rows, i64 nb, i64 G, i64 gstride) {
  sdpv::EncodeTiledFn fn = sdpv::encode_tiled_fn();
  if (!fn) return false;
  cuuint64_t dims[4] = {(cuuint64_t)K, (cuuint64_t)rows, (cuuint64_t)nb, (cuuint64_t)G};
  cuuint64_t strides[3] = {(cuuint64_t)K, (cuuint64_t)(K * rows), (cuuint64_t)gstride};
  cuuint32_t box[4] = {128, 128, 1, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace

extern "C" int sdpv_rns_gemm(const sdpv_ctx* c, const int8_t* Ahi, const int8_t* Alo, const int8_t* Bhi,
                             const int8_t* Blo, int64_t a_stride, int64_t b_stride, int16_t* acc, int64_t ldc, int g0,
                             int G, int64_t nb, int64_t M, int64_t N, int64_t KC, int mode, void* stream) {
  if (!c || g0 < 0 || G < 1 || g0 + G > c->d.n || nb < 1 || M < 0 || N < 0 || KC < 0 || KC > 65536 ||
      (KC & 15) || (mode != 0 && mode != 1) || nb > 65535 || G > 65535)
    return SDPV_EINVAL;
  if (mode == 1) {
    Bhi = Ahi;
    Blo = Alo;
    N = M;
    b_stride = a_stride;
  }
  if (!a_stride) a_stride = KC * M * nb;
  if (!b_stride) b_stride = KC * N * nb;
  if (a_stride < KC * M * nb || b_stride < KC * N * nb || (a_stride & 15) || (b_stride & 15)) return SDPV_EINVAL;
  if (ldc < N) return SDPV_EINVAL;
  if (M == 0 || N == 0 || KC == 0) return SDPV_OK;
  if (((uintptr_t)Ahi | (uintptr_t)Alo | (uintptr_t)Bhi | (uintptr_t)Blo) & 15) return SDPV_EINVAL;
  CUtensorMap mAh, mAl, mBh, mBl;
  if (!make_map(&mAh, Ahi, KC, M, nb, G, a_stride) || !make_map(&mAl, Alo, KC, M, nb, G, a_stride) ||
      !make_map(&mBh, Bhi, KC, N, nb, G, b_stride) || !make_map(&mBl, Blo, KC, N, nb, G, b_stride))
    return SDPV_EINVAL;
  size_t smem = sizeof(GemmSmem) + 1024;
  static std::once_flag attr;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(attr, [&] {
    attr_err = cudaFuncSetAttribute(rns_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
  if (attr_err != cudaSuccess) return sdpv::set_cuda_error(attr_err);
  int ntm = (int)((M + 127) / 128), ntn = (int)((N + 127) / 128);
  i64 tiles = mode == 0 ? (i64)ntm * ntn : (i64)ntm * (ntm + 1) / 2;
  if (tiles > 0x7fffffff) return SDPV_EINVAL;
  dim3 grid((unsigned)tiles, (unsigned)nb, (unsigned)G);
  rns_gemm_kernel<<<grid, kThreads, smem, sdpv::as_stream(stream)>>>(
      mAh, mAl, mBh, mBl, acc, ldc, c->d.mods, c->d.minv, c->d.c14, g0, nb, M, N, KC, mode, ntn,
      sdpv::device_error_word());
  return sdpv::launch_status();
}
