// Residue decomposition (north-star item (a)): limb planes -> int8 hi/lo residues modulo 15-bit primes.
//
// For an entry x with bytes u_j (j < 4L, little endian, two's complement) and a modulus m:
//   x mod m = (sum_j (u_j - 128) T_j + C1 - neg*C2) mod m,  T_j = centred 256^j mod m = 128 Thi_j + Tlo_j
// (sdpvibe/rns.py:66-103, tables rns.py:179-184).  The byte-by-table contraction runs on the tensor
// cores as D = T * X^T with tcgen05.mma kind::i8: A = the table (128 moduli x 4L bytes, resident in
// shared memory for the whole persistent CTA), B = 128 entries x 4L bytes staged from the limb
// planes, D = two int32 accumulators (Tlo, Thi) of 128 x 128 in TMEM.  TMEM lane = modulus, so in the
// epilogue each thread reduces one modulus for 32 consecutive entries and stores 32 contiguous
// residue bytes per plane.  The next tile's limbs are loaded into registers while the current tile
// is reduced, and two CTAs share each SM, so the kernel stays close to HBM speed.
#include "common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kTile = 128;          // entries per tile (MMA N)
constexpr u32 kTileBytes = 128 * 128;

template <int KT>
struct ResSmem {
  uint8_t tab_lo[KT][kTileBytes];   // A operand images (1024-aligned)
  uint8_t tab_hi[KT][kTileBytes];
  uint8_t xb[KT][kTileBytes];       // B operand: entry bytes
  uint8_t neg[kTile];
  u64 bar_tab, bar_mma;
  u32 tmem_slot;
  int abort;
};

template <int KT>
__global__ void __launch_bounds__(kThreads, 2)
    residues_kernel(const int32_t* __restrict__ X, int L, i64 rows, i64 ld, i64 k0, i64 kc, i64 kp, int g0, int G,
                    int group0, const uint8_t* __restrict__ tab, int ngroups_ctx, const int32_t* __restrict__ mods,
                    const float* __restrict__ minvs, const int32_t* __restrict__ c1s,
                    const int32_t* __restrict__ c1m2s, int n, int8_t* __restrict__ Rhi, int8_t* __restrict__ Rlo,
                    unsigned* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  ResSmem<KT>& S = *reinterpret_cast<ResSmem<KT>*>((uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int grp = group0 + blockIdx.y;                 // 128-modulus group of the table
  const i64 nent = rows * kp;
  const i64 ntiles = (nent + kTile - 1) / kTile;
  const i64 plane = rows * ld;
  const int nchunks = (L + 3) / 4;                     // 16-byte chunks of an entry (4 limbs each)

  if (tid == 0) {
    mbar_init(&S.bar_tab, 1);
    mbar_init(&S.bar_mma, 1);
    S.abort = 0;
    mbar_fence_init();
  }
  if (warp == 0) {
    tmem_alloc(&S.tmem_slot, 256);
    tmem_relinquish();
  }
  __syncthreads();
  tc_fence_after();
  const u32 tmem = S.tmem_slot;
  if (tid == 0) {
    mbar_expect_tx(&S.bar_tab, 2 * KT * kTileBytes);
    const uint8_t* src = tab + (size_t)grp * 2 * KT * kTileBytes;
    bulk_load(&S.tab_lo[0][0], src, KT * kTileBytes, &S.bar_tab);
    bulk_load(&S.tab_hi[0][0], src + (size_t)KT * kTileBytes, KT * kTileBytes, &S.bar_tab);
  }

  // Each thread stages chunks c = half, half+2, ... of entry `ent` (4 limbs = one 16-byte chunk).
  const int ent = tid & (kTile - 1), half = tid >> 7;
  constexpr int kMaxChunks = 8 * KT;                   // 16-byte chunks per entry row, split over two threads
  uint4 regs[(kMaxChunks + 1) / 2];
  int negbit = 0;
  auto load_tile = [&](i64 tile) {
    i64 e = tile * kTile + ent;
    i64 i = e / kp, k = e - (e / kp) * kp;
    bool ok = (e < nent) && (k < kc);
    const int32_t* base = X + i * ld + k0 + k;
    negbit = 0;
#pragma unroll
    for (int q = 0; q < (kMaxChunks + 1) / 2; q++) {
      int c = half + 2 * q;
      u32 w[4] = {0u, 0u, 0u, 0u};
      if (c < nchunks && ok) {
#pragma unroll
        for (int t = 0; t < 4; t++) {
          int l = 4 * c + t;
          if (l < L) w[t] = (u32)__ldg(base + (i64)l * plane);
        }
      }
      if (ok && c == (L - 1) / 4) negbit = (int)(w[(L - 1) & 3] >> 31);
      regs[q] = make_uint4(w[0] ^ 0x80808080u, w[1] ^ 0x80808080u, w[2] ^ 0x80808080u, w[3] ^ 0x80808080u);
    }
  };
  auto store_tile = [&]() {
#pragma unroll
    for (int q = 0; q < (kMaxChunks + 1) / 2; q++) {
      int c = half + 2 * q;
      if (c < 8 * KT) {
        int kt = c >> 3, cc = c & 7;
        *reinterpret_cast<uint4*>(&S.xb[kt][sw128_off(ent, cc)]) = regs[q];
      }
    }
    if (half == (((L - 1) / 4) & 1)) S.neg[ent] = (uint8_t)negbit;
  };

  // Per-thread modulus (TMEM lane) and column half for the epilogue.
  const int quarter = warp & 3, colhalf = warp >> 2;
  const int row = quarter * 32 + lane;
  const int g = grp * 128 + row;
  const bool gvalid = (g >= g0) && (g < g0 + G) && (g < n);
  int m = 1, c1 = 0, c1m2 = 0;
  float minv = 1.f;
  if (gvalid) {
    m = mods[g];
    minv = minvs[g];
    c1 = c1s[g];
    c1m2 = c1m2s[g];
  }
  int8_t* outh = Rhi + (i64)(g - g0) * nent;
  int8_t* outl = Rlo + (i64)(g - g0) * nent;
  const u32 idesc = idesc_i8(128, kTile);

  i64 tile = blockIdx.x;
  if (tile < ntiles) load_tile(tile);
  if (!mbar_wait(&S.bar_tab, 0, err)) S.abort = 1;
  u32 phase = 0;
  for (; tile < ntiles; tile += gridDim.x) {
    store_tile();
    fence_proxy_async_smem();
    __syncthreads();
    if (S.abort) break;
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int kt = 0; kt < KT; kt++)
#pragma unroll
        for (int s = 0; s < 4; s++) {
          u64 bd = sdesc_sw128(smem_u32(&S.xb[kt][0]) + 32 * s);
          u32 accum = (kt | s) ? 1u : 0u;
          mma_i8(tmem + 0, sdesc_sw128(smem_u32(&S.tab_lo[kt][0]) + 32 * s), bd, idesc, accum);
          mma_i8(tmem + 128, sdesc_sw128(smem_u32(&S.tab_hi[kt][0]) + 32 * s), bd, idesc, accum);
        }
      mma_commit(&S.bar_mma);
    }
    i64 next = tile + gridDim.x;
    if (next < ntiles) load_tile(next);                // overlaps the MMA and the epilogue below
    if (!mbar_wait(&S.bar_mma, phase, err)) S.abort = 1;
    phase ^= 1;
    tc_fence_after();
#pragma unroll 1
    for (int c = 0; c < 2; c++) {
      const int col = colhalf * 64 + c * 32;
      u32 lo[32], hi[32];
      tmem_ld32(tmem + ((u32)(quarter * 32) << 16) + col, lo);
      tmem_ld32(tmem + ((u32)(quarter * 32) << 16) + 128 + col, hi);
      tmem_ld_wait();
      if (!gvalid) continue;
      const i64 e0 = tile * kTile + col;
      u32 ph[8], pl[8];
#pragma unroll
      for (int j = 0; j < 32; j++) {
        int v = 128 * (int)hi[j] + (int)lo[j] + (S.neg[col + j] ? c1m2 : c1);
        int r = mod_exact(v, m, minv);
        r -= (r > (m >> 1)) ? m : 0;
        int l8 = ((r + 64) & 127) - 64;
        int h8 = (r - l8) >> 7;
        if ((j & 3) == 0) {
          ph[j >> 2] = 0;
          pl[j >> 2] = 0;
        }
        ph[j >> 2] |= (u32)(h8 & 255) << (8 * (j & 3));
        pl[j >> 2] |= (u32)(l8 & 255) << (8 * (j & 3));
      }
      if (e0 + 32 <= nent && ((((uintptr_t)(outh + e0)) | ((uintptr_t)(outl + e0))) & 15) == 0) {
        uint4* dh = reinterpret_cast<uint4*>(outh + e0);
        uint4* dl = reinterpret_cast<uint4*>(outl + e0);
        dh[0] = make_uint4(ph[0], ph[1], ph[2], ph[3]);
        dh[1] = make_uint4(ph[4], ph[5], ph[6], ph[7]);
        dl[0] = make_uint4(pl[0], pl[1], pl[2], pl[3]);
        dl[1] = make_uint4(pl[4], pl[5], pl[6], pl[7]);
      } else {
        for (int j = 0; j < 32 && e0 + j < nent; j++) {
          outh[e0 + j] = (int8_t)(ph[j >> 2] >> (8 * (j & 3)));
          outl[e0 + j] = (int8_t)(pl[j >> 2] >> (8 * (j & 3)));
        }
      }
    }
    tc_fence_before();
    __syncthreads();
    if (S.abort) break;
  }
  if (S.abort && tid == 0) {
    // A wait gave up: let any committed MMAs drain (bounded) before TMEM is released.
    mbar_wait(&S.bar_mma, phase, err);
  }
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 256);
}

int num_sms() {
  static int cached[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < 64 && cached[dev]) return cached[dev];
  int v = 148;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  if (dev >= 0 && dev < 64) cached[dev] = v;
  return v;
}

template <int KT>
int launch_residues(const sdpv_ctx* c, const int32_t* X, i64 rows, i64 ld, i64 k0, i64 kc, i64 kp, int g0, int G,
                    int8_t* Rhi, int8_t* Rlo, cudaStream_t st) {
  const sdpv::CtxDev& d = c->d;
  size_t smem = sizeof(ResSmem<KT>) + 1024;
  if (smem < 80 * 1024) smem = 80 * 1024;               // at most two CTAs (2 x 256 TMEM columns) per SM
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(residues_kernel<KT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return sdpv::set_cuda_error(e);
    attr_set[dev & 63] = true;
  }
  int grp0 = g0 / 128, grp1 = (g0 + G - 1) / 128;
  i64 ntiles = (rows * kp + kTile - 1) / kTile;
  i64 gx = 2 * (i64)num_sms();
  if (gx > ntiles) gx = ntiles;
  dim3 grid((unsigned)gx, (unsigned)(grp1 - grp0 + 1));
  residues_kernel<KT><<<grid, kThreads, smem, st>>>(X, d.L, rows, ld, k0, kc, kp, g0, G, grp0, d.tab, d.npad / 128,
                                                     d.mods, d.minv, d.c1, d.c1m2, d.n, Rhi, Rlo,
                                                     sdpv::device_error_word());
  return sdpv::launch_status();
}

}  // namespace

extern "C" int sdpv_residues(const sdpv_ctx* c, const int32_t* X, int64_t rows, int64_t ld, int64_t k0, int64_t kc,
                             int g0, int G, int8_t* Rhi, int8_t* Rlo, void* stream) {
  if (!c || rows < 0 || kc < 0 || k0 < 0 || k0 + kc > ld || g0 < 0 || G < 1 || g0 + G > c->d.n) return SDPV_EINVAL;
  i64 kp = (kc + 15) / 16 * 16;
  if (rows == 0 || kp == 0) return SDPV_OK;
  cudaStream_t st = sdpv::as_stream(stream);
  switch (c->d.kt) {
    case 1: return launch_residues<1>(c, X, rows, ld, k0, kc, kp, g0, G, Rhi, Rlo, st);
    case 2: return launch_residues<2>(c, X, rows, ld, k0, kc, kp, g0, G, Rhi, Rlo, st);
    default: return SDPV_EINVAL;                        // L > 64
  }
}
