// Residue decomposition: limb planes -> int8 hi/lo residues modulo 15-bit primes.
//
// For an entry x with bytes u_j (j < 4L, little endian, two's complement) and a modulus m:
//   x mod m = (sum_j (u_j - 128) T_j + C1 - neg*C2) mod m,  T_j = centred 256^j mod m = 128 Thi_j + Tlo_j
// (sdpvibe/rns.py:66-103, tables rns.py:179-184).  The byte-by-table contraction runs on the tensor
// cores as D = T * X^T with tcgen05.mma kind::i8; two extra K columns (a constant byte 1 against C1
// and the sign byte against -C2) make the product congruent to x itself, so the epilogue is only an
// exact centred reduction and the int8 digit split.  A = the table (128 moduli x 4L+2 bytes, resident in
// shared memory for the whole persistent CTA), B = 128 entries x 4L bytes staged from the limb
// planes, D = two int32 accumulators (Tlo, Thi) of 128 x 128 in TMEM.  TMEM lane = modulus, so in the
// epilogue each thread reduces one modulus for 32 consecutive entries and stores 32 contiguous
// residue bytes per plane.  The next tile's limbs are loaded into registers while the current tile
// is reduced, and several CTAs share each SM so their phases overlap.
//
// The warp-specialised kernel (L <= 63) uses unsigned operands instead: the limb bytes u_j as they are
// and a sign byte against the canonical digits of 256^j mod m (hi = t >> 7, lo = t & 127) and of
// (-2^(32L)) mod m, as u8 x u8 products.  v = 128 D_hi + D_lo is then congruent to x, non-negative and
// below 2^31, so the canonical residue comes from an exact Barrett quotient floor(v ceil(2^46/m) / 2^46)
// with no float estimate and no correction step.
#include <cstdlib>
#include <cstring>

#include "common.cuh"

namespace {

constexpr u32 kTileBytes = 128 * 128;

// TILE entries per MMA (N), THREADS per CTA; TMEM holds the two accumulators (2*TILE columns), so
// 512 / (2*TILE) CTAs share an SM and overlap each other's load / MMA / reduce phases.
constexpr int kStages = 3;          // raw limb tiles in flight per CTA

template <int KT, int TILE>
struct ResSmem {
  uint8_t tab_lo[KT][kTileBytes];   // A operand images (1024-aligned)
  uint8_t tab_hi[KT][kTileBytes];
  uint8_t xb[KT][TILE * 128];       // B operand: entry bytes (TILE rows of 128 bytes per K tile)
  u32 raw[kStages][32 * KT - 1][TILE];  // limb planes of the next tiles, filled by cp.async
  u64 bar_tab, bar_mma;
  u32 tmem_slot;
  int abort;
};

// Digits of the residue of v (congruent to the entry mod m): round(v / m) from the float estimate (off by
// at most one), then either the centred residue r in [-(m >> 1), m >> 1] split r = 128 hi + lo, lo in
// [-64, 64) (the API format, int8 digits) or, for the GEMM's internal operands (U8), the canonical residue
// r in [0, m) split hi = r >> 7 in [0, 256), lo = r & 127 (unsigned digits, one correction fewer).
template <bool U8>
__device__ __forceinline__ void residue_digits(int v, int m, int hm, float minv, int& hb, int& lb) {
  const float t = fmaf((float)v, minv, 12582912.0f);               // round(v/m) in the low mantissa
  int r = v - (__float_as_int(t) - 0x4B400000) * m;                // |r| <= m/2 + m/300
  if (U8) {
    r += (r < 0) ? m : 0;
    hb = r >> 7;
    lb = r & 127;
  } else {
    r -= (r > hm) ? m : 0;                                         // exact centring
    r += (r < -hm) ? m : 0;
    hb = (r + 64) >> 7;
    lb = r - (hb << 7);
  }
}

template <int KT, int TILE, int THREADS, bool U8>
__global__ void __launch_bounds__(THREADS, 512 / (2 * TILE))
    residues_kernel(const int32_t* __restrict__ X, int L, i64 rows, i64 ld, i64 k0, i64 kc, i64 kp, int g0, int G,
                    int group0, const uint8_t* __restrict__ tab, const int32_t* __restrict__ mods,
                    const float* __restrict__ minvs, int n, int8_t* __restrict__ Rhi, int8_t* __restrict__ Rlo, i64 pstride,
                    unsigned* __restrict__ err) {
  constexpr int P = THREADS / TILE;                    // loader threads per entry
  constexpr int W = THREADS / 32;
  constexpr int COLS_PER_WARP = TILE * 4 / W;          // epilogue columns per warp (multiple of 32)
  constexpr int kMaxChunks = 8 * KT;                   // 16-byte chunks per entry row
  constexpr int kRegs = (kMaxChunks + P - 1) / P;
  constexpr u32 TCOLS = 2 * TILE;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  ResSmem<KT, TILE>& S =
      *reinterpret_cast<ResSmem<KT, TILE>*>((uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int grp = group0 + blockIdx.y;                 // 128-modulus group of the table
  const i64 nent = rows * kp;
  const i64 ntiles = (nent + TILE - 1) / TILE;
  const i64 plane = rows * ld;

  if (tid == 0) {
    mbar_init(&S.bar_tab, 1);
    mbar_init(&S.bar_mma, 1);
    S.abort = 0;
    mbar_fence_init();
  }
  if (warp == 0) {
    tmem_alloc(&S.tmem_slot, TCOLS);
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

  // Loader: the limb words of a tile land in raw[stage][limb][entry] by 4-byte cp.async (zero fill for
  // entries past the end or in the k padding); the transform then packs entry rows of 16-byte chunks:
  // limbs XOR 0x80808080 (signed bytes u - 128), word L = constant byte 1 | sign byte << 8, zeros after.
  const int ent = tid % TILE, part = tid / TILE;
  auto issue_tile = [&](i64 tile, int stage) {
    if (tile < ntiles) {
      i64 e = tile * TILE + ent;
      i64 i = e / kp, k = e - (e / kp) * kp;
      bool ok = (e < nent) && (k < kc);
      const int32_t* base = X + (ok ? i * ld + k0 + k : 0);
      for (int l = part; l < L; l += P) cp_async4(&S.raw[stage][l][ent], base + (ok ? (i64)l * plane : 0), ok ? 4u : 0u);
    }
    cp_async_commit();
  };
  auto transform = [&](int stage) {
#pragma unroll
    for (int q = 0; q < kRegs; q++) {
      int c = part + P * q;
      if (c >= kMaxChunks) continue;
      u32 w[4];
#pragma unroll
      for (int t = 0; t < 4; t++) {
        int l = 4 * c + t;
        if (l < L) w[t] = S.raw[stage][l][ent] ^ 0x80808080u;
        else if (l == L) w[t] = 1u | ((S.raw[stage][L - 1][ent] >> 31) << 8);
        else w[t] = 0u;
      }
      *reinterpret_cast<uint4*>(&S.xb[c >> 3][sw128_off(ent, c & 7)]) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  };

  // Epilogue: TMEM lane = modulus of this 128-modulus group.
  const int quarter = warp & 3, colgroup = warp >> 2;
  const int row = quarter * 32 + lane;
  const int g = grp * 128 + row;
  const bool gvalid = (g >= g0) && (g < g0 + G) && (g < n);
  int m = 1;
  float minv = 1.f;
  if (gvalid) {
    m = mods[g];
    minv = minvs[g];
  }
  const int hm = m >> 1;
  int8_t* outh = Rhi + (i64)(g - g0) * pstride;
  int8_t* outl = Rlo + (i64)(g - g0) * pstride;
  const u32 idesc = idesc_i8(128, TILE);

  i64 tile = blockIdx.x;
#pragma unroll
  for (int st = 0; st < kStages; st++) issue_tile(tile + (i64)st * gridDim.x, st);
  if (!mbar_wait(&S.bar_tab, 0, err)) S.abort = 1;
  u32 phase = 0;
  for (int it = 0; tile < ntiles; tile += gridDim.x, it++) {
    const int stage = it % kStages;
    cp_async_wait<kStages - 1>();
    __syncthreads();
    transform(stage);
    fence_proxy_async_smem();
    __syncthreads();
    if (S.abort) break;
    issue_tile(tile + (i64)kStages * gridDim.x, stage);   // refill the stage just consumed
    if (tid == 0) {
      tc_fence_after();
#pragma unroll
      for (int kt = 0; kt < KT; kt++)
#pragma unroll
        for (int s = 0; s < 4; s++) {
          u64 bd = sdesc_sw128(smem_u32(&S.xb[kt][0]) + 32 * s);
          u32 accum = (kt | s) ? 1u : 0u;
          mma_i8(tmem + 0, sdesc_sw128(smem_u32(&S.tab_lo[kt][0]) + 32 * s), bd, idesc, accum);
          mma_i8(tmem + TILE, sdesc_sw128(smem_u32(&S.tab_hi[kt][0]) + 32 * s), bd, idesc, accum);
        }
      mma_commit(&S.bar_mma);
    }
    if (!mbar_wait(&S.bar_mma, phase, err)) S.abort = 1;
    phase ^= 1;
    tc_fence_after();
#pragma unroll 1
    for (int c = 0; c < COLS_PER_WARP / 32; c++) {
      const int col = colgroup * COLS_PER_WARP + c * 32;
      u32 lo[32], hi[32];
      tmem_ld32(tmem + ((u32)(quarter * 32) << 16) + col, lo);
      tmem_ld32(tmem + ((u32)(quarter * 32) << 16) + TILE + col, hi);
      tmem_ld_wait();
      if (!gvalid) continue;
      const i64 e0 = tile * TILE + col;
      u32 ph[8], pl[8];
#pragma unroll
      for (int j = 0; j < 32; j += 4) {
        int hb[4], lb[4];
#pragma unroll
        for (int u = 0; u < 4; u++)
          residue_digits<U8>(128 * (int)hi[j + u] + (int)lo[j + u], m, hm, minv, hb[u], lb[u]);
        ph[j >> 2] = __byte_perm(__byte_perm(hb[0], hb[1], 0x0040), __byte_perm(hb[2], hb[3], 0x0040), 0x5410);
        pl[j >> 2] = __byte_perm(__byte_perm(lb[0], lb[1], 0x0040), __byte_perm(lb[2], lb[3], 0x0040), 0x5410);
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
  if (warp == 0) tmem_dealloc(tmem, TCOLS);
}

// ---------------------------------------------------------------- warp-specialised persistent variant
// One CTA per SM, 6 + RW warps (RW = 8 reducer warps, or 16):
//   warps 0-3  loaders: the next tiles' limb planes into a raw ring (RAW stages) -- one 3-D TMA copy per
//              tile (MODE 2) or per-thread 16- / 4-byte cp.async (MODE 0) -- then the transform into a
//              double-buffered K-major entry tile (xb[2]); in MODE 1 one thread streams operand rows by TMA;
//   warp 4     MMA issuer (one lane): D_lo / D_hi of a 128-entry tile into one of two TMEM buffers;
//   warps 5..  reducers: TMEM lane quarter = warp % 4, 128 / (RW / 4) entries each; exact residue, digit
//              split, staging of the residue tile (or direct stores where bulk stores cannot be used);
//   last warp  store warp (one lane): the bulk tensor stores of each staged tile, releasing its staging
//              buffer once read (stg_full: reducer arrivals, stg_empty: the store lane).
// mbarriers: xb_full (loader arrivals, or the TMA bytes in MODE 1), xb_empty (MMA commit), tm_full (MMA
// commit), tm_empty (reducer arrivals), raw_full (TMA bytes, MODE 2).  Every wait is bounded; a timeout
// aborts all roles.
constexpr int WS_TILE = 128, WS_LOADERS = 128;
// RW reducer warps (8 or 16): RW / 4 per TMEM lane quarter, 128 / (RW / 4) columns each
template <int RW>
constexpr int ws_threads() { return WS_LOADERS + 32 + 32 * RW + 32; }      // + the store warp

template <int KT, int RAW, int STG>
struct WsSmem {
  uint8_t tab_lo[KT][kTileBytes];
  uint8_t tab_hi[KT][kTileBytes];
  uint8_t xb[2][KT][WS_TILE * 128];
  uint8_t out[STG][2][kTileBytes];      // residue tiles (128 moduli x 128 entries, hi | lo), 128-byte swizzle
  u32 raw[RAW][32 * KT - 1][WS_TILE];
  u64 bar_tab, xb_full[2], xb_empty[2], tm_full[2], tm_empty[2], raw_full[RAW];
  u64 stg_full[STG], stg_empty[STG];     // staged residue tile complete / read by its bulk store
  u32 tmem_slot;
  volatile int abort;
};

__device__ __forceinline__ void named_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}
// Named barrier that also ORs a predicate over the participating threads (uniform decision).
__device__ __forceinline__ bool named_sync_or(int id, int nthreads, bool pred) {
  u32 out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, %2, %3, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(out)
      : "r"((u32)pred), "r"(id), "r"(nthreads)
      : "memory");
  return out != 0;
}

// MODE 0: limb planes by per-thread cp.async, tiles of 128 consecutive entries (i kp + k enumeration), 2-D
//   residue stores (or per-thread stores).
// MODE 1: operand rows (4 L limb bytes, a sign byte, zeros; 128 KT bytes per entry) from sdpv_align_rows,
//   entry (i, k) at row i Rp + k0 + k: thread 0 of the loaders streams each tile's rows straight into the
//   K-major operand buffer with TMA (map_in); no transform.
// MODE 2: limb planes by TMA: thread 0 loads each tile's L x 128 words with one 3-D copy (map_in over
//   (kc, rows, L) from X + k0; words past kc zero filled) into the raw ring; the loaders transform as in
//   MODE 0.
// MODEs 1 and 2 use tiles (i, 128-entry block of k) (tpi blocks per i) and 3-D residue stores over
// (kp, rows, G), clipped at kp.
template <int KT, int RAW, int STG, bool U8, int RW, int MODE>
__global__ void __launch_bounds__(ws_threads<RW>(), 1)
    residues_ws_kernel(const __grid_constant__ CUtensorMap map_hi, const __grid_constant__ CUtensorMap map_lo,
                       const __grid_constant__ CUtensorMap map_in, i64 Rp, i64 tpi,
                       int use_tma, int vec, const int32_t* __restrict__ X, int L, i64 rows, i64 ld, i64 k0, i64 kc, i64 kp,
                       int g0, int G,
                       int group0, const uint8_t* __restrict__ tab, const int32_t* __restrict__ mods,
                       const float* __restrict__ minvs, int n, int8_t* __restrict__ Rhi, int8_t* __restrict__ Rlo, i64 pstride,
                       unsigned* __restrict__ err) {
  constexpr int kMaxChunks = 8 * KT;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  WsSmem<KT, RAW, STG>& S =
      *reinterpret_cast<WsSmem<KT, RAW, STG>*>((uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int grp = group0 + blockIdx.y;
  const i64 nent = rows * kp;
  constexpr bool TILED = MODE != 0;
  const i64 ntiles = TILED ? rows * tpi : (nent + WS_TILE - 1) / WS_TILE;
  const i64 plane = rows * ld;
  const int niter = blockIdx.x < ntiles ? (int)((ntiles - 1 - blockIdx.x) / gridDim.x + 1) : 0;

  if (tid == 0) {
    mbar_init(&S.bar_tab, 1);
    for (int b = 0; b < 2; b++) {
      mbar_init(&S.xb_full[b], MODE == 1 ? 1 : WS_LOADERS);
      mbar_init(&S.xb_empty[b], 1);
      mbar_init(&S.tm_full[b], 1);
      mbar_init(&S.tm_empty[b], 32 * RW);
    }
    for (int r = 0; r < RAW; r++) mbar_init(&S.raw_full[r], 1);
    for (int r = 0; r < STG; r++) {
      mbar_init(&S.stg_full[r], 32 * RW);
      mbar_init(&S.stg_empty[r], 1);
    }
    S.abort = 0;
    mbar_fence_init();
  }
  if (warp == 4) {
    tmem_alloc(&S.tmem_slot, 512);
    tmem_relinquish();
  }
  __syncthreads();
  tc_fence_after();
  const u32 tmem = S.tmem_slot;

  if (MODE == 1 && warp < 4) {
    // ------------------------------------------------ operand rows by TMA (one thread)
    if (tid == 0) {
      mbar_expect_tx(&S.bar_tab, 2 * KT * kTileBytes);
      const uint8_t* src = tab + (size_t)grp * 2 * KT * kTileBytes;
      bulk_load(&S.tab_lo[0][0], src, KT * kTileBytes, &S.bar_tab);
      bulk_load(&S.tab_hi[0][0], src + (size_t)KT * kTileBytes, KT * kTileBytes, &S.bar_tab);
      for (int it = 0; it < niter; it++) {
        const int slot = it & 1;
        if (it >= 2 && !mbar_wait(&S.xb_empty[slot], ((it >> 1) - 1) & 1, err)) {
          S.abort = 1;
          break;
        }
        if (S.abort) break;
        const i64 tile = blockIdx.x + (i64)it * gridDim.x;
        const i64 i = tile / tpi, kb = tile - i * tpi;
        mbar_expect_tx(&S.xb_full[slot], KT * kTileBytes);
#pragma unroll
        for (int kt = 0; kt < KT; kt++)
          tma_load_2d(&S.xb[slot][kt][0], &map_in, &S.xb_full[slot], 128 * kt, (int)(i * Rp + k0 + kb * 128));
      }
    }
  } else if (warp < 4) {
    // ------------------------------------------------ loaders
    const int ent = tid;
    auto issue = [&](int it) {
      if (MODE == 2) {                           // one 3-D copy of the tile's L x 128 limb words
        if (tid == 0 && it < niter) {
          const i64 tile = blockIdx.x + (i64)it * gridDim.x;
          const i64 i = tile / tpi, kb = tile - i * tpi;
          mbar_expect_tx(&S.raw_full[it % RAW], (u32)L * WS_TILE * 4);
          tma_load_3d(&S.raw[it % RAW][0][0], &map_in, &S.raw_full[it % RAW], (int)(kb * WS_TILE), (int)i, 0);
        }
        return;
      }
      if (it < niter) {
        i64 tile = blockIdx.x + (i64)it * gridDim.x;
        if (vec) {
          // 16-byte copies: thread = (4-entry group ent & 31, limbs ent / 32 + 4 s); a group never straddles
          // an entry row (kp is a multiple of 16) and its words past kc are zero filled
          const int gi = ent & 31;
          const i64 e = tile * WS_TILE + 4 * gi;
          const i64 i = e / kp, k = e - i * kp;
          const bool ok = (e < nent) && (k < kc);
          const u32 nb = ok ? (u32)(4 * (kc - k < 4 ? kc - k : 4)) : 0u;
          const int32_t* base = X + (ok ? i * ld + k0 + k : 0);
          for (int l = ent >> 5; l < L; l += 4)
            cp_async16(&S.raw[it % RAW][l][4 * gi], base + (ok ? (i64)l * plane : 0), nb);
        } else {
          i64 e = tile * WS_TILE + ent;
          i64 i = e / kp, k = e - (e / kp) * kp;
          bool ok = (e < nent) && (k < kc);
          const int32_t* base = X + (ok ? i * ld + k0 + k : 0);
          u32* dst = &S.raw[it % RAW][0][ent];
          for (int l = 0; l < L; l++) cp_async4(dst + l * WS_TILE, base + (ok ? (i64)l * plane : 0), ok ? 4u : 0u);
        }
      }
      cp_async_commit();
    };
    if (tid == 0) {
      mbar_expect_tx(&S.bar_tab, 2 * KT * kTileBytes);
      const uint8_t* src = tab + (size_t)grp * 2 * KT * kTileBytes;
      bulk_load(&S.tab_lo[0][0], src, KT * kTileBytes, &S.bar_tab);
      bulk_load(&S.tab_hi[0][0], src + (size_t)KT * kTileBytes, KT * kTileBytes, &S.bar_tab);
    }
    for (int it = 0; it < RAW - 1; it++) issue(it);
    int it = 0;
    for (; it < niter; it++) {
      named_sync(1, WS_LOADERS);                 // everyone is done reading the raw stage refilled next
      issue(it + RAW - 1);
      bool fail = false;
      if (MODE == 2) fail = !mbar_wait(&S.raw_full[it % RAW], (it / RAW) & 1, err);
      else cp_async_wait<RAW - 1>();
      const int slot = it & 1;
      fail = fail || (it >= 2 && !mbar_wait(&S.xb_empty[slot], ((it >> 1) - 1) & 1, err));
      // tile it's words (from all loaders) have landed; the abort decision is uniform across loaders
      if (named_sync_or(1, WS_LOADERS, fail || S.abort)) {
        S.abort = 1;
        break;
      }
      const u32* raw = &S.raw[it % RAW][0][0];
      u32 w[4 * kMaxChunks];                         // all words first, then the stores (no load-store chain)
#pragma unroll
      for (int l = 0; l < 4 * kMaxChunks; l++) {
        if (l < L) w[l] = raw[l * WS_TILE + ent];                       // the limb's bytes, unsigned
        else if (l == L) w[l] = raw[(L - 1) * WS_TILE + ent] >> 31;     // sign byte (column 4L)
        else w[l] = 0u;
      }
#pragma unroll
      for (int c = 0; c < kMaxChunks; c++)
        *reinterpret_cast<uint4*>(&S.xb[slot][c >> 3][sw128_off(ent, c & 7)]) =
            make_uint4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
      fence_proxy_async_smem();
      mbar_arrive(&S.xb_full[slot]);
    }
    cp_async_wait<0>();
    if (MODE == 2 && tid == 0)                   // after an abort: let the copies in flight land (bounded)
      for (int j = it; j < niter && j < it + RAW; j++) mbar_wait(&S.raw_full[j % RAW], (j / RAW) & 1, err);
  } else if (warp == 4) {
    // ------------------------------------------------ MMA issuer
    if (lane == 0) {
      const u32 idesc = idesc_u8(128, WS_TILE);
      if (!mbar_wait(&S.bar_tab, 0, err)) S.abort = 1;
      int issued = 0;
      for (int it = 0; it < niter && !S.abort; it++) {
        const int b = it & 1;
        if (!mbar_wait(&S.xb_full[b], (it >> 1) & 1, err)) { S.abort = 1; break; }
        if (it >= 2 && !mbar_wait(&S.tm_empty[b], ((it >> 1) - 1) & 1, err)) { S.abort = 1; break; }
        tc_fence_after();
        const u32 d = tmem + (u32)b * 256;
#pragma unroll
        for (int kt = 0; kt < KT; kt++)
#pragma unroll
          for (int s = 0; s < 4; s++) {
            u64 bd = sdesc_sw128(smem_u32(&S.xb[b][kt][0]) + 32 * s);
            u32 accum = (kt | s) ? 1u : 0u;
            mma_i8(d, sdesc_sw128(smem_u32(&S.tab_lo[kt][0]) + 32 * s), bd, idesc, accum);
            mma_i8(d + WS_TILE, sdesc_sw128(smem_u32(&S.tab_hi[kt][0]) + 32 * s), bd, idesc, accum);
          }
        mma_commit(&S.xb_empty[b]);
        mma_commit(&S.tm_full[b]);
        issued = it + 1;
      }
      // on an abort, let the last committed products finish before TMEM is released (bounded)
      if (S.abort && issued > 0) mbar_wait(&S.tm_full[(issued - 1) & 1], ((issued - 1) >> 1) & 1, err);
    }
  } else if (warp == 5 + RW) {
    // ------------------------------------------------ bulk stores of the staged residue tiles (one lane), off the
    // reducers' path: staging sb is released once its store has read it
    if (lane == 0 && use_tma) {
      for (int it = 0; it < niter; it++) {
        const int sb = it % STG;
        if (!mbar_wait(&S.stg_full[sb], (it / STG) & 1, err)) {
          S.abort = 1;
          break;
        }
        const i64 tile = blockIdx.x + (i64)it * gridDim.x;
        // moduli rows beyond g0 + G and entries beyond nent (kp in the tiled modes) are clipped by the bounds
        const int y = grp * 128 - g0;
        if (TILED) {                                     // (k block, entry row i, moduli)
          const i64 i = tile / tpi, kb = tile - i * tpi;
          tma_store_3d(&map_hi, &S.out[sb][0][0], (int)(kb * WS_TILE), (int)i, y);
          tma_store_3d(&map_lo, &S.out[sb][1][0], (int)(kb * WS_TILE), (int)i, y);
        } else {
          tma_store_2d(&map_hi, &S.out[sb][0][0], (int)(tile * WS_TILE), y);
          tma_store_2d(&map_lo, &S.out[sb][1][0], (int)(tile * WS_TILE), y);
        }
        bulk_commit();
        bulk_wait_read<STG - 1>();                       // the store of tile it - (STG - 1) has read its staging
        if (it >= STG - 1) mbar_arrive(&S.stg_empty[(it - (STG - 1)) % STG]);
      }
      bulk_wait<0>();
    }
  } else {
    // ------------------------------------------------ reducers
    constexpr int CHUNKS = 16 / RW;                              // 32-column chunks per warp and tile
    const int quarter = warp & 3, part = (warp - 5) >> 2;
    const int row = quarter * 32 + lane;
    const int g = grp * 128 + row;
    const bool gvalid = (g >= g0) && (g < g0 + G) && (g < n);
    int m = 32639;                                       // rows past the moduli: any 15-bit modulus
    if (gvalid) m = mods[g];
    const int hm = m >> 1;
    const u32 bm = (u32)(((1ull << 46) + (u64)m - 1) / (u64)m);   // ceil(2^46 / m) < 2^32 (m > 2^14)
    int8_t* outh = Rhi + (i64)(g - g0) * pstride;
    int8_t* outl = Rlo + (i64)(g - g0) * pstride;
    for (int it = 0; it < niter; it++) {
      const int b = it & 1, sb = it % STG;
      bool fail = !mbar_wait(&S.tm_full[b], (it >> 1) & 1, err);
      // staging sb free: the store of tile it - STG has read it
      if (use_tma && it >= STG) fail = fail || !mbar_wait(&S.stg_empty[sb], ((it / STG) - 1) & 1, err);
      // uniform across the warp (warp-collective TMEM loads)
      if (__any_sync(0xffffffffu, fail || S.abort)) {
        S.abort = 1;
        break;
      }
      tc_fence_after();
      const i64 tile = blockIdx.x + (i64)it * gridDim.x;
#pragma unroll 1
      for (int c = 0; c < CHUNKS; c++) {
        const int col = part * (32 * CHUNKS) + c * 32;
        u32 lo[32], hi[32];
        const u32 taddr = tmem + ((u32)(quarter * 32) << 16) + (u32)b * 256 + col;
        tmem_ld32(taddr, lo);
        tmem_ld32(taddr + WS_TILE, hi);
        tmem_ld_wait();
        u32 ph[8], pl[8];
#pragma unroll
        for (int j = 0; j < 32; j += 4) {
          u32 r[4];
#pragma unroll
          for (int u = 0; u < 4; u++) {
            // v = 128 D_hi + D_lo: a sum of unsigned digit products, 0 <= v < 2^31, v = entry (mod m);
            // floor(v / m) = floor(v ceil(2^46 / m) / 2^46) exactly for v < 2^31, m < 2^15
            const u32 v = 128u * hi[j + u] + lo[j + u];
            const u32 q = __umulhi(v, bm) >> 14;
            r[u] = v - q * (u32)m;                                   // canonical residue in [0, m)
          }
          if (U8) {
            // pairs of 15-bit residues in 16-bit halves; hi = r >> 7 is byte 0 / 2 of (pair >> 7), lo byte 0 / 2
            // of the pair masked to 7 bits
            const u32 p01 = r[0] + (r[1] << 16), p23 = r[2] + (r[3] << 16);
            ph[j >> 2] = __byte_perm(p01 >> 7, p23 >> 7, 0x6420);
            pl[j >> 2] = __byte_perm(p01, p23, 0x6420) & 0x7F7F7F7Fu;
          } else {
            int hb[4], lb[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {                            // centred, split 128 hi + lo, lo in [-64, 64)
              const int c = (int)r[u] - (((int)r[u] > hm) ? m : 0);
              hb[u] = (c + 64) >> 7;
              lb[u] = c - (hb[u] << 7);
            }
            ph[j >> 2] = __byte_perm(__byte_perm(hb[0], hb[1], 0x0040), __byte_perm(hb[2], hb[3], 0x0040), 0x5410);
            pl[j >> 2] = __byte_perm(__byte_perm(lb[0], lb[1], 0x0040), __byte_perm(lb[2], lb[3], 0x0040), 0x5410);
          }
        }
        if (use_tma) {
          // row = modulus within the group, 16-byte chunks col/16 and col/16 + 1 (128-byte swizzle)
          uint8_t* oh = &S.out[sb][0][0];
          uint8_t* ol = &S.out[sb][1][0];
          *reinterpret_cast<uint4*>(oh + sw128_off(row, col >> 4)) = make_uint4(ph[0], ph[1], ph[2], ph[3]);
          *reinterpret_cast<uint4*>(oh + sw128_off(row, (col >> 4) + 1)) = make_uint4(ph[4], ph[5], ph[6], ph[7]);
          *reinterpret_cast<uint4*>(ol + sw128_off(row, col >> 4)) = make_uint4(pl[0], pl[1], pl[2], pl[3]);
          *reinterpret_cast<uint4*>(ol + sw128_off(row, (col >> 4) + 1)) = make_uint4(pl[4], pl[5], pl[6], pl[7]);
          continue;
        }
        if (!gvalid) continue;
        const i64 e0 = tile * WS_TILE + col;
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
      mbar_arrive(&S.tm_empty[b]);
      if (use_tma) {
        fence_proxy_async_smem();                          // staging writes visible to the bulk copy engine
        mbar_arrive(&S.stg_full[sb]);
      }
    }
  }
  __syncthreads();
  if (warp == 4) tmem_dealloc(tmem, 512);
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

template <int KT, int TILE, int THREADS, bool U8>
int launch_residues(const sdpv_ctx* c, const int32_t* X, i64 rows, i64 ld, i64 k0, i64 kc, i64 kp, int g0, int G,
                    int8_t* Rhi, int8_t* Rlo, i64 ps, cudaStream_t st) {
  const sdpv::CtxDev& d = c->d;
  size_t smem = sizeof(ResSmem<KT, TILE>) + 1024;
  int per_sm = 512 / (2 * TILE);                        // CTAs per SM allowed by TMEM ...
  int by_smem = (int)((228 * 1024) / (smem + 1024));    // ... and by shared memory
  if (by_smem < per_sm) per_sm = by_smem;
  if (per_sm < 1) return SDPV_EINVAL;
  size_t floor_smem = (228 * 1024) / (per_sm + 1) + 1024;   // keep a TMEM-starved extra CTA off the SM
  if (smem < floor_smem) smem = floor_smem;
  if (smem > 227 * 1024) return SDPV_EINVAL;
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(residues_kernel<KT, TILE, THREADS, U8>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return sdpv::set_cuda_error(e);
    attr_set[dev & 63] = true;
  }
  int grp0 = g0 / 128, grp1 = (g0 + G - 1) / 128;
  i64 ntiles = (rows * kp + TILE - 1) / TILE;
  i64 gx = per_sm * (i64)num_sms();
  if (gx > ntiles) gx = ntiles;
  dim3 grid((unsigned)gx, (unsigned)(grp1 - grp0 + 1));
  residues_kernel<KT, TILE, THREADS, U8><<<grid, THREADS, smem, st>>>(X, d.L, rows, ld, k0, kc, kp, g0, G, grp0, d.tab,
                                                                   d.mods, d.minv, d.n, Rhi, Rlo, ps,
                                                                   sdpv::device_error_word());
  return sdpv::launch_status();
}

// 2-D int8 map over one residue plane set: (nent entries, G moduli), plane stride ps, 128 x 128 boxes.
bool res_store_map(CUtensorMap* map, void* base, i64 nent, i64 G, i64 ps) {
  sdpv::EncodeTiledFn fn = sdpv::encode_tiled_fn();
  if (!fn) return false;
  cuuint64_t dims[2] = {(cuuint64_t)nent, (cuuint64_t)G};
  cuuint64_t strides[1] = {(cuuint64_t)ps};
  cuuint32_t box[2] = {128, 128};
  cuuint32_t estr[2] = {1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

// 3-D uint8 map over residue planes (kp entries, nI rows, G moduli), plane stride ps: 128 x 1 x 128 boxes.
bool res_store_map3(CUtensorMap* map, void* base, i64 kp, i64 nI, i64 G, i64 ps) {
  sdpv::EncodeTiledFn fn = sdpv::encode_tiled_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {(cuuint64_t)kp, (cuuint64_t)nI, (cuuint64_t)G};
  cuuint64_t strides[2] = {(cuuint64_t)kp, (cuuint64_t)ps};
  cuuint32_t box[3] = {128, 1, 128};
  cuuint32_t estr[3] = {1, 1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
         CUDA_SUCCESS;
}

template <int KT, int RAW, int STG, bool U8, int RW, int MODE>
bool ws_attr(size_t smem) {
  static bool attr_set[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63]) {
    if (cudaFuncSetAttribute(residues_ws_kernel<KT, RAW, STG, U8, RW, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
      return false;
    attr_set[dev & 63] = true;
  }
  return true;
}

template <int KT, int RAW, int STG, bool U8, int RW>
int launch_ws(const sdpv_ctx* c, const int32_t* X, i64 rows, i64 ld, i64 k0, i64 kc, i64 kp, int g0, int G,
              int8_t* Rhi, int8_t* Rlo, i64 ps, cudaStream_t st) {
  const sdpv::CtxDev& d = c->d;
  size_t smem = sizeof(WsSmem<KT, RAW, STG>) + 1024;
  if (smem > 227 * 1024) return SDPV_EINVAL;
  const i64 nent = rows * kp;
  int grp0 = g0 / 128, grp1 = (g0 + G - 1) / 128;
  i64 gx = num_sms();
  const bool out_ok = (g0 % 128 == 0) && ((((uintptr_t)Rhi) | ((uintptr_t)Rlo)) & 15) == 0;
  // TMA both ways (MODE 2) when the limb rows start 16-byte aligned, the residue planes allow bulk stores and
  // tiling per entry row leaves at most 1/8 of the tiles' entries idle (short rows keep the packed tiles)
  const i64 row_pad = (kp + WS_TILE - 1) / WS_TILE * WS_TILE - kp;
  if (out_ok && ld % 4 == 0 && k0 % 4 == 0 && ((((uintptr_t)X) & 15) == 0) && d.L <= 256 && rows < (1ll << 31) &&
      kc < (1ll << 31) && 8 * row_pad <= kp) {
    sdpv::EncodeTiledFn fn = sdpv::encode_tiled_fn();
    CUtensorMap mi, mh, ml;
    cuuint64_t dims[3] = {(cuuint64_t)kc, (cuuint64_t)rows, (cuuint64_t)d.L};
    cuuint64_t strides[2] = {(cuuint64_t)(ld * 4), (cuuint64_t)(rows * ld * 4)};
    cuuint32_t box[3] = {128, 1, (cuuint32_t)d.L};
    cuuint32_t estr[3] = {1, 1, 1};
    if (fn && fn(&mi, CU_TENSOR_MAP_DATA_TYPE_UINT32, 3, const_cast<int32_t*>(X + k0), dims, strides, box, estr,
                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                 CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
        res_store_map3(&mh, Rhi, kp, rows, G, ps) && res_store_map3(&ml, Rlo, kp, rows, G, ps)) {
      if (!ws_attr<KT, RAW, STG, U8, RW, 2>(smem)) return sdpv::set_cuda_error(cudaGetLastError());
      const i64 tpi = (kp + WS_TILE - 1) / WS_TILE, ntiles = rows * tpi;
      if (gx > ntiles) gx = ntiles;
      dim3 grid((unsigned)gx, (unsigned)(grp1 - grp0 + 1));
      residues_ws_kernel<KT, RAW, STG, U8, RW, 2><<<grid, ws_threads<RW>(), smem, st>>>(
          mh, ml, mi, 0, tpi, 1, 1, X, d.L, rows, ld, k0, kc, kp, g0, G, grp0, d.tabu, d.mods, d.minv, d.n, Rhi, Rlo,
          ps, sdpv::device_error_word());
      return sdpv::launch_status();
    }
  }
  if (!ws_attr<KT, RAW, STG, U8, RW, 0>(smem)) return sdpv::set_cuda_error(cudaGetLastError());
  // bulk tensor stores need 16-byte aligned planes and a box that starts at modulus row >= 0
  CUtensorMap mh, ml;
  int use_tma = out_ok && nent < (1ll << 31) && res_store_map(&mh, Rhi, nent, G, ps) &&
                res_store_map(&ml, Rlo, nent, G, ps);
  if (!use_tma) {
    memset(&mh, 0, sizeof(mh));
    memset(&ml, 0, sizeof(ml));
  }
  // 16-byte limb copies when every 4-entry group of a row starts 16-byte aligned
  const int vec = (ld % 4 == 0) && (k0 % 4 == 0) && ((((uintptr_t)X) & 15) == 0);
  i64 ntiles = (nent + WS_TILE - 1) / WS_TILE;
  if (gx > ntiles) gx = ntiles;
  dim3 grid((unsigned)gx, (unsigned)(grp1 - grp0 + 1));
  CUtensorMap unused;
  memset(&unused, 0, sizeof(unused));
  residues_ws_kernel<KT, RAW, STG, U8, RW, 0><<<grid, ws_threads<RW>(), smem, st>>>(
      mh, ml, unused, 0, 1, use_tma, vec, X, d.L, rows, ld, k0, kc, kp, g0, G, grp0, d.tabu, d.mods, d.minv, d.n, Rhi, Rlo, ps,
      sdpv::device_error_word());
  return sdpv::launch_status();
}

// Operand-row input (unsigned digits out): tiles (i, 128-entry block of k), TMA in and out.
template <int KT, int RW>
int launch_ws_rows(const sdpv_ctx* c, const uint8_t* rows_in, i64 nI, i64 Rp, i64 k0, i64 kc, i64 kp, int g0, int G,
                   uint8_t* Rhi, uint8_t* Rlo, i64 ps, cudaStream_t st) {
  constexpr int RAW = 1, STG = KT == 1 ? 2 : 1;
  const sdpv::CtxDev& d = c->d;
  size_t smem = sizeof(WsSmem<KT, RAW, STG>) + 1024;
  if (smem > 227 * 1024) return SDPV_EINVAL;
  if (!ws_attr<KT, RAW, STG, true, RW, 1>(smem)) return sdpv::set_cuda_error(cudaGetLastError());
  sdpv::EncodeTiledFn fn = sdpv::encode_tiled_fn();
  if (!fn) return SDPV_EINVAL;
  const i64 rb = 128 * KT;                                 // bytes per operand row
  CUtensorMap mi, mh, ml;
  {
    cuuint64_t dims[2] = {(cuuint64_t)rb, (cuuint64_t)(nI * Rp)};
    cuuint64_t strides[1] = {(cuuint64_t)rb};
    cuuint32_t box[2] = {128, 128};
    cuuint32_t estr[2] = {1, 1};
    if (fn(&mi, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(rows_in), dims, strides, box, estr,
           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return SDPV_EINVAL;
  }
  if (!res_store_map3(&mh, Rhi, kp, nI, G, ps) || !res_store_map3(&ml, Rlo, kp, nI, G, ps)) return SDPV_EINVAL;
  const i64 tpi = (kp + WS_TILE - 1) / WS_TILE;
  const i64 ntiles = nI * tpi;
  int grp0 = g0 / 128, grp1 = (g0 + G - 1) / 128;
  i64 gx = num_sms();
  if (gx > ntiles) gx = ntiles;
  dim3 grid((unsigned)gx, (unsigned)(grp1 - grp0 + 1));
  residues_ws_kernel<KT, RAW, STG, true, RW, 1><<<grid, ws_threads<RW>(), smem, st>>>(
      mh, ml, mi, Rp, tpi, 1, 0, nullptr, d.L, nI, 0, k0, kc, kp, g0, G, grp0, d.tabu, d.mods, d.minv, d.n,
      reinterpret_cast<int8_t*>(Rhi), reinterpret_cast<int8_t*>(Rlo), ps, sdpv::device_error_word());
  return sdpv::launch_status();
}

template <int KT, bool U8>
int launch_kt(const sdpv_ctx* c, const int32_t* X, i64 rows, i64 ld, i64 k0, i64 kc, i64 kp, int g0, int G,
              int8_t* Rhi, int8_t* Rlo, i64 ps, cudaStream_t st) {
  static int tile = [] {
    // tuning override: "ws" (warp-specialised, default for L <= 63), 64 or 128 (phase-serial CTAs)
    const char* v = getenv("SDPV_RES_TILE");
    if (v && atoi(v) == 128) return 128;
    if (v && atoi(v) == 64) return 64;
    return 0;
  }();
  const bool rw16 = sdpv::tune(SDPV_TUNE_RES_WARPS) == 16;
  if (tile == 0 && KT == 1)
    return rw16 ? launch_ws<1, 3, 2, U8, 16>(c, X, rows, ld, k0, kc, kp, g0, G, Rhi, Rlo, ps, st)
                : launch_ws<1, 3, 2, U8, 8>(c, X, rows, ld, k0, kc, kp, g0, G, Rhi, Rlo, ps, st);
  if (tile == 0 && KT == 2)
    return rw16 ? launch_ws<2, 2, 1, U8, 16>(c, X, rows, ld, k0, kc, kp, g0, G, Rhi, Rlo, ps, st)
                : launch_ws<2, 2, 1, U8, 8>(c, X, rows, ld, k0, kc, kp, g0, G, Rhi, Rlo, ps, st);
  if (tile == 128) return launch_residues<KT, 128, 256, U8>(c, X, rows, ld, k0, kc, kp, g0, G, Rhi, Rlo, ps, st);
  return launch_residues<KT, 64, 128, U8>(c, X, rows, ld, k0, kc, kp, g0, G, Rhi, Rlo, ps, st);
}

}  // namespace

template <bool U8>
int residues_entry(const sdpv_ctx* c, const int32_t* X, int64_t rows, int64_t ld, int64_t k0, int64_t kc, int g0, int G,
                   int8_t* Rhi, int8_t* Rlo, int64_t plane_stride, void* stream) {
  if (!c || rows < 0 || kc < 0 || k0 < 0 || k0 + kc > ld || g0 < 0 || G < 1 || g0 + G > c->d.n) return SDPV_EINVAL;
  i64 kp = (kc + 15) / 16 * 16;
  i64 ps = plane_stride ? plane_stride : rows * kp;
  if (ps < rows * kp || (ps & 15)) return SDPV_EINVAL;
  if (rows == 0 || kp == 0) return SDPV_OK;
  cudaStream_t st = sdpv::as_stream(stream);
  switch (c->d.kt) {
    case 1: return launch_kt<1, U8>(c, X, rows, ld, k0, kc, kp, g0, G, Rhi, Rlo, ps, st);
    case 2: return launch_kt<2, U8>(c, X, rows, ld, k0, kc, kp, g0, G, Rhi, Rlo, ps, st);
    case 3: return launch_kt<3, U8>(c, X, rows, ld, k0, kc, kp, g0, G, Rhi, Rlo, ps, st);
    default: return SDPV_EINVAL;                        // L > 94
  }
}

extern "C" int sdpv_residues(const sdpv_ctx* c, const int32_t* X, int64_t rows, int64_t ld, int64_t k0, int64_t kc,
                             int g0, int G, int8_t* Rhi, int8_t* Rlo, int64_t plane_stride, void* stream) {
  return residues_entry<false>(c, X, rows, ld, k0, kc, g0, G, Rhi, Rlo, plane_stride, stream);
}

extern "C" int sdpv_residues_u8(const sdpv_ctx* c, const int32_t* X, int64_t rows, int64_t ld, int64_t k0, int64_t kc,
                                int g0, int G, uint8_t* Rhi, uint8_t* Rlo, int64_t plane_stride, void* stream) {
  return residues_entry<true>(c, X, rows, ld, k0, kc, g0, G, reinterpret_cast<int8_t*>(Rhi),
                              reinterpret_cast<int8_t*>(Rlo), plane_stride, stream);
}

extern "C" int sdpv_residues_rows(const sdpv_ctx* c, const uint8_t* rows, int64_t nI, int64_t Rp, int64_t k0,
                                  int64_t kc, int g0, int G, uint8_t* Rhi, uint8_t* Rlo, int64_t plane_stride,
                                  void* stream) {
  if (!c || !rows || nI < 0 || kc < 0 || k0 < 0 || (k0 & 127) || Rp < 0 || (Rp & 127) || k0 + kc > Rp || g0 < 0 ||
      (g0 & 127) || G < 1 || g0 + G > c->d.n || (c->d.kt != 1 && c->d.kt != 2))
    return SDPV_EINVAL;
  const i64 kp = (kc + 15) / 16 * 16;
  const i64 ps = plane_stride ? plane_stride : nI * kp;
  if (ps < nI * kp || (ps & 15) || ((((uintptr_t)rows) | ((uintptr_t)Rhi) | ((uintptr_t)Rlo)) & 15) ||
      nI * Rp >= (1ll << 31) || nI >= (1ll << 31))
    return SDPV_EINVAL;
  if (nI == 0 || kc == 0) return SDPV_OK;
  cudaStream_t st = sdpv::as_stream(stream);
  const bool rw16 = sdpv::tune(SDPV_TUNE_RES_WARPS) == 16;
  if (c->d.kt == 1)
    return rw16 ? launch_ws_rows<1, 16>(c, rows, nI, Rp, k0, kc, kp, g0, G, Rhi, Rlo, ps, st)
                : launch_ws_rows<1, 8>(c, rows, nI, Rp, k0, kc, kp, g0, G, Rhi, Rlo, ps, st);
  return rw16 ? launch_ws_rows<2, 16>(c, rows, nI, Rp, k0, kc, kp, g0, G, Rhi, Rlo, ps, st)
              : launch_ws_rows<2, 8>(c, rows, nI, Rp, k0, kc, kp, g0, G, Rhi, Rlo, ps, st);
}
