// Residue GEMM on INT8 tensor cores (the exact products and the Gram accumulation).
//
// Per modulus m (and block b):  acc <- (acc + A B^T) mod m  with A = 128 Ahi + Alo, B = 128 Bhi + Blo,
// i.e. 2^14 Ahi Bhi^T + 2^7 (Ahi Blo^T + Alo Bhi^T) + Alo Blo^T  (sdpvibe/rns.py:106-137,
// sdpvibe/batched.py:96-162).
//
// Persistent: one CTA per SM loops over the work items (128 x 128 output tile, block, modulus); per item:
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
//     canonical residue back, 16 bytes at a time where the row stride allows.  As soon as an item's
//     accumulators are in registers the epilogue releases TMEM (mbarrier), so the next item's MMAs run
//     while it reduces and stores; the producer streams the next item's slices through the same ring.
// int32 accumulation is exact for K <= 65536 (|hh|, |hl + lh| <= K 2^14).
// Syrk mode (Gram): B = A, only lower-triangle tiles are scheduled and only entries i >= j written.  When
// the last row block has at most 32 rows (N = 274: 256 + 18), the diagonal items also multiply their row
// block by those tail rows (slot 2 of the ring, TMEM columns 384..479), so the row blocks are not read a
// second time for the tail; one small launch adds the tail rows against themselves.
#include <mutex>

#include "common.cuh"

namespace {

constexpr int kStages = 3;
constexpr u32 kSlice = 128 * 128;            // one operand slice: 128 rows x 128 bytes
constexpr int kThreads = 320;                // producer, MMA issuer, 8 epilogue warps
constexpr int kThreadsN = 576;               // narrow items of at most 32 short-side rows: 16 epilogue warps
constexpr int kCornerKB = 8;                // syrk corner: K blocks of [Thi; Tlo] (8 KB) per ring stage

constexpr int kSlots = 16;                  // compact narrow slots in the ring's memory (short K), at most
constexpr int kMaxG = 128;                  // moduli per launch (more are split over launches)
constexpr int kStg = 130;                   // staging row pitch (int16): 65 words, conflict-free by row

struct GemmSmem {
  uint8_t stage[kStages][4][kSlice];        // [ah, al, bh, bl], each 1024-aligned
  int16_t stg[128][kStg];                   // epilogue staging of one output tile (coalesced global I/O)
  u64 full[kSlots], empty[kSlots], acc_full, tmem_empty;
  u64 nacc_full[4], ntmem_empty[4];          // narrow items: a TMEM buffer per epilogue group (2 or 4)
  u32 tmem_slot;
  int abort;
  float tminv[kMaxG];                       // this launch's moduli, staged once per CTA
  int16_t tmod[kMaxG], tc14[kMaxG];
};

// Named barrier 1 over the 256 epilogue threads; the _or form returns the OR of pred over them.
__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }
__device__ __forceinline__ bool epi_sync_or(bool pred) {
  int r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.s32 p, %1, 0;\n\tbar.red.or.pred q, 1, 256, p;\n\tselp.s32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((int)pred)
      : "memory");
  return r != 0;
}

// Named barrier 2 + grp over one group of four epilogue warps (narrow items), with the OR of pred.
__device__ __forceinline__ bool grp_sync_or(int grp, bool pred) {
  int r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.s32 p, %1, 0;\n\tbar.red.or.pred q, %2, 128, p;\n\tselp.s32 %0, 1, 0, q;\n\t}"
      : "=r"(r)
      : "r"((int)pred), "r"(2 + grp)
      : "memory");
  return r != 0;
}

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

// Epilogue arithmetic of one thread's row (TMEM lane quarter q, column half ch): (hh mod m) 2^14 + (hx mod m)
// 2^7 + ll + old -> canonical residue, two per u32.  TMEM is released (tmem_empty) once both 32-column
// chunks are in registers.
__device__ __forceinline__ void epi_compute(u32 tmem, int q, int ch, int lane, int m, int c14, float minv,
                                            const u32 (&olds)[2][16], u32 (&outp)[2][16], u64* tmem_empty) {
#pragma unroll
  for (int c = 0; c < 2; c++) {
    u32 hh[32], hx[32], ll[32];
    u32 base = tmem + ((u32)(q * 32) << 16) + 64 * ch + 32 * c;
    tmem_ld32(base, hh);
    tmem_ld32(base + 128, hx);
    tmem_ld32(base + 256, ll);
    tmem_ld_wait();
    if (c == 1) {                                       // accumulators read: the next item's MMAs may start
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(tmem_empty);
    }
#pragma unroll
    for (int j2 = 0; j2 < 16; j2++) {
      u32 pair = 0;
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const int j = 2 * j2 + h;
        // (hh mod m) and (hx mod m) as |r| <= m/2 + m/300 representatives, then the canonical residue
        const int old = (int)(int16_t)(olds[c][j2] >> (16 * h));
        int a = (int)hh[j], x = (int)hx[j];
        int ra = a - (__float_as_int(fmaf((float)a, minv, 12582912.0f)) - 0x4B400000) * m;
        int rx = x - (__float_as_int(fmaf((float)x, minv, 12582912.0f)) - 0x4B400000) * m;
        int v = ra * c14 + rx * 128 + (int)ll[j] + old;
        int r = v - (__float_as_int(fmaf((float)v, minv, 12582912.0f)) - 0x4B400000) * m;
        r += (r < 0) ? m : 0;
        r -= (r >= m) ? m : 0;
        pair |= ((u32)r & 0xffffu) << (16 * h);
      }
      outp[c][j2] = pair;
    }
  }
}

// NW epilogue warps: 8 (every mode) or 16 (narrow items with TB <= 32 only: four epilogue groups, four TMEM
// buffers of 128 columns, so four items are reduced at once)
template <int NW>
__global__ void __launch_bounds__(64 + 32 * NW, 1)
    rns_gemm_kernel(const __grid_constant__ CUtensorMap mAh, const __grid_constant__ CUtensorMap mAl,
                    const __grid_constant__ CUtensorMap mBh, const __grid_constant__ CUtensorMap mBl,
                    const __grid_constant__ CUtensorMap mTh, const __grid_constant__ CUtensorMap mTl, int tailTB,
                    int nfull, int ftail, int tfirst, int nmode, int nTB, int u8ops, int nrb,
                    int16_t* __restrict__ acc, i64 ldc, const int32_t* __restrict__ mods, const float* __restrict__ minvs,
                    const int32_t* __restrict__ c14s, int g0, int gofs, int G, i64 nb, i64 M, i64 N, i64 KC, int mode, int ntn,
                    i64 tiles, i64 nitems, bool fresh, int pack, const int32_t* __restrict__ gtab,
                    unsigned* __restrict__ err) {
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  GemmSmem& S = *reinterpret_cast<GemmSmem*>((uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023));
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nk = (int)((KC + 127) / 128);
  constexpr int NT = 64 + 32 * NW;
  constexpr bool kNarrowOnly = NW == 16;
  constexpr int NGRP = NW / 4;                  // narrow epilogue groups = narrow TMEM buffers
  constexpr u32 kNBuf = kNarrowOnly ? 128 : 256; // TMEM columns per narrow buffer (3 TB <= 96 when TB <= 32)
  // compact narrow slots (16-warp narrow items whose K fits one row of nrb = 32 or 64 bytes): A hi, A lo and
  // [B hi; B lo] of one item with nrb-byte swizzled rows, NS of them in the ring's memory, one item each
  const bool compact = kNarrowOnly && nrb > 0;
  const u32 SB = compact ? (u32)(((256 + 2 * nTB) * nrb + 1023) & ~1023) : 0u;
  const u32 NS = compact ? min((u32)kSlots, (u32)(kStages * 4 * kSlice) / SB) : (u32)kStages;

  if (tid == 0) {
    for (int s = 0; s < kSlots; s++) {
      mbar_init(&S.full[s], 1);
      mbar_init(&S.empty[s], 1);
    }
    mbar_init(&S.acc_full, 1);
    mbar_init(&S.tmem_empty, 8);                // one arrival per epilogue warp
    for (int u = 0; u < NGRP; u++) {
      mbar_init(&S.nacc_full[u], 1);
      mbar_init(&S.ntmem_empty[u], 4);            // one arrival per warp of the item's epilogue group
    }
    S.abort = 0;
    mbar_fence_init();
  }
  if (warp == 1) {
    tmem_alloc(&S.tmem_slot, 512);
    tmem_relinquish();
  }
  for (int g = tid; g < G; g += NT) {                    // moduli < 2^15
    S.tmod[g] = (int16_t)mods[g0 + gofs + g];
    S.tc14[g] = (int16_t)c14s[g0 + gofs + g];
    S.tminv[g] = minvs[g0 + gofs + g];
  }
  __syncthreads();
  tc_fence_after();
  const u32 tmem = S.tmem_slot;

  // Work items (tile, block, modulus), round robin over the CTAs; item = (g * nb + b) * tiles + t.
  if (warp == 0) {
    if (lane == 0) {
      u32 kbg = 0;                              // k-blocks issued by this CTA so far (ring position)
      for (i64 item = blockIdx.x; item < nitems && !*(volatile int*)&S.abort; item += gridDim.x) {
        const i64 t = item % tiles, bg = item / tiles;
        int b, g, m0, n0;
        int nki = nk;                             // K blocks of this item
        if (tailTB || nmode) {                    // syrk tail / narrow: big-side row block t against TB rows
          b = (int)(bg % nb);
          g = gofs + (int)(bg / nb);
          m0 = (int)(t + tfirst) * 128;
          n0 = tailTB ? nfull : 0;
          if (gtab) {                             // grouped: the item's rows and K length from its table row
            const int32_t* it = gtab + 8 * t;
            m0 = it[0];
            n0 = it[2];
            nki = (it[4] + 127) / 128;
          }
        } else if (pack > 1) {                    // packed: tile t holds blocks t*pack .. (rows stacked)
          b = 0;
          g = gofs + (int)bg;
          m0 = (int)(t * pack * M);
          n0 = (int)(t * pack * N);
        } else {
          b = (int)(bg % nb);
          g = gofs + (int)(bg / nb);              // modulus plane of the operands
          int tm, tn;
          tile_of((int)t, mode, ntn, tm, tn);
          m0 = tm * 128;
          n0 = tn * 128;
        }
        const bool diag = mode == 1 && !tailTB && !nmode && pack <= 1 && m0 == n0;   // syrk diagonal: B = A
        if (tailTB) {
          // syrk corner (the tail rows against themselves): A = B = [Thi; Tlo], so one K block is the 2 TB
          // rows of [Thi; Tlo] (8 KB) and a ring stage holds kCornerKB of them
          for (int k8 = 0; k8 < nk; k8 += kCornerKB, kbg++) {
            const u32 s = kbg % kStages;
            if (kbg >= kStages && !mbar_wait(&S.empty[s], ((kbg / kStages) - 1) & 1, err)) {
              *(volatile int*)&S.abort = 1;
              break;
            }
            const int nkb = nk - k8 < kCornerKB ? nk - k8 : kCornerKB;
            mbar_expect_tx(&S.full[s], (u32)nkb * 2 * tailTB * 128);
            for (int j = 0; j < nkb; j++) {
              uint8_t* blk = &S.stage[s][0][0] + j * 2 * tailTB * 128;
              tma_load_4d(blk, &mTh, &S.full[s], (k8 + j) * 128, nfull, b, g);
              tma_load_4d(blk + tailTB * 128, &mTl, &S.full[s], (k8 + j) * 128, nfull, b, g);
            }
          }
          continue;
        }
        if (compact) {                            // one slot: the item's whole K in one row of nrb bytes
          const u32 s = kbg % NS;
          if (kbg >= NS && !mbar_wait(&S.empty[s], ((kbg / NS) - 1) & 1, err)) {
            *(volatile int*)&S.abort = 1;
            break;
          }
          uint8_t* sl = &S.stage[0][0][0] + s * SB;
          mbar_expect_tx(&S.full[s], (u32)((256 + 2 * nTB) * nrb));
          tma_load_4d(sl, &mAh, &S.full[s], 0, m0, b, g);
          tma_load_4d(sl + 128 * nrb, &mAl, &S.full[s], 0, m0, b, g);
          tma_load_4d(sl + 256 * nrb, &mTh, &S.full[s], 0, n0, b, g);
          tma_load_4d(sl + (256 + nTB) * nrb, &mTl, &S.full[s], 0, n0, b, g);
          kbg++;
          continue;
        }
        for (int kb = 0; kb < nki; kb++, kbg++) {
          const u32 s = kbg % kStages;
          if (kbg >= kStages && !mbar_wait(&S.empty[s], ((kbg / kStages) - 1) & 1, err)) {
            *(volatile int*)&S.abort = 1;
            break;
          }
          const int kx = kb * 128;
          if (tailTB || nmode) {                  // [Bhi; Blo] of the TB small-side rows back to back
            const int TB = tailTB ? tailTB : nTB;
            mbar_expect_tx(&S.full[s], 2 * kSlice + 2 * TB * 128);
            tma_load_4d(S.stage[s][0], &mAh, &S.full[s], kx, m0, b, g);
            tma_load_4d(S.stage[s][1], &mAl, &S.full[s], kx, m0, b, g);
            tma_load_4d(S.stage[s][2], &mTh, &S.full[s], kx, n0, b, g);
            tma_load_4d(S.stage[s][2] + TB * 128, &mTl, &S.full[s], kx, n0, b, g);
            continue;
          }
          mbar_expect_tx(&S.full[s], (diag ? 2 * kSlice + 2 * ftail * 128 : 4 * kSlice));
          tma_load_4d(S.stage[s][0], &mAh, &S.full[s], kx, m0, b, g);
          tma_load_4d(S.stage[s][1], &mAl, &S.full[s], kx, m0, b, g);
          if (diag) {                             // [Ahi; Alo] in slots 0, 1 serve as [Bhi; Blo]
            if (ftail) {                          // fused syrk tail: [Thi; Tlo] of the last rows in slot 2
              tma_load_4d(S.stage[s][2], &mTh, &S.full[s], kx, nfull, b, g);
              tma_load_4d(S.stage[s][2] + ftail * 128, &mTl, &S.full[s], kx, nfull, b, g);
            }
            continue;
          }
          tma_load_4d(S.stage[s][2], &mBh, &S.full[s], kx, n0, b, g);
          tma_load_4d(S.stage[s][3], &mBl, &S.full[s], kx, n0, b, g);
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0 && nmode) {
      // narrow items: as the tail items, N = 2 TB over [Bhi; Blo], in two TMEM buffers (256 columns apart)
      // so that an item's MMAs run while the epilogue still reads the previous item
      const int TB = nTB;
      const u32 idesc = u8ops ? idesc_u8(128, 2 * TB) : idesc_i8(128, 2 * TB);
      const u32 idescT = u8ops ? idesc_u8(128, TB) : idesc_i8(128, TB);
      u32 kbg = 0, li = 0;
      for (i64 item = blockIdx.x; item < nitems && !*(volatile int*)&S.abort; item += gridDim.x, li++) {
        const u32 buf = li % NGRP;
        if (li >= NGRP && !mbar_wait(&S.ntmem_empty[buf], ((li / NGRP) - 1) & 1, err)) {
          *(volatile int*)&S.abort = 1;
          break;
        }
        tc_fence_after();
        const u32 tb = tmem + buf * kNBuf;
        bool ok = true;
        int nki = nk;
        i64 klen = KC;
        if (gtab) {
          klen = gtab[8 * (item % tiles) + 4];
          nki = (int)((klen + 127) / 128);
        }
        if (compact) {
          const u32 s = kbg % NS;
          if (!mbar_wait(&S.full[s], (kbg / NS) & 1, err)) {
            *(volatile int*)&S.abort = 1;
            break;
          }
          tc_fence_after();
          const u32 sl = smem_u32(&S.stage[0][0][0]) + s * SB;
          const u32 bh = sl + 256 * nrb;
          const u64 dah = sdesc_sw(sl, nrb), dal = sdesc_sw(sl + 128 * nrb, nrb), dbh = sdesc_sw(bh, nrb);
          for (int ks = 0; ks < (int)((klen + 31) / 32); ks++) {       // klen <= nrb: K steps of 32 bytes
            const u64 bd = dbh + 2 * ks;
            if (ks == 0) {
              mma_i8(tb + 0, dah, bd, idesc, 0u);                                              // hh | hl
              mma_i8(tb + 2 * TB, dal, sdesc_sw(bh + TB * nrb, nrb), idescT, 0u);              // ll
              mma_i8(tb + TB, dal, bd, idescT, 1u);                                            // hl += lh
            } else {
              mma_i8(tb + 0, dah + 2 * ks, bd, idesc, 1u);
              mma_i8(tb + TB, dal + 2 * ks, bd, idesc, 1u);
            }
          }
          mma_commit(&S.empty[s]);
          mma_commit(&S.nacc_full[buf]);
          kbg++;
          continue;
        }
        for (int kb = 0; kb < nki; kb++, kbg++) {
          const u32 s = kbg % kStages;
          if (!mbar_wait(&S.full[s], (kbg / kStages) & 1, err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const u32 ah = smem_u32(S.stage[s][0]), al = smem_u32(S.stage[s][1]), bh = smem_u32(S.stage[s][2]);
          const u64 dah = sdesc_sw128(ah), dal = sdesc_sw128(al), dbh = sdesc_sw128(bh);
          auto step = [&](int ks) {
            const u64 bd = dbh + 2 * ks;
            if ((kb | ks) == 0) {
              mma_i8(tb + 0, dah, bd, idesc, 0u);                                              // hh | hl
              mma_i8(tb + 2 * TB, dal, sdesc_sw128(bh + TB * 128), idescT, 0u);                // ll
              mma_i8(tb + TB, dal, bd, idescT, 1u);                                            // hl += lh
            } else {
              mma_i8(tb + 0, dah + 2 * ks, bd, idesc, 1u);
              mma_i8(tb + TB, dal + 2 * ks, bd, idesc, 1u);
            }
          };
          const i64 krem = klen - kb * 128;                               // K steps past the item's K are zero
          if (krem >= 128) {
#pragma unroll
            for (int ks = 0; ks < 4; ks++) step(ks);
          } else {
            for (int ks = 0; ks < (int)((krem + 31) / 32); ks++) step(ks);
          }
          mma_commit(&S.empty[s]);
        }
        if (!ok) {
          *(volatile int*)&S.abort = 1;
          break;
        }
        mma_commit(&S.nacc_full[buf]);
      }
    } else if (lane == 0 && !kNarrowOnly) {
      // tail items: N = 2 TB over [Bhi; Blo] (hh | hl at column 0, (hl + lh) | ll at column TB)
      const int TB = tailTB ? tailTB : 128;
      const u32 idesc = u8ops ? idesc_u8(128, 2 * TB) : idesc_i8(128, 2 * TB);
      const u32 idesc128 = u8ops ? idesc_u8(128, TB) : idesc_i8(128, TB);
      const int FT = ftail ? ftail : 16;          // fused tail of the diagonal tiles: TMEM columns 384 ..
      const u32 idescF = u8ops ? idesc_u8(128, 2 * FT) : idesc_i8(128, 2 * FT);
      const u32 idescF1 = u8ops ? idesc_u8(128, FT) : idesc_i8(128, FT);
      u32 kbg = 0, li = 0;
      for (i64 item = blockIdx.x; item < nitems && !*(volatile int*)&S.abort; item += gridDim.x, li++) {
        bool diag = false;
        if (mode == 1 && !tailTB && pack <= 1) {
          int tm, tn;
          tile_of((int)(item % tiles), mode, ntn, tm, tn);
          diag = tm == tn;
        }
        // the epilogue must have read the previous item's accumulators out of TMEM
        if (li > 0 && !mbar_wait(&S.tmem_empty, (li - 1) & 1, err)) {
          *(volatile int*)&S.abort = 1;
          break;
        }
        tc_fence_after();
        bool ok = true;
        for (int k8 = 0; tailTB && k8 < nk; k8 += kCornerKB, kbg++) {
          // syrk corner: K block j of the stage at byte 8 KB j: A hi = Thi, A lo = Tlo (the M = 128 operand reads
          // on past the 32 loaded rows, into TMEM lanes whose entries the epilogue never stores; the reads stay
          // inside the shared-memory allocation), B = [Thi; Tlo]
          const u32 s = kbg % kStages;
          if (!mbar_wait(&S.full[s], (kbg / kStages) & 1, err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const int nkb = nk - k8 < kCornerKB ? nk - k8 : kCornerKB;
          for (int j = 0; j < nkb; j++) {
            const int kb = k8 + j;
            const u32 blk = smem_u32(&S.stage[s][0][0]) + j * 2 * TB * 128;
            const u64 dah = sdesc_sw128(blk), dal = sdesc_sw128(blk + TB * 128);
            auto cstep = [&](int ks) {
              const u64 bd = dah + 2 * ks;
              if ((kb | ks) == 0) {
                mma_i8(tmem + 0, dah, bd, idesc, 0u);                                            // hh | hl
                mma_i8(tmem + 2 * TB, dal, dal, idesc128, 0u);                                   // ll
                mma_i8(tmem + TB, dal, bd, idesc128, 1u);                                        // hl += lh
              } else {
                mma_i8(tmem + 0, dah + 2 * ks, bd, idesc, 1u);
                mma_i8(tmem + TB, dal + 2 * ks, bd, idesc, 1u);
              }
            };
            const i64 krem = KC - (i64)kb * 128;                          // K steps past KC are zero
            if (krem >= 128) {
#pragma unroll
              for (int ks = 0; ks < 4; ks++) cstep(ks);
            } else {
              for (int ks = 0; ks < (int)((krem + 31) / 32); ks++) cstep(ks);
            }
          }
          mma_commit(&S.empty[s]);
        }
        for (int kb = 0; !tailTB && kb < nk; kb++, kbg++) {
          const u32 s = kbg % kStages;
          if (!mbar_wait(&S.full[s], (kbg / kStages) & 1, err)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const u32 ah = smem_u32(S.stage[s][0]), al = smem_u32(S.stage[s][1]);
          const u32 bh = diag ? ah : smem_u32(S.stage[s][2]);
          // descriptors of K step ks: start address + 32 ks bytes = field + 2 ks (no carry out of the field)
          const u64 dah = sdesc_sw128(ah), dal = sdesc_sw128(al), dbh = sdesc_sw128(bh);
          const bool dt = diag && ftail;
          const u32 th = smem_u32(S.stage[s][2]);
          const u64 dth = sdesc_sw128(th);
          auto step = [&](int ks) {
            const u64 bd = dbh + 2 * ks;
            if ((kb | ks) == 0) {
              mma_i8(tmem + 0, dah, bd, idesc, 0u);                                              // hh | hl
              mma_i8(tmem + 2 * TB, dal, sdesc_sw128(bh + TB * 128), idesc128, 0u);              // ll
              mma_i8(tmem + TB, dal, bd, idesc128, 1u);                                          // hl += lh
            } else {
              mma_i8(tmem + 0, dah + 2 * ks, bd, idesc, 1u);
              mma_i8(tmem + TB, dal + 2 * ks, bd, idesc, 1u);
            }
            if (dt) {                             // A [Thi; Tlo]^T, N = 2 FT, at columns 384 ..
              const u64 td = dth + 2 * ks;
              if ((kb | ks) == 0) {
                mma_i8(tmem + 384, dah, td, idescF, 0u);
                mma_i8(tmem + 384 + 2 * FT, dal, sdesc_sw128(th + FT * 128), idescF1, 0u);
                mma_i8(tmem + 384 + FT, dal, td, idescF1, 1u);
              } else {
                mma_i8(tmem + 384, dah + 2 * ks, td, idescF, 1u);
                mma_i8(tmem + 384 + FT, dal + 2 * ks, td, idescF, 1u);
              }
            }
          };
          const i64 krem = KC - kb * 128;                                 // K steps past KC are zero
          if (krem >= 128) {
#pragma unroll
            for (int ks = 0; ks < 4; ks++) step(ks);
          } else {
            for (int ks = 0; ks < (int)((krem + 31) / 32); ks++) step(ks);
          }
          mma_commit(&S.empty[s]);
        }
        if (!ok) {
          *(volatile int*)&S.abort = 1;
          break;
        }
        mma_commit(&S.acc_full);
      }
    }
  } else {
    // Epilogue: warps 2..9 -> TMEM lane quarter (warp & 3), column half (warp - 2) / 4; one output row per
    // thread.  Rows whose stride allows 16-byte access (vec) are read and written directly, 16 bytes per
    // access; other strides go through the shared staging tile, one warp per row (coalesced).  With
    // `fresh` the accumulator is known to be zero: old residues are not read.
    const int q = warp & 3, ch = (warp - 2) >> 2, ew = warp - 2;
    const bool vec = ((ldc & 7) == 0) && ((((uintptr_t)acc) & 15) == 0);
    u32 li = 0;
    // narrow items: two epilogue groups of four warps (group ch takes this CTA's items li with li % 2 == ch, the
    // TMEM buffer of the same parity), so two items are reduced at once; each warp covers its lane quarter and
    // all TB columns, in two passes of TB / 2; the group's own named barrier (2 + ch) makes its decisions
    // uniform
    for (i64 item = blockIdx.x; item < nitems && nmode; item += gridDim.x, li++) {
      if ((int)(li % NGRP) != ch) continue;
      // narrow items: TMEM lane = big-side row r, columns = the TB small-side entries; nmode 1: C[r][j]
      // (A is the big side), nmode 2: C[j][r] (B is the big side; a warp's lanes are consecutive r, so each
      // output row's stores coalesce)
      const i64 t = item % tiles, bg = item / tiles;
      const int b = (int)(bg % nb), g = (int)(bg / nb);
      const int gg = g0 + gofs + g;
      const int m = S.tmod[g], c14 = S.tc14[g];
      const float minv = S.tminv[g];
      const u32 buf = li % NGRP;
      const int TB = nTB, half = nTB >> 1;
      i64 r = t * 128 + q * 32 + lane;
      i64 big = nmode == 1 ? M : N, small = nmode == 1 ? N : M;
      i64 rowA = (i64)gg * nb * M + (i64)b * M;                        // acc row of block row 0
      i64 col0 = 0;
      if (gtab) {
        // grouped: big-side rows r < it[1] of the item against small-side rows j < it[3]; nmode 1 stores
        // C[out_row0 + r][j], nmode 2 C[out_row0 + j][out_col0 + r] (acc planes of M rows per modulus)
        const int32_t* it = gtab + 8 * t;
        r = q * 32 + lane;
        big = it[1];
        small = it[3];
        rowA = (i64)gg * M + it[5];
        col0 = it[6];
      }
      int16_t* bp = nmode == 1 ? acc + (rowA + r) * ldc : acc + rowA * ldc + col0 + r;
      const i64 js = nmode == 1 ? 1 : ldc;
      const bool ok_me = mbar_wait(&S.nacc_full[buf], (li / NGRP) & 1, err);
      const bool fail = grp_sync_or(ch, !ok_me);
      if (fail) break;
      tc_fence_after();
      // grouped items with K <= 64 on unsigned digits: hx < 2 K 255 127 < 2^22, so 128 hx needs no reduction
      // of its own (the sum below stays under 2^30 with an old residue < 2^15)
      const bool small_k = u8ops && (gtab ? gtab[8 * t + 4] <= 64 : KC <= 64);
      const bool fast = gtab && nmode == 1 && half == 16 && fresh && small_k;
      for (int pass = 0; pass < 2; pass++) {
        const int j0 = pass * half;
        const bool skip = gtab && (q * 32 >= big || j0 >= small);    // warp-uniform: no valid output here
        u32 hh[32], hx[32], ll[32];
        if (!skip) {
          const u32 base = tmem + buf * kNBuf + ((u32)(q * 32) << 16) + j0;
          if (kNarrowOnly || half <= 16) {               // TB <= 32: a 16-column load suffices
            tmem_ld16(base, *reinterpret_cast<u32(*)[16]>(hh));
            tmem_ld16(base + TB, *reinterpret_cast<u32(*)[16]>(hx));
            tmem_ld16(base + 2 * TB, *reinterpret_cast<u32(*)[16]>(ll));
          } else {
            tmem_ld32(base, hh);
            tmem_ld32(base + TB, hx);
            tmem_ld32(base + 2 * TB, ll);
          }
          tmem_ld_wait();
        }
        if (pass == 1) {                                 // both passes' accumulators read: release the buffer
          tc_fence_before();
          __syncwarp();
          if (lane == 0) mbar_arrive(&S.ntmem_empty[buf]);
        }
        if (skip) continue;
        if (fast) {
          // grouped items of 32 small-side rows and K <= 64 on unsigned digits: ll < K 127^2 < 2^20 and
          // hx = hl + lh < 2 K 255 127 < 2^22, so (hh mod m) 2^14 + 128 hx + ll stays below 2^30 and needs one
          // reduction after hh's; the thread's 16 results of this pass leave as two 16-byte stores
          u32 pk[8];
#pragma unroll
          for (int u = 0; u < 16; u++) {
            const int a = (int)hh[u];
            const int ra = a - (__float_as_int(fmaf((float)a, minv, 12582912.0f)) - 0x4B400000) * m;
            const int v = ra * c14 + (int)hx[u] * 128 + (int)ll[u];
            int rr = v - (__float_as_int(fmaf((float)v, minv, 12582912.0f)) - 0x4B400000) * m;
            rr += (rr < 0) ? m : 0;                      // the rounded quotient: one correction (see below)
            if (u & 1)
              pk[u >> 1] |= ((u32)rr & 0xffffu) << 16;
            else
              pk[u >> 1] = (u32)rr & 0xffffu;
          }
          if (r < big) {
            if (j0 + 16 <= small && (ldc & 7) == 0 && (((uintptr_t)acc) & 15) == 0) {
              uint4* dst = reinterpret_cast<uint4*>(bp + j0);
              dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
              dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
            } else {
              for (int u = 0; u < 16; u++)
                if (j0 + u < small) bp[j0 + u] = (int16_t)(pk[u >> 1] >> (16 * (u & 1)));
            }
          }
          continue;
        }
        // this pass's outputs of this thread: u < nval (the row test and the column bound taken once)
        const int nval = r < big ? (int)(small - j0 < half ? (small - j0 > 0 ? small - j0 : 0) : half) : 0;
        // x - (round(x / m) as the float magic number's bits - 0x4B400000) m, with 0x4B400000 m folded into one
        // constant (arithmetic mod 2^32; the true value is below m in magnitude)
        const u32 mu = (u32)m, k0 = 0x4B400000u * mu;
        auto red = [&](int x) -> int {
          return (int)((u32)x + k0 - (u32)__float_as_int(fmaf((float)x, minv, 12582912.0f)) * mu);
        };
        // v - q m with q = v / m rounded to nearest within 1/64 (|v| < 2^31, float rounding of v and of 1/m)
        // lies in (-0.52 m, 0.52 m): one correction gives the canonical residue
        int16_t* q = bp + (i64)j0 * js;
        if (fresh) {
#pragma unroll
          for (int u = 0; u < (kNarrowOnly ? 16 : 32); u++, q += js) {
            if (u >= half) break;
            const int rx = small_k ? (int)hx[u] : red((int)hx[u]);
            int rr = red(red((int)hh[u]) * c14 + rx * 128 + (int)ll[u]);
            rr += (rr < 0) ? m : 0;
            if (u < nval) *q = (int16_t)rr;
          }
        } else {
#pragma unroll
          for (int u = 0; u < (kNarrowOnly ? 16 : 32); u++, q += js) {
            if (u >= half) break;
            const bool in = u < nval;
            const int o = in ? (int)*q : 0;                         // old residue (K chunks)
            const int rx = small_k ? (int)hx[u] : red((int)hx[u]);
            int rr = red(red((int)hh[u]) * c14 + rx * 128 + (int)ll[u] + o);
            rr += (rr < 0) ? m : 0;
            if (in) *q = (int16_t)rr;
          }
        }
      }
    }
    for (i64 item = blockIdx.x; item < nitems && !kNarrowOnly && tailTB; item += gridDim.x, li++) {
      // syrk tail: entry (A row i, tail row j) = Q[nfull + j][i], written transposed into the lower triangle;
      // a warp's lanes are consecutive i, so the accesses of one tail row coalesce
      const i64 t = item % tiles, bg = item / tiles;
      const int b = (int)(bg % nb), g = (int)(bg / nb);
      const int gg = g0 + gofs + g;
      const int m = S.tmod[g], c14 = S.tc14[g];
      const float minv = S.tminv[g];
      const i64 i = (t + tfirst) * 128 + q * 32 + lane;             // A row (output column)
      const int tail = (int)(N - nfull);
      int16_t* colp = acc + ((i64)gg * nb * M + (i64)b * M + nfull) * ldc + i;
      int old[16];
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int j = 16 * ch + u;
        old[u] = (i < M && j < tail && nfull + j >= i && !fresh) ? (int)colp[(i64)j * ldc] : 0;
      }
      const bool ok_me = mbar_wait(&S.acc_full, li & 1, err);
      const bool fail = epi_sync_or(!ok_me);
      if (fail) break;
      tc_fence_after();
      u32 hh[32], hx[32], ll[32];
      const u32 base = tmem + ((u32)(q * 32) << 16);
      tmem_ld32(base, hh);
      tmem_ld32(base + tailTB, hx);
      tmem_ld32(base + 2 * tailTB, ll);
      tmem_ld_wait();
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&S.tmem_empty);
#pragma unroll
      for (int u = 0; u < 16; u++) {
        const int j = 16 * ch + u;
        int a = (int)hh[j], x = (int)hx[j];
        int ra = a - (__float_as_int(fmaf((float)a, minv, 12582912.0f)) - 0x4B400000) * m;
        int rx = x - (__float_as_int(fmaf((float)x, minv, 12582912.0f)) - 0x4B400000) * m;
        int v = ra * c14 + rx * 128 + (int)ll[j] + old[u];
        int r = v - (__float_as_int(fmaf((float)v, minv, 12582912.0f)) - 0x4B400000) * m;
        r += (r < 0) ? m : 0;
        r -= (r >= m) ? m : 0;
        if (i < M && j < tail && nfull + j >= i) colp[(i64)j * ldc] = (int16_t)r;
      }
    }
    for (i64 item = blockIdx.x; item < nitems && !kNarrowOnly && pack > 1 && !nmode; item += gridDim.x, li++) {
      // packed small blocks: tile rows are the stacked rows of blocks t*pack .. t*pack + nbt - 1, tile
      // columns their stacked B rows; only the diagonal sub-blocks are outputs (staged, coalesced)
      const i64 t = item % tiles;
      const int g = (int)(item / tiles);
      const int gg = g0 + gofs + g;
      const int m = S.tmod[g], c14 = S.tc14[g];
      const float minv = S.tminv[g];
      const i64 b0 = t * pack;
      const int nbt = (int)(nb - b0 < pack ? nb - b0 : pack);
      const int nrow = nbt * (int)M;
      const i64 rowbase = (i64)gg * nb * M + b0 * M;               // acc row of tile row 0
      const int rrow = q * 32 + lane;
      u32 olds[2][16];
#pragma unroll
      for (int c = 0; c < 2; c++)
#pragma unroll
        for (int j = 0; j < 16; j++) olds[c][j] = 0;
      if (!fresh) {
        epi_sync();
        for (int r = ew; r < nrow; r += 8) {
          const int bi = r / (int)M;
          const int16_t* src = acc + (rowbase + r) * ldc;
          for (int j = lane; j < N; j += 32) S.stg[r][bi * N + j] = src[j];
        }
        epi_sync();
#pragma unroll
        for (int c = 0; c < 2; c++)
#pragma unroll
          for (int j = 0; j < 16; j++)
            olds[c][j] = *reinterpret_cast<const u32*>(&S.stg[rrow][64 * ch + 32 * c + 2 * j]);
      }
      const bool ok_me = mbar_wait(&S.acc_full, li & 1, err);
      const bool fail = epi_sync_or(!ok_me);
      if (fail) break;
      tc_fence_after();
      u32 outp[2][16];
      epi_compute(tmem, q, ch, lane, m, c14, minv, olds, outp, &S.tmem_empty);
      epi_sync();
#pragma unroll
      for (int c = 0; c < 2; c++)
#pragma unroll
        for (int j2 = 0; j2 < 16; j2++)
          *reinterpret_cast<u32*>(&S.stg[rrow][64 * ch + 32 * c + 2 * j2]) = outp[c][j2];
      epi_sync();
      for (int r = ew; r < nrow; r += 8) {
        const int bi = r / (int)M;
        int16_t* dst = acc + (rowbase + r) * ldc;
        for (int j = lane; j < N; j += 32) dst[j] = S.stg[r][bi * N + j];
      }
    }
    for (i64 item = blockIdx.x; item < nitems && !kNarrowOnly && pack <= 1 && !tailTB && !nmode; item += gridDim.x, li++) {
      const i64 t = item % tiles, bg = item / tiles;
      const int b = (int)(bg % nb), g = (int)(bg / nb);
      int tm, tn;
      tile_of((int)t, mode, ntn, tm, tn);
      const int m0 = tm * 128, n0 = tn * 128;
      const int gg = g0 + gofs + g;
      const int m = S.tmod[g], c14 = S.tc14[g];
      const float minv = S.tminv[g];
      const i64 rowbase = (i64)gg * nb * M + (i64)b * M + m0;       // acc row of tile row 0
      const int nrow = (int)(M - m0 < 128 ? M - m0 : 128), ncol = (int)(N - n0 < 128 ? N - n0 : 128);
      const int rrow = q * 32 + lane;
      const i64 i = m0 + rrow;                                      // output row within the block
      int16_t* rowp = acc + (rowbase + rrow) * ldc;
      // fused syrk tail of a diagonal tile: entry (A row i, tail row j) = Q[nfull + j][i], stored transposed
      // (a warp's lanes are consecutive i: coalesced); this thread takes tail rows 16 ch .. 16 ch + 15
      const bool dt = ftail && tm == tn;
      const int tail = (int)(N - nfull);
      int16_t* colp = acc + ((i64)gg * nb * M + (i64)b * M + nfull) * ldc + i;
      int told[16];
#pragma unroll
      for (int u = 0; u < 16; u++) told[u] = (dt && !fresh && 16 * ch + u < tail) ? (int)colp[(i64)(16 * ch + u) * ldc] : 0;
      u32 olds[2][16];                                              // old residues of this row, in pairs
#pragma unroll
      for (int c = 0; c < 2; c++)
#pragma unroll
        for (int j = 0; j < 16; j++) olds[c][j] = 0;
      if (!fresh) {
        if (vec) {
#pragma unroll
          for (int c = 0; c < 2; c++) {
            const int nc = n0 + 64 * ch + 32 * c;
            const bool full = rrow < nrow && nc + 32 <= N && (mode == 0 || nc + 31 <= i);
            if (full) {
#pragma unroll
              for (int v4 = 0; v4 < 4; v4++) {
                const uint4 x = reinterpret_cast<const uint4*>(rowp + nc)[v4];
                olds[c][4 * v4] = x.x;
                olds[c][4 * v4 + 1] = x.y;
                olds[c][4 * v4 + 2] = x.z;
                olds[c][4 * v4 + 3] = x.w;
              }
            } else if (rrow < nrow) {
              for (int j = 0; j < 32; j++)
                if (nc + j < N && (mode == 0 || nc + j <= i))
                  olds[c][j >> 1] |= ((u32)(uint16_t)rowp[nc + j]) << (16 * (j & 1));
            }
          }
        } else {
          epi_sync();                                    // the previous tile has left the staging area
          for (int r0 = ew; r0 < nrow; r0 += 32) {       // 4 rows x 4 column groups of loads in flight
            int16_t v[4][4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
              const int r = r0 + 8 * u;
              const int jmax = r >= nrow ? 0 : (mode == 0 ? ncol : min(ncol, m0 + r - n0 + 1));
              const int16_t* src = acc + (rowbase + r) * ldc + n0;
#pragma unroll
              for (int w = 0; w < 4; w++) v[u][w] = (lane + 32 * w < jmax) ? src[lane + 32 * w] : (int16_t)0;
            }
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
              for (int w = 0; w < 4; w++)
                if (r0 + 8 * u < nrow) S.stg[r0 + 8 * u][lane + 32 * w] = v[u][w];
          }
          epi_sync();
#pragma unroll
          for (int c = 0; c < 2; c++)
#pragma unroll
            for (int j = 0; j < 16; j++)
              olds[c][j] = *reinterpret_cast<const u32*>(&S.stg[rrow][64 * ch + 32 * c + 2 * j]);
        }
      }
      const bool ok_me = mbar_wait(&S.acc_full, li & 1, err);
      const bool fail = epi_sync_or(!ok_me);             // uniform over the epilogue warps
      if (fail) break;
      tc_fence_after();
      if (dt) {                                          // read before epi_compute releases TMEM
        u32 hh[16], hx[16], ll[16];
        const u32 base = tmem + ((u32)(q * 32) << 16) + 384 + 16 * ch;
        tmem_ld16(base, hh);
        tmem_ld16(base + ftail, hx);
        tmem_ld16(base + 2 * ftail, ll);
        tmem_ld_wait();
#pragma unroll
        for (int u = 0; u < 16; u++) {
          const int j = 16 * ch + u;
          int a = (int)hh[u], x = (int)hx[u];
          int ra = a - (__float_as_int(fmaf((float)a, minv, 12582912.0f)) - 0x4B400000) * m;
          int rx = x - (__float_as_int(fmaf((float)x, minv, 12582912.0f)) - 0x4B400000) * m;
          int v = ra * c14 + rx * 128 + (int)ll[u] + told[u];
          int r = v - (__float_as_int(fmaf((float)v, minv, 12582912.0f)) - 0x4B400000) * m;
          r += (r < 0) ? m : 0;
          r -= (r >= m) ? m : 0;
          if (j < tail) colp[(i64)j * ldc] = (int16_t)r;
        }
      }
      u32 outp[2][16];
      epi_compute(tmem, q, ch, lane, m, c14, minv, olds, outp, &S.tmem_empty);
      if (vec) {
        if (rrow < nrow) {
#pragma unroll
          for (int c = 0; c < 2; c++) {
            const int nc = n0 + 64 * ch + 32 * c;
            if (nc >= N) continue;
            const bool full = nc + 32 <= N && (mode == 0 || nc + 31 <= i);
            if (full) {
#pragma unroll
              for (int v4 = 0; v4 < 4; v4++)
                reinterpret_cast<uint4*>(rowp + nc)[v4] =
                    make_uint4(outp[c][4 * v4], outp[c][4 * v4 + 1], outp[c][4 * v4 + 2], outp[c][4 * v4 + 3]);
            } else {
              for (int j = 0; j < 32; j++)
                if (nc + j < N && (mode == 0 || nc + j <= i)) rowp[nc + j] = (int16_t)(outp[c][j >> 1] >> (16 * (j & 1)));
            }
          }
        }
      } else {
        epi_sync();                                      // (fresh: the previous tile's stores are done)
#pragma unroll
        for (int c = 0; c < 2; c++)
#pragma unroll
          for (int j2 = 0; j2 < 16; j2++)
            *reinterpret_cast<u32*>(&S.stg[rrow][64 * ch + 32 * c + 2 * j2]) = outp[c][j2];
        epi_sync();
        for (int r = ew; r < nrow; r += 8) {
          int16_t* dst = acc + (rowbase + r) * ldc + n0;
          const int jmax = mode == 0 ? ncol : min(ncol, m0 + r - n0 + 1);
          for (int j = lane; j < jmax; j += 32) dst[j] = S.stg[r][j];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) tmem_dealloc(tmem, 512);
}

// 4-D int8 map over (K, rows, nb, G) with 128 x 128 boxes and 128-byte swizzle; gstride = bytes between
// the planes of consecutive moduli (>= K*rows*nb).
// box_x: row bytes of the box (128, or 32 / 64 for compact narrow slots), swizzled by the same width
bool make_map(CUtensorMap* map, const void* base, i64 K, i64 rows, i64 nb, i64 G, i64 gstride, int box_rows = 128,
              int box_x = 128) {
  sdpv::EncodeTiledFn fn = sdpv::encode_tiled_fn();
  if (!fn) return false;
  cuuint64_t dims[4] = {(cuuint64_t)K, (cuuint64_t)rows, (cuuint64_t)nb, (cuuint64_t)G};
  cuuint64_t strides[3] = {(cuuint64_t)K, (cuuint64_t)(K * rows), (cuuint64_t)gstride};
  cuuint32_t box[4] = {(cuuint32_t)box_x, (cuuint32_t)box_rows, 1, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUtensorMapSwizzle sw = box_x == 32   ? CU_TENSOR_MAP_SWIZZLE_32B
                                : box_x == 64 ? CU_TENSOR_MAP_SWIZZLE_64B
                                              : CU_TENSOR_MAP_SWIZZLE_128B;
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<void*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, sw, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

// A non-blocking side stream and two timing-free events per device (created once), for launches that may
// run beside the caller's stream; joined back with an event before the entry point returns.
int side_stream(int dev, cudaStream_t* s, cudaEvent_t* fork_ev, cudaEvent_t* join_ev) {
  static std::mutex mu;
  static cudaStream_t streams[64] = {};
  static cudaEvent_t evs[64][2] = {};
  if (dev < 0 || dev >= 64) return SDPV_EINVAL;
  std::lock_guard<std::mutex> g(mu);
  if (!streams[dev]) {
    cudaError_t e = cudaStreamCreateWithFlags(&streams[dev], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&evs[dev][0], cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&evs[dev][1], cudaEventDisableTiming);
    if (e != cudaSuccess) {
      streams[dev] = nullptr;
      return sdpv::set_cuda_error(e);
    }
  }
  *s = streams[dev];
  *fork_ev = evs[dev][0];
  *join_ev = evs[dev][1];
  return SDPV_OK;
}

// Dynamic shared memory of both kernel instantiations, set once per process.
int gemm_attr(size_t smem) {
  static std::once_flag attr;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(attr, [&] {
    attr_err = cudaFuncSetAttribute(rns_gemm_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (attr_err == cudaSuccess)
      attr_err = cudaFuncSetAttribute(rns_gemm_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  });
  return attr_err == cudaSuccess ? SDPV_OK : sdpv::set_cuda_error(attr_err);
}

}  // namespace

extern "C" int sdpv_rns_gemm(const sdpv_ctx* c, const int8_t* Ahi, const int8_t* Alo, const int8_t* Bhi,
                             const int8_t* Blo, int64_t a_stride, int64_t b_stride, int16_t* acc, int64_t ldc, int g0,
                             int G, int64_t nb, int64_t M, int64_t N, int64_t KC, int mode, void* stream) {
  if (!c || g0 < 0 || G < 1 || g0 + G > c->d.n || nb < 1 || M < 0 || N < 0 || KC < 0 || KC > 65536 ||
      (KC & 15) || (mode & ~7) || nb > 65535 || G > 65535)
    return SDPV_EINVAL;
  const bool fresh = (mode & 2) != 0;                  // accumulator known to be zero: overwrite
  const int u8ops = (mode & 4) ? 1 : 0;                // unsigned digits: int32 sums exact for K <= 32768
  if (u8ops && KC > 32768) return SDPV_EINVAL;
  mode &= 1;
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
  // Small blocks (M, N <= 64, not syrk) are packed: pack blocks share one 128 x 128 tile (their stacked rows
  // against their stacked B rows; only the diagonal sub-blocks are kept), so fewer, fuller tiles run.
  int pack = 1;
  const int pack_max = sdpv::tune(SDPV_TUNE_PACK_MAX), narrow_max = sdpv::tune(SDPV_TUNE_NARROW_MAX);
  if (mode == 0 && nb > 1 && M <= pack_max && N <= pack_max) {
    i64 p = 128 / M < 128 / N ? 128 / M : 128 / N;
    pack = (int)(p < nb ? p : nb);
  }
  // One side at most 64 rows, the other longer (not syrk, not packed): narrow items.  The long side fills the
  // 128 MMA rows, the short side's TB rows (rounded up to 16) are the MMA's N = 2 TB as [hi; lo]; nmode 1:
  // A is the long side, 2: B is (C stored transposed from the tile).
  int nmode = 0, nTB = 0;
  if (mode == 0 && pack <= 1) {
    if (N <= narrow_max && M > narrow_max) nmode = 1;
    else if (M <= narrow_max && N > narrow_max) nmode = 2;
    if (nmode) nTB = (int)(((nmode == 1 ? N : M) + 15) / 16 * 16);
  }
  CUtensorMap mAh, mAl, mBh, mBl;
  const i64 ra = pack > 1 ? M * nb : M, rb = pack > 1 ? N * nb : N, nbm = pack > 1 ? 1 : nb;
  // 16-warp narrow items whose K fits a row of 32 or 64 bytes load into compact slots (many items in flight)
  const int nrb = (nmode && nTB <= 32 && KC <= 64) ? (KC <= 32 ? 32 : 64) : 0, bx = nrb ? nrb : 128;
  if (nmode == 2) {                                    // big side B into the A slots, A as the TB rows
    if (!make_map(&mAh, Bhi, KC, rb, nbm, G, b_stride, 128, bx) || !make_map(&mAl, Blo, KC, rb, nbm, G, b_stride, 128, bx) ||
        !make_map(&mBh, Ahi, KC, ra, nbm, G, a_stride, nTB, bx) || !make_map(&mBl, Alo, KC, ra, nbm, G, a_stride, nTB, bx))
      return SDPV_EINVAL;
  } else if (nmode == 1) {
    if (!make_map(&mAh, Ahi, KC, ra, nbm, G, a_stride, 128, bx) || !make_map(&mAl, Alo, KC, ra, nbm, G, a_stride, 128, bx) ||
        !make_map(&mBh, Bhi, KC, rb, nbm, G, b_stride, nTB, bx) || !make_map(&mBl, Blo, KC, rb, nbm, G, b_stride, nTB, bx))
      return SDPV_EINVAL;
  } else if (!make_map(&mAh, Ahi, KC, ra, nbm, G, a_stride) || !make_map(&mAl, Alo, KC, ra, nbm, G, a_stride) ||
             !make_map(&mBh, Bhi, KC, rb, nbm, G, b_stride) || !make_map(&mBl, Blo, KC, rb, nbm, G, b_stride)) {
    return SDPV_EINVAL;
  }
  const size_t smem = sizeof(GemmSmem) + 1024;
  const int attr_st = gemm_attr(smem);
  if (attr_st != SDPV_OK) return attr_st;
  int ntm = (int)((M + 127) / 128), ntn = (int)((N + 127) / 128);
  // syrk whose last row block has at most 32 rows: full lower tiles over the first nfull rows, the tail rows
  // against each full row block inside that row block's diagonal item (its operand slices are in shared
  // memory already; N = 64 products at TMEM columns 384.., stored transposed), and the tail rows against
  // themselves in one more small launch -- not 128 x 128 tiles that are mostly padding
  const int nfull = (int)(N / 128) * 128, tailTB = (mode == 1 && N > 128 && N - nfull > 0 && N - nfull <= 32) ? 32 : 0;
  if (tailTB) ntm = nfull / 128;
  i64 tiles = mode == 0 ? (i64)ntm * ntn : (i64)ntm * (ntm + 1) / 2;
  if (pack > 1) tiles = (nb + pack - 1) / pack;
  if (nmode) tiles = ((nmode == 1 ? M : N) + 127) / 128;
  CUtensorMap mTh = mBh, mTl = mBl;
  if (tailTB && (!make_map(&mTh, Bhi, KC, rb, nbm, G, b_stride, tailTB) ||
                 !make_map(&mTl, Blo, KC, rb, nbm, G, b_stride, tailTB)))
    return SDPV_EINVAL;
  if (tiles > 0x7fffffff) return SDPV_EINVAL;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // The corner launch of a fused-tail syrk runs on a side stream beside the full-tile launch (they write
  // different accumulator entries): its CTAs take the SMs that the full-tile launch's last partial wave leaves.
  cudaStream_t main_s = sdpv::as_stream(stream), side_s = main_s;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  if (tailTB) {
    const int st = side_stream(dev, &side_s, &fork_ev, &join_ev);
    if (st != SDPV_OK) return st;
    cudaError_t e = cudaEventRecord(fork_ev, main_s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(side_s, fork_ev, 0);
    if (e != cudaSuccess) return sdpv::set_cuda_error(e);
  }
  for (int gofs = 0; gofs < G; gofs += kMaxG) {        // at most kMaxG moduli per launch
    const int Gl = G - gofs < kMaxG ? G - gofs : kMaxG;
    for (int part = (tailTB ? 1 : 0); part >= 0; part--) {   // the corner first, on the side stream
      const int tb = part ? tailTB : 0;
      // the diagonal items of the full tiles also take the tail rows against their row block (fused tail);
      // the tail launch is left with the last row block against the tail rows (the corner)
      const int ftail = (tailTB && !part) ? tailTB : 0, tfirst = part ? nfull / 128 : 0;
      const i64 ptiles = part ? 1 : tiles;
      const i64 nitems = ptiles * (pack > 1 ? 1 : nb) * Gl;
      if (nitems == 0) continue;
      const unsigned gx = (unsigned)(nitems < sms ? nitems : sms);  // one resident CTA per SM, items looped
      cudaStream_t ls = part ? side_s : main_s;
      if (nmode && nTB <= 32)                          // 16 epilogue warps for the short narrow items
        rns_gemm_kernel<16><<<gx, kThreadsN, smem, ls>>>(
            mAh, mAl, mBh, mBl, mTh, mTl, tb, nfull, ftail, tfirst, nmode, nTB, u8ops, nrb, acc, ldc, c->d.mods, c->d.minv,
            c->d.c14, g0, gofs, Gl, nb, M, N, KC, mode, ntn, ptiles, nitems, fresh, pack, nullptr,
            sdpv::device_error_word());
      else
        rns_gemm_kernel<8><<<gx, kThreads, smem, ls>>>(
            mAh, mAl, mBh, mBl, mTh, mTl, tb, nfull, ftail, tfirst, nmode, nTB, u8ops, 0, acc, ldc, c->d.mods, c->d.minv,
            c->d.c14, g0, gofs, Gl, nb, M, N, KC, mode, ntn, ptiles, nitems, fresh, pack, nullptr,
            sdpv::device_error_word());
      const int st = sdpv::launch_status();
      if (st != SDPV_OK) return st;
    }
  }
  if (tailTB) {
    cudaError_t e = cudaEventRecord(join_ev, side_s);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(main_s, join_ev, 0);
    if (e != cudaSuccess) return sdpv::set_cuda_error(e);
  }
  return SDPV_OK;
}

// Grouped narrow products over a device item table: every item multiplies up to 128 rows of the big side
// against up to TB rows of the small side over its own K length, and stores its output block at its own place
// in the accumulator.  Items of different shapes and K run in one launch (one CTA per SM loops over
// (item, modulus)); the operands are two stacked residue buffers (unsigned digits) with one row length KP.
extern "C" int sdpv_rns_gemm_grouped(const sdpv_ctx* c, const uint8_t* bigHi, const uint8_t* bigLo, int64_t big_rows,
                                     int64_t big_stride, const uint8_t* smallHi, const uint8_t* smallLo,
                                     int64_t small_rows, int64_t small_stride, int64_t KP, int TB, int out_mode,
                                     const int32_t* items, int64_t nitems, int16_t* acc, int64_t ldc, int64_t rows_out,
                                     int g0, int G, void* stream) {
  if (!c || g0 < 0 || G < 1 || g0 + G > c->d.n || G > 65535 || KP <= 0 || KP > 32768 || (KP & 15) || TB < 16 ||
      TB > 64 || (TB & 15) || (out_mode != 1 && out_mode != 2) || nitems < 0 || nitems > 0x7fffffff || big_rows < 1 ||
      small_rows < 1 || rows_out < 1 || ldc < 1 || !items)
    return SDPV_EINVAL;
  if (nitems == 0) return SDPV_OK;
  if (big_stride < KP * big_rows || small_stride < KP * small_rows || (big_stride & 15) || (small_stride & 15) ||
      (((uintptr_t)bigHi | (uintptr_t)bigLo | (uintptr_t)smallHi | (uintptr_t)smallLo) & 15))
    return SDPV_EINVAL;
  CUtensorMap mAh, mAl, mBh, mBl;
  const int nrb = (TB <= 32 && KP <= 64) ? (KP <= 32 ? 32 : 64) : 0, bx = nrb ? nrb : 128;   // compact slots
  if (!make_map(&mAh, bigHi, KP, big_rows, 1, G, big_stride, 128, bx) ||
      !make_map(&mAl, bigLo, KP, big_rows, 1, G, big_stride, 128, bx) ||
      !make_map(&mBh, smallHi, KP, small_rows, 1, G, small_stride, TB, bx) ||
      !make_map(&mBl, smallLo, KP, small_rows, 1, G, small_stride, TB, bx))
    return SDPV_EINVAL;
  const size_t smem = sizeof(GemmSmem) + 1024;
  const int attr_st = gemm_attr(smem);
  if (attr_st != SDPV_OK) return attr_st;
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  for (int gofs = 0; gofs < G; gofs += kMaxG) {
    const int Gl = G - gofs < kMaxG ? G - gofs : kMaxG;
    const i64 n_all = nitems * Gl;
    const unsigned gx = (unsigned)(n_all < sms ? n_all : sms);
    // M = rows_out: the accumulator planes (one per modulus) hold rows_out rows of ldc entries
    if (TB <= 32)
      rns_gemm_kernel<16><<<gx, kThreadsN, smem, sdpv::as_stream(stream)>>>(
          mAh, mAl, mBh, mBl, mBh, mBl, 0, 0, 0, 0, out_mode, TB, 1, nrb, acc, ldc, c->d.mods, c->d.minv, c->d.c14, g0,
          gofs, Gl, 1, rows_out, TB, KP, 0, 1, nitems, n_all, true, 1, items, sdpv::device_error_word());
    else
      rns_gemm_kernel<8><<<gx, kThreads, smem, sdpv::as_stream(stream)>>>(
          mAh, mAl, mBh, mBl, mBh, mBl, 0, 0, 0, 0, out_mode, TB, 1, 0, acc, ldc, c->d.mods, c->d.minv, c->d.c14, g0,
          gofs, Gl, 1, rows_out, TB, KP, 0, 1, nitems, n_all, true, 1, items, sdpv::device_error_word());
    const int st = sdpv::launch_status();
    if (st != SDPV_OK) return st;
  }
  return SDPV_OK;
}
