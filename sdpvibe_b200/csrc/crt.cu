// CRT reconstruction fused with rounding.
//
// For an entry with residues a_i (n moduli m_i, M = prod m_i, |value| < M/4):
//   y_i = a_i (M/m_i)^-1 mod m_i  (centred),  k = round(sum y_i / m_i),
//   value = sum_i y_i (M/m_i) - k M = sum_t (Z_t - k Md_t) 256^t,  Z_t = sum_i Ct[t][i] y_i
// with Ct[t][i] the signed base-256 digits of M/m_i (sdpvibe/rns.py:140-159, 227-245;
// sdpvibe/limbops.py:85-152).  A CTA handles one or two tiles of 128 entries; each tile goes through:
//   * pre-pass (one thread per entry): y_i from the int16 accumulator, split y = 128 yh + yl into
//     two K-major int8 tiles in shared memory, and k;
//   * digit contraction on the tensor cores, 64 digits at a time: Zh = Yh Ct^T, Zl = Yl Ct^T
//     (tcgen05.mma kind::i8, M = 128 entries, N = 64 digits, K = moduli), Ct resident in shared memory;
//   * epilogue (the same thread, TMEM lane = entry): z = 128 Zh + Zl - k Md, carried into 32-bit words;
//     then either the words + bit length (crt_block) or the MPF renormalisation of mpf_norm
//     (magnitude rounded half up to NB = 32L-2 bits) written straight to the output limb planes.
// No intermediate leaves the SM; one launch replaces crt_pre + digit GEMM + crt_carry + normalize.
#include "common.cuh"
#include "mpcore.cuh"

namespace {
using namespace sdpv;

constexpr int kThreads = 128;              // per 128-entry tile (TPC tiles per CTA: 128 TPC threads)
constexpr int kDig = 64;                    // digits per MMA chunk (N)
constexpr u32 kSlice = 128 * 128;

struct CrtSmemHead {
  u64 bar_ct, bar_mma[2];
  u32 tmem_slot;
  int abort;
};

constexpr int kNmax = 320;                  // moduli tables staged in shared memory (n <= 320)
constexpr int kEmax = 640;                  // CRT digits staged in shared memory (E <= 640)
struct CrtTables {
  int m[kNmax], inv[kNmax];
  float minv[kNmax];
  int md[kEmax];
};

// Dynamic shared memory: [head (8 KB)] per tile [Yh: ktc slices] [Yl: ktc slices], then [Ct: Epad/128 * ktc
// slices].  TPC tiles per CTA (1 or 2): with 2 the digit table Ct is staged once for two tiles, so two CTAs of
// 2 x 128 entries fit an SM where three of 128 did (the tables, not the tiles, fill shared memory).
template <int MODE, int TPC>
__global__ void __launch_bounds__(kThreads * TPC)
    crt_kernel(const int16_t* __restrict__ acc, i64 ldg, i64 N, i64 j0, i64 w, i64 rows, i64 rows_per_block,
               const int64_t* __restrict__ rowexp, const int64_t* __restrict__ colexp, int L, int n, int E, int W,
               int ktc, int Epad, const int32_t* __restrict__ mods, const float* __restrict__ minvs,
               const int32_t* __restrict__ invs, const int32_t* __restrict__ md, const uint8_t* __restrict__ ct,
               int32_t* __restrict__ out, int64_t* __restrict__ out2, const int32_t* __restrict__ pred,
               unsigned* __restrict__ err) {
  if (pred && *pred == 0) return;                      // predicated launch: nothing to do this time
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* base = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  CrtSmemHead& H = *reinterpret_cast<CrtSmemHead*>(base);
  CrtTables& TB = *reinterpret_cast<CrtTables*>(base + 64);
  const int tid = threadIdx.x, warp = tid >> 5, half = tid >> 7, lt = tid & 127;   // tile of the CTA, entry
  uint8_t* Yh = base + 8192 + (size_t)half * 2 * ktc * kSlice;
  uint8_t* Yl = Yh + (size_t)ktc * kSlice;
  uint8_t* Ct = base + 8192 + (size_t)TPC * 2 * ktc * kSlice;
  const i64 B = rows * w;
  const i64 ntiles = (B + 127) / 128;

  if (tid == 0) {
    mbar_init(&H.bar_ct, 1);
    for (int h = 0; h < TPC; h++) mbar_init(&H.bar_mma[h], 1);
    H.abort = 0;
    mbar_fence_init();
  }
  if (warp == 0) {
    tmem_alloc(&H.tmem_slot, 2 * kDig * TPC);
    tmem_relinquish();
  }
  for (int g = tid; g < kNmax; g += kThreads * TPC) {
    TB.m[g] = g < n ? mods[g] : 1;
    TB.inv[g] = g < n ? invs[g] : 0;
    TB.minv[g] = g < n ? minvs[g] : 1.f;
  }
  for (int t = tid; t < kEmax; t += kThreads * TPC) TB.md[t] = t < E ? md[t] : 0;
  __syncthreads();
  tc_fence_after();
  const u32 tmem = H.tmem_slot + (u32)half * 2 * kDig;              // this tile's Zh, Zl columns
  if (tid == 0) {
    u32 bytes = (u32)(Epad / 128) * ktc * kSlice;
    mbar_expect_tx(&H.bar_ct, bytes);
    for (u32 off = 0; off < bytes; off += kSlice) bulk_load(Ct + off, ct + off, kSlice, &H.bar_ct);
  }
  if (!mbar_wait(&H.bar_ct, 0, err)) H.abort = 1;

  const u32 idesc = idesc_i8(128, kDig);
  const int ksteps = (n + 31) / 32;
  const int nchunk = (E + kDig - 1) / kDig;
  u32 phase = 0;
  u32 words[160];

  for (i64 tile2 = blockIdx.x; tile2 * TPC < ntiles && !H.abort; tile2 += gridDim.x) {
    // ---- pre-pass: y_i, its int8 digits, k
    const i64 tile = tile2 * TPC + half;
    const i64 e = tile * 128 + lt;
    const bool valid = e < B;
    const i64 r = valid ? e / w : 0, jj = valid ? e - (e / w) * w : 0;
    const int16_t* ap = acc + r * N + j0 + jj;
    float ks = 0.f;
    for (int gb = 0; gb < ktc * 128; gb += 64) {
      // the 64 loads of this group of moduli issued before any is used (they are independent): the pre-pass
      // is bound by memory latency, one per group
      int av[64];
#pragma unroll
      for (int q = 0; q < 64; q++) av[q] = (valid && gb + q < n) ? (int)__ldcs(ap + (i64)(gb + q) * ldg) : 0;
#pragma unroll
      for (int h = 0; h < 4; h++) {                              // 16 moduli per 16-byte digit chunk
        u32 ph[4], pl[4];
#pragma unroll
        for (int q = 0; q < 16; q++) {
          const int g = gb + 16 * h + q;
          int y = 0;
          if (valid && g < n) {
            const int m = TB.m[g];
            const float mi = TB.minv[g];
            // centred residue of x = a inv (0 <= x < 2^30): nearest quotient from the float estimate (off by
            // at most one), then at most one correction each way into [-(m >> 1), m >> 1]
            const int x = av[16 * h + q] * TB.inv[g];
            y = x - __float2int_rn(__int2float_rn(x) * mi) * m;
            y -= (y > (m >> 1)) ? m : 0;
            y += (y < -(m >> 1)) ? m : 0;
            ks += (float)y * mi;
          }
          int yl = ((y + 64) & 127) - 64, yh = (y - yl) >> 7;
          if ((q & 3) == 0) ph[q >> 2] = pl[q >> 2] = 0;
          ph[q >> 2] |= (u32)(yh & 255) << (8 * (q & 3));
          pl[q >> 2] |= (u32)(yl & 255) << (8 * (q & 3));
        }
        const int g16 = gb + 16 * h;
        int kt = g16 >> 7, chunk = (g16 & 127) >> 4;
        *reinterpret_cast<uint4*>(Yh + kt * kSlice + sw128_off(lt, chunk)) = make_uint4(ph[0], ph[1], ph[2], ph[3]);
        *reinterpret_cast<uint4*>(Yl + kt * kSlice + sw128_off(lt, chunk)) = make_uint4(pl[0], pl[1], pl[2], pl[3]);
      }
    }
    const i64 kq = (i64)__float2int_rd(ks + 0.5f);
    const int kq32 = (int)kq;                                          // |k| <= n / 2
    fence_proxy_async_smem();
    __syncthreads();

    // ---- digit chunks: MMA, then carry into words (crt_block streams them straight out, tracking the
    //      highest word that differs from each possible sign extension for the bit length)
    i64 carry = 0;
    int nw = 0;
    int hz = -1, ho = -1;                              // highest word != 0, != 0xffffffff
    u32 hzv = 0, hov = 0, wtop = 0;
    for (int ch = 0; ch < nchunk; ch++) {
      if (lt == 0) {                                   // one issuing thread per tile
        tc_fence_after();
        const u32 ctc = smem_u32(Ct) + (u32)((ch * kDig) / 128) * ktc * kSlice + (u32)((ch * kDig) % 128) * 128;
        for (int s = 0; s < ksteps; s++) {
          int kt = s >> 2, ko = (s & 3) * 32;
          u64 bd = sdesc_sw128(ctc + kt * kSlice + ko);
          mma_i8(tmem + 0, sdesc_sw128(smem_u32(Yh) + kt * kSlice + ko), bd, idesc, s ? 1u : 0u);
          mma_i8(tmem + kDig, sdesc_sw128(smem_u32(Yl) + kt * kSlice + ko), bd, idesc, s ? 1u : 0u);
        }
        mma_commit(&H.bar_mma[half]);
      }
      if (!mbar_wait(&H.bar_mma[half], phase, err)) H.abort = 1;
      phase ^= 1;
      tc_fence_after();
#pragma unroll 1
      for (int c32 = 0; c32 < kDig; c32 += 32) {
        u32 zh[32], zl[32];
        tmem_ld32(tmem + ((u32)((warp & 3) * 32) << 16) + c32, zh);
        tmem_ld32(tmem + ((u32)((warp & 3) * 32) << 16) + kDig + c32, zl);
        tmem_ld_wait();
#pragma unroll
        for (int j = 0; j < 32; j += 4) {
          int t0 = ch * kDig + c32 + j;
          if (t0 >= E) break;
          // z = 128 Zh + Zl - k Md fits int32: |Zh| <= n 2^14 <= 320 2^14 < 2^23, |Zl| < 2^21, |k Md| < 2^15.
          // The word's four digits are summed apart from the carry (a tree, independent of the previous
          // word), so only one 64-bit add per word waits on the carry chain
          i64 z4[4];
#pragma unroll
          for (int u = 0; u < 4; u++)
            z4[u] = (i64)(128 * (int)zh[j + u] + (int)zl[j + u] - kq32 * TB.md[t0 + u]) * (i64)(1 << (8 * u));
          const i64 v = carry + ((z4[0] + z4[1]) + (z4[2] + z4[3]));
          const u32 wv = (u32)v;
          if (MODE == 0) {
            if (valid) out[(i64)nw * B + e] = (int32_t)wv;
            if (wv != 0u) hz = nw, hzv = wv;
            if (wv != 0xffffffffu) ho = nw, hov = wv;
            wtop = wv;
          } else {
            words[nw] = wv;
          }
          nw++;
          carry = v >> 32;
        }
      }
      tc_fence_before();
      __syncthreads();
    }

    // ---- outputs
    if (valid) {
      if (MODE == 0) {
        // bit length of v (v >= 0) or of ~v (v < 0): the highest word differing from the extension
        const bool ng = (wtop >> 31) != 0;
        const int k = ng ? ho : hz;
        const u32 x = ng ? ~hov : hzv;
        out2[e] = k < 0 ? 0 : 32 * (i64)k + 32 - __clz(x);
      } else {
        bool ng = words[W - 1] >> 31;
        if (ng) neg_words(words, W);
        int bl = bitlen_mag(words, W);
        if (!bl) {
          for (int k = 0; k < L; k++) out[(i64)k * B + e] = 0;
          out2[e] = SDPV_EZ;
        } else {
          u32 rr[160];
          int s = bl - (32 * L - 2);
          mag_shift(words, W, s, rr, L);
          if (ng) neg_words(rr, L);
          for (int k = 0; k < L; k++) out[(i64)k * B + e] = (int32_t)rr[k];
          out2[e] = rowexp[r] + colexp[(r / rows_per_block) * N + j0 + jj] + s;
        }
      }
    }
  }
  __syncthreads();
  if (warp == 0) tmem_dealloc(H.tmem_slot, 2 * kDig * TPC);
}

template <int MODE, int TPC>
int launch_crt_t(const sdpv_ctx* c, const int16_t* acc, i64 ldg, i64 N, i64 j0, i64 w, i64 rows, i64 rpb,
                 const int64_t* rowexp, const int64_t* colexp, int L, int32_t* out, int64_t* out2, cudaStream_t st,
                 const int32_t* pred, size_t smem) {
  const CtxDev& d = c->d;
  static bool attr_set[64] = {};
  static size_t attr_val[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr_set[dev & 63] || attr_val[dev & 63] < smem) {
    cudaError_t e = cudaFuncSetAttribute(crt_kernel<MODE, TPC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return set_cuda_error(e);
    attr_set[dev & 63] = true;
    attr_val[dev & 63] = smem;
  }
  i64 B = rows * w;
  i64 ntiles = (B + 127) / 128, nunits = (ntiles + TPC - 1) / TPC;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // CTAs per SM: the tuned count for one-tile CTAs; two-tile CTAs as many as shared memory holds (at most 2)
  i64 per_sm = TPC == 1 ? (i64)sdpv::tune(SDPV_TUNE_CRT_CTAS) : (i64)((228 * 1024) / (smem + 1024));
  if (per_sm < 1) per_sm = 1;
  if (TPC == 2 && per_sm > 2) per_sm = 2;
  i64 gx = per_sm * sms;
  if (gx > nunits) gx = nunits;
  crt_kernel<MODE, TPC><<<(unsigned)gx, kThreads * TPC, smem, st>>>(
      acc, ldg, N, j0, w, rows, rpb, rowexp, colexp, L, d.n, d.E, d.W, d.ktc, d.Epad, d.mods, d.minv, d.inv, d.md,
      d.ct, out, out2, pred, device_error_word());
  return launch_status();
}

template <int MODE>
int launch_crt(const sdpv_ctx* c, const int16_t* acc, i64 ldg, i64 N, i64 j0, i64 w, i64 rows, i64 rpb,
               const int64_t* rowexp, const int64_t* colexp, int L, int32_t* out, int64_t* out2, cudaStream_t st,
               const int32_t* pred = nullptr) {
  const CtxDev& d = c->d;
  if (d.n > kNmax || d.E > kEmax) return SDPV_EINVAL;
  const size_t tables = (size_t)(d.Epad / 128) * d.ktc * kSlice, tile = (size_t)2 * d.ktc * kSlice;
  const size_t smem1 = 1024 + 8192 + tile + tables, smem2 = 1024 + 8192 + 2 * tile + tables;
  // two tiles per CTA when two such CTAs fit an SM (shared memory) and there are tiles for them
  if (smem2 <= 112 * 1024 && rows * w > 128 * 148)
    return launch_crt_t<MODE, 2>(c, acc, ldg, N, j0, w, rows, rpb, rowexp, colexp, L, out, out2, st, pred, smem2);
  if (smem1 > 227 * 1024) return SDPV_EINVAL;
  return launch_crt_t<MODE, 1>(c, acc, ldg, N, j0, w, rows, rpb, rowexp, colexp, L, out, out2, st, pred, smem1);
}

}  // namespace

extern "C" int sdpv_crt_block(const sdpv_ctx* c, const int16_t* acc, int64_t ldg, int64_t N, int64_t j0, int64_t w,
                              int64_t rows, int32_t* words, int64_t* bitlen, void* stream) {
  if (!c || N < 0 || j0 < 0 || w < 0 || j0 + w > N || rows < 0 || c->d.W > 160) return SDPV_EINVAL;
  if (rows == 0 || w == 0) return SDPV_OK;
  return launch_crt<0>(c, acc, ldg, N, j0, w, rows, rows, nullptr, nullptr, c->d.L, words, bitlen,
                       sdpv::as_stream(stream));
}

extern "C" int sdpv_crt_norm(const sdpv_ctx* c, const int16_t* acc, int64_t ldg, int64_t N, int64_t j0, int64_t w,
                             int64_t rows, int64_t rows_per_block, const int64_t* rowexp, const int64_t* colexp, int L,
                             int32_t* O, int64_t* eO, void* stream) {
  if (!c || N < 0 || j0 < 0 || w < 0 || j0 + w > N || rows < 0 || rows_per_block < 1 || L < 1 || L > 160 ||
      c->d.W > 160)
    return SDPV_EINVAL;
  if (rows == 0 || w == 0) return SDPV_OK;
  return launch_crt<1>(c, acc, ldg, N, j0, w, rows, rows_per_block, rowexp, colexp, L, O, eO,
                       sdpv::as_stream(stream));
}

extern "C" int sdpv_crt_norm_if(const sdpv_ctx* c, const int16_t* acc, int64_t ldg, int64_t N, int64_t j0, int64_t w,
                                int64_t rows, int64_t rows_per_block, const int64_t* rowexp, const int64_t* colexp,
                                int L, int32_t* O, int64_t* eO, const int32_t* pred, void* stream) {
  if (!c || !pred || N < 0 || j0 < 0 || w < 0 || j0 + w > N || rows < 0 || rows_per_block < 1 || L < 1 || L > 160 ||
      c->d.W > 160)
    return SDPV_EINVAL;
  if (rows == 0 || w == 0) return SDPV_OK;
  return launch_crt<1>(c, acc, ldg, N, j0, w, rows, rows_per_block, rowexp, colexp, L, O, eO,
                       sdpv::as_stream(stream), pred);
}
