// Grouped Cholesky / triangular-solve support kernels: every launch works through a device descriptor table
// whose rows may belong to blocks of different sizes, so one launch serves all blocks of a wave.
//
// Storage (limb planes, plane stride = the arena's entry count):
//   factor arena   (L, T, 32, 32)  lower tiles (b, i, j), i >= j, of every block, fixed point at one exponent e;
//   inverse arena  (L, D, 32, 32)  the inverse X_j of every diagonal tile, exponent xe[d] per tile;
//   solve arena    (L, RT, 32, m)  32-row tiles of the right-hand sides / solutions, exponents Pe (RT, m) per
//                                  (row tile, column);
//   workspaces     (L, rows, KP)   operand rows gathered for one grouped residue product.
// The kernels: tile copies into workspaces (grp_copy, optional transpose, shared-memory staged), the rounding
// of CRT outputs to a fixed exponent combined into a destination (grp_finish_fixed), the solves' per-column
// exponents, rounding and aligned sums (grp_solve_round) and rescales (grp_merge), and the tile conversions
// around the base-case kernels (grp_tile_widen, grp_tile_narrow).  Roundings are the reference's:
// floor(x / 2^s + 1/2) on two's-complement words (sdpvibe/limbops.py:31-62), the aligned sum of two operands
// rounded independently to max(ea, eb) + 1 (sdpvibe/batched.py:55-79), per-column output exponents from the
// maximal bit length (sdpvibe/batched.py:200-231).
#include "common.cuh"

namespace {

constexpr int kArenas = 4;
constexpr int kLMax = 128;                 // limbs of an intermediate kept in registers / local memory
constexpr int kMaxSrc = 7;                 // rounded products summed into one destination by grp_finish_fixed

struct Arenas {
  int32_t* p[kArenas];
  i64 plane[kArenas];
};

// Word i of a two's-complement number of n words read through `at` (sign-extended above, zero below).
template <class At>
__device__ __forceinline__ u64 word_ext(At at, int n, i64 i, u64 ext) {
  if (i < 0) return 0;
  if (i >= n) return ext;
  return (u64)at(i);
}

// Streaming floor(x / 2^s + 1/2): output word k of the rounded value, produced in increasing k.
struct ShiftStream {
  i64 q;
  int r;
  u64 lo, carry, ext;
};
template <class At>
__device__ __forceinline__ void shr_begin(ShiftStream& st, At at, int n, i64 s) {
  st.ext = ((u32)at(n - 1) >> 31) ? 0xffffffffull : 0ull;
  st.q = s >> 5;
  st.r = (int)(s - 32 * st.q);
  const i64 sb = s - 1, qb = sb >> 5;
  const int rb = (int)(sb - 32 * qb);
  st.carry = sb >= 0 ? ((word_ext(at, n, qb, st.ext) >> rb) & 1ull) : 0ull;
  st.lo = word_ext(at, n, st.q, st.ext);
}
template <class At>
__device__ __forceinline__ u32 shr_next(ShiftStream& st, At at, int n, int k) {
  const u64 hi = word_ext(at, n, st.q + k + 1, st.ext);
  const u64 v = ((((hi << 32) | st.lo) >> st.r) & 0xffffffffull) + st.carry;
  st.lo = hi;
  st.carry = v >> 32;
  return (u32)v;
}
// The whole rounded value into out[0 .. nout).
template <class At>
__device__ __forceinline__ void shr_all(At at, int n, i64 s, u32* out, int nout) {
  ShiftStream st;
  shr_begin(st, at, n, s);
  for (int k = 0; k < nout; k++) out[k] = shr_next(st, at, n, k);
}

__device__ __forceinline__ int bitlen_words(const u32* x, int n) {
  const u32 ext = (x[n - 1] >> 31) ? 0xffffffffu : 0u;
  for (int k = n - 1; k >= 0; k--) {
    const u32 v = x[k] ^ ext;
    if (v) return 32 * k + 32 - __clz(v);
  }
  return 0;
}

// ---------------------------------------------------------------- tile copies into a workspace
// desc (8 int64): src arena, src base entry, src row stride, dst base entry, dst row stride, rows, cols (<= 32),
// transpose.  One CTA per descriptor and limb plane (grid y); dst[r][c] = src[r][c], or dst[c][r] = src[r][c]
// staged through shared memory so that both sides are read / written along rows.
__global__ void __launch_bounds__(256) grp_copy_kernel(Arenas src, int32_t* __restrict__ dst, i64 dplane, int L,
                                                       const i64* __restrict__ desc) {
  __shared__ int32_t t[32][33];
  const i64* d = desc + 8 * (i64)blockIdx.x;
  const int sid = (int)d[0], rows = (int)d[5], cols = (int)d[6], trans = (int)d[7];
  const i64 sbase = d[1], sld = d[2], dbase = d[3], dld = d[4];
  const int tid = threadIdx.x;
  for (int k = blockIdx.y; k < L; k += gridDim.y) {
    const int32_t* S = src.p[sid] + (i64)k * src.plane[sid] + sbase;
    int32_t* D = dst + (i64)k * dplane + dbase;
    if (!trans) {
      for (int idx = tid; idx < rows * 32; idx += 256) {
        const int r = idx >> 5, c = idx & 31;
        if (c < cols) D[r * dld + c] = S[r * sld + c];
      }
    } else {
      for (int idx = tid; idx < 1024; idx += 256) {
        const int r = idx >> 5, c = idx & 31;
        t[r][c] = (r < rows && c < cols) ? S[r * sld + c] : 0;
      }
      __syncthreads();
      for (int idx = tid; idx < 1024; idx += 256) {
        const int c = idx >> 5, r = idx & 31;          // destination row c, column r
        if (r < rows && c < cols) D[c * dld + r] = t[r][c];
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------- fixed-exponent rounding into a destination
// desc (40 int64): out arena, out base, out ld, base arena (-1: zero), base base, base ld, rows, cols, nsrc (<= 7),
// then per source: CRT entry base, sign (+1 / -1), shift constant, exponent index (-1: none).  Entry (r, c):
//   out = base + sum_i sign_i round(W_i[r][c] / 2^s_i) mod 2^(32 L),  s_i = cst_i - xe[idx_i]
// where W_i[r][c] is the CRT value (W words, planes Ntot apart) at entry crt_base_i + r * w + c.  Four CTAs
// per descriptor (grid y), each a quarter of the rows: one entry per thread for a 32 x 32 block.
__global__ void __launch_bounds__(256) grp_finish_fixed_kernel(const int32_t* __restrict__ Wd, int W, i64 Ntot, i64 w,
                                                               Arenas ar, int L, const i64* __restrict__ xe,
                                                               const i64* __restrict__ desc) {
  const i64* d = desc + 40 * (i64)blockIdx.x;
  const int oid = (int)d[0], bid = (int)d[3], rows = (int)d[6], cols = (int)d[7];
  const int ns = (int)d[8] < kMaxSrc ? (int)d[8] : kMaxSrc;
  const i64 obase = d[1], old_ = d[2], bbase = d[4], bld = d[5];
  const int rpart = (rows + gridDim.y - 1) / gridDim.y, rlo = blockIdx.y * rpart;   // this CTA's rows
  const int rhi = rlo + rpart < rows ? rlo + rpart : rows;
  for (int idx = threadIdx.x; idx < (rhi - rlo) * cols; idx += blockDim.x) {
    const int r = rlo + idx / cols, c = idx % cols;
    ShiftStream st[kMaxSrc];
    i64 sg[kMaxSrc];
    const int32_t* src[kMaxSrc];
    for (int i = 0; i < ns; i++) {
      const i64* si = d + 9 + 4 * i;
      src[i] = Wd + si[0] + (i64)r * w + c;
      sg[i] = si[1];
      const i64 s = si[2] - (si[3] >= 0 ? xe[si[3]] : 0);
      const int32_t* p = src[i];
      shr_begin(st[i], [&](i64 k) { return (u32)p[k * Ntot]; }, W, s);
    }
    const int32_t* bp = bid >= 0 ? ar.p[bid] + bbase + (i64)r * bld + c : nullptr;
    int32_t* op = ar.p[oid] + obase + (i64)r * old_ + c;
    i64 carry = 0;
    for (int k = 0; k < L; k++) {
      i64 t = carry + (bp ? (i64)(u32)bp[(i64)k * ar.plane[bid]] : 0);
      for (int i = 0; i < ns; i++) {
        const int32_t* p = src[i];
        const u32 v = shr_next(st[i], [&](i64 kk) { return (u32)p[kk * Ntot]; }, W, k);
        t += sg[i] * (i64)v;
      }
      op[(i64)k * ar.plane[oid]] = (int32_t)(u32)t;
      carry = t >> 32;
    }
  }
}

// ---------------------------------------------------------------- triangular solves: fused 'col' rounding
// desc (10 int64): CRT row0, rows (32 nrt), column c0, ncols (<= 32), eA constant, eA index (-1 none, else +
// xe[idx]), B row tile (its column exponents), mode, base row tile 0, destination row tile 0.  One CTA per
// group and column chunk: for each column c, mx = max over the group's rows of the CRT bit length,
// s = mx - (32 L - 32), e_in = eA + Pe[B row tile][c], eU = e_in + s ('col' rounding, sdpvibe/batched.py:
// 200-231); then every entry u = round(U / 2^s) goes to the destination row tiles dst0 .. dst0 + nrt - 1:
// mode 0 stores it (exponent eU), modes 1 / 2 form the aligned difference / sum with the base row tiles
// base0 .. (exponent eb): e2 = max(eb, eU) + 1, round(b / 2^(e2 - eb)) -/+ round(u / 2^(e2 - eU))
// (sdpvibe/batched.py:82-92).
__global__ void __launch_bounds__(256) grp_solve_round_kernel(const int32_t* __restrict__ Wd, const i64* __restrict__ bl,
                                                              int W, i64 Ntot, i64 w, int32_t* __restrict__ P,
                                                              i64 Pplane, i64* __restrict__ Pe, i64 m, int L,
                                                              const i64* __restrict__ xe,
                                                              const i64* __restrict__ desc) {
  __shared__ i64 s_part[8][32];
  __shared__ i64 s_su[32], s_eu[32];
  const i64* d = desc + 10 * (i64)blockIdx.x;
  const i64 row0 = d[0], rows = d[1], c0 = d[2], brt0 = d[8], drt0 = d[9];
  const int ncols = (int)d[3], mode = (int)d[7];
  const int tid = threadIdx.x, c = tid & 31, rg = tid >> 5;
  i64 mx = 0;
  if (c < ncols)
    for (i64 r = rg; r < rows; r += 8) {
      const i64 v = bl[(row0 + r) * w + c0 + c];
      mx = v > mx ? v : mx;
    }
  s_part[rg][c] = mx;
  __syncthreads();
  if (tid < ncols) {
    i64 v = s_part[0][tid];
    for (int q = 1; q < 8; q++) v = s_part[q][tid] > v ? s_part[q][tid] : v;
    const i64 s = v - (32 * (i64)L - 32);
    const i64 eA = d[4] + (d[5] >= 0 ? xe[d[5]] : 0);
    s_su[tid] = s;
    s_eu[tid] = eA + Pe[d[6] * m + c0 + tid] + s;
  }
  __syncthreads();
  const i64 nrt = rows / 32;
  for (i64 idx = tid; idx < rows * ncols; idx += blockDim.x) {
    const int cc = (int)(idx % ncols);
    const i64 rr = idx / ncols, t = rr / 32, r = rr % 32;
    const int32_t* u = Wd + (row0 + rr) * w + c0 + cc;
    auto uat = [&](i64 k) { return (u32)u[k * Ntot]; };
    int32_t* dst = P + (drt0 + t) * 32 * m + r * m + c0 + cc;
    if (mode == 0) {
      ShiftStream st;
      shr_begin(st, uat, W, s_su[cc]);
      for (int k = 0; k < L; k++) dst[(i64)k * Pplane] = (int32_t)shr_next(st, uat, W, k);
      continue;
    }
    u32 uv[kLMax];
    shr_all(uat, W, s_su[cc], uv, L);
    const i64 eb = Pe[(brt0 + t) * m + c0 + cc];
    const i64 eu = s_eu[cc];
    const i64 e2 = (eb > eu ? eb : eu) + 1;
    const int32_t* b = P + (brt0 + t) * 32 * m + r * m + c0 + cc;
    auto bat = [&](i64 k) { return (u32)b[k * Pplane]; };
    auto vat = [&](i64 k) { return uv[k]; };
    ShiftStream sb, su;
    shr_begin(sb, bat, L, e2 - eb);
    shr_begin(su, vat, L, e2 - eu);
    const i64 sgn = mode == 1 ? -1 : 1;
    i64 carry = 0;
    u32 out[kLMax];
    for (int k = 0; k < L; k++) {
      const u32 x = shr_next(sb, bat, L, k), y = shr_next(su, vat, L, k);
      const i64 tt = (i64)x + sgn * (i64)y + carry;
      out[k] = (u32)tt;
      carry = tt >> 32;
    }
    for (int k = 0; k < L; k++) dst[(i64)k * Pplane] = (int32_t)out[k];
  }
  __syncthreads();
  if (tid < ncols) {
    for (i64 t = 0; t < nrt; t++) {
      i64 e = s_eu[tid];
      if (mode) {
        const i64 eb = Pe[(brt0 + t) * m + c0 + tid];
        e = (eb > e ? eb : e) + 1;
      }
      Pe[(drt0 + t) * m + c0 + tid] = e;
    }
  }
}

// ---------------------------------------------------------------- triangular solves: common column exponents
// desc (4 int64): first row tile, row tiles, column c0, ncols (<= 32).  ee[c] = max over the row tiles of
// Pe[rt][c]; every entry is re-rounded to it (sdpvibe/batched.py:45-52) and Pe set to ee.
__global__ void __launch_bounds__(256) grp_merge_kernel(int32_t* __restrict__ P, i64 Pplane, i64* __restrict__ Pe,
                                                        i64 m, int L, const i64* __restrict__ desc) {
  __shared__ i64 s_ee[32];
  const i64* d = desc + 4 * (i64)blockIdx.x;
  const i64 rt0 = d[0], nrt = d[1], c0 = d[2];
  const int ncols = (int)d[3];
  if (threadIdx.x < ncols) {
    i64 ee = Pe[rt0 * m + c0 + threadIdx.x];
    for (i64 t = 1; t < nrt; t++) {
      const i64 v = Pe[(rt0 + t) * m + c0 + threadIdx.x];
      ee = v > ee ? v : ee;
    }
    s_ee[threadIdx.x] = ee;
  }
  __syncthreads();
  const i64 n = nrt * 32 * ncols;
  for (i64 idx = threadIdx.x; idx < n; idx += blockDim.x) {
    const int c = (int)(idx % ncols);
    const i64 rr = idx / ncols, t = rr / 32, r = rr % 32;
    const i64 s = s_ee[c] - Pe[(rt0 + t) * m + c0 + c];
    if (s == 0) continue;
    int32_t* x = P + (rt0 + t) * 32 * m + r * m + c0 + c;
    auto at = [&](i64 k) { return (u32)x[k * Pplane]; };
    ShiftStream st;                          // in place: word k is written after words >= k were read
    shr_begin(st, at, L, s);
    for (int k = 0; k < L; k++) {
      const u32 v = shr_next(st, at, L, k);
      x[(i64)k * Pplane] = (int32_t)v;
    }
  }
  __syncthreads();
  if (threadIdx.x < ncols)
    for (i64 t = 0; t < nrt; t++) Pe[(rt0 + t) * m + c0 + threadIdx.x] = s_ee[threadIdx.x];
}

// ---------------------------------------------------------------- base-tile conversions
// Diagonal tile (factor arena entry base fbase[t], exponent e) -> wide fixed point (WL words, exponent -F):
// the exact shift by e + F; entries above the diagonal are zero.  Out entry-major (tiles, 32, 32, WL).
__global__ void __launch_bounds__(256) grp_tile_widen_kernel(const int32_t* __restrict__ Fa, i64 Fplane, int L,
                                                             i64 e, int WL, int LF, const i64* __restrict__ fbase,
                                                             u32* __restrict__ out) {
  const i64 base = fbase[blockIdx.x];
  const i64 s = -32 * (i64)LF - e;
  for (int idx = threadIdx.x; idx < 1024; idx += blockDim.x) {
    const int r = idx >> 5, c = idx & 31;
    u32* o = out + ((i64)blockIdx.x * 1024 + idx) * WL;
    if (c > r) {
      for (int k = 0; k < WL; k++) o[k] = 0;
      continue;
    }
    const int32_t* x = Fa + base + idx;
    auto at = [&](i64 k) { return (u32)x[k * Fplane]; };
    ShiftStream st;
    shr_begin(st, at, L, s);
    for (int k = 0; k < WL; k++) o[k] = shr_next(st, at, L, k);
  }
}

// Factored tile (wide, exponent -F) -> the factor arena at exponent e (L limbs, zero above the diagonal);
// its inverse (wide) -> the inverse arena at xe = max bit length - F - (32 L - 32) over the tile (one exponent
// per tile, sdpvibe/batched.py:243-262).
__global__ void __launch_bounds__(256) grp_tile_narrow_kernel(const u32* __restrict__ Lw, const u32* __restrict__ Xw,
                                                              int WL, int LF, int32_t* __restrict__ Fa, i64 Fplane,
                                                              int L, i64 e, const i64* __restrict__ fbase,
                                                              int32_t* __restrict__ Xa, i64 Xplane,
                                                              const i64* __restrict__ xidx, i64* __restrict__ xe) {
  __shared__ int s_max[8];
  const i64 F = 32 * (i64)LF;
  const i64 base = fbase[blockIdx.x], xi = xidx[blockIdx.x];
  int mx = 0;
  for (int idx = threadIdx.x; idx < 1024; idx += blockDim.x) {
    const int r = idx >> 5, c = idx & 31;
    const u32* lw = Lw + ((i64)blockIdx.x * 1024 + idx) * WL;
    int32_t* fo = Fa + base + idx;
    if (c > r) {
      for (int k = 0; k < L; k++) fo[(i64)k * Fplane] = 0;
    } else {
      auto at = [&](i64 k) { return lw[k]; };
      ShiftStream st;
      shr_begin(st, at, WL, e + F);
      for (int k = 0; k < L; k++) fo[(i64)k * Fplane] = (int32_t)shr_next(st, at, WL, k);
    }
    const int b = bitlen_words(Xw + ((i64)blockIdx.x * 1024 + idx) * WL, WL);
    mx = b > mx ? b : mx;
  }
  for (int o = 16; o; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x < 32) {
    int v = threadIdx.x < (blockDim.x >> 5) ? s_max[threadIdx.x] : 0;
    for (int o = 16; o; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) s_max[0] = v;
  }
  __syncthreads();
  const i64 ex = (i64)s_max[0] - F - (32 * (i64)L - 32);
  for (int idx = threadIdx.x; idx < 1024; idx += blockDim.x) {
    const u32* xw = Xw + ((i64)blockIdx.x * 1024 + idx) * WL;
    auto at = [&](i64 k) { return xw[k]; };
    ShiftStream st;
    shr_begin(st, at, WL, ex + F);
    int32_t* xo = Xa + xi * 1024 + idx;
    for (int k = 0; k < L; k++) xo[(i64)k * Xplane] = (int32_t)shr_next(st, at, WL, k);
  }
  if (threadIdx.x == 0) xe[xi] = ex;
}

Arenas make_arenas(int32_t* const* ptrs, const int64_t* planes, int n) {
  Arenas a{};
  for (int i = 0; i < kArenas; i++) {
    a.p[i] = i < n ? ptrs[i] : nullptr;
    a.plane[i] = i < n ? planes[i] : 0;
  }
  return a;
}

}  // namespace

extern "C" int sdpv_grp_copy(int32_t* const* src_host, const int64_t* src_planes_host, int nsrc, int32_t* dst,
                             int64_t dst_plane, int L, const int64_t* desc, int64_t ndesc, void* stream) {
  if (nsrc < 1 || nsrc > kArenas || !src_host || !src_planes_host || !dst || L < 1 || ndesc < 0 ||
      ndesc > 0x7fffffff || (ndesc && !desc))
    return SDPV_EINVAL;
  if (ndesc == 0) return SDPV_OK;
  const dim3 grid((unsigned)ndesc, (unsigned)(L < 65535 ? L : 65535));
  grp_copy_kernel<<<grid, 256, 0, sdpv::as_stream(stream)>>>(make_arenas(src_host, src_planes_host, nsrc), dst,
                                                              dst_plane, L, desc);
  return sdpv::launch_status();
}

extern "C" int sdpv_grp_finish_fixed(const int32_t* Wd, int W, int64_t Ntot, int64_t w, int32_t* const* ar_host,
                                     const int64_t* planes_host, int nar, int L, const int64_t* xe, const int64_t* desc,
                                     int64_t ndesc, void* stream) {
  if (!Wd || W < 1 || nar < 1 || nar > kArenas || !ar_host || !planes_host || L < 1 || ndesc < 0 ||
      ndesc > 0x7fffffff || (ndesc && !desc))
    return SDPV_EINVAL;
  if (ndesc == 0) return SDPV_OK;
  grp_finish_fixed_kernel<<<dim3((unsigned)ndesc, 4), 256, 0, sdpv::as_stream(stream)>>>(
      Wd, W, Ntot, w, make_arenas(ar_host, planes_host, nar), L, xe, desc);
  return sdpv::launch_status();
}

extern "C" int sdpv_grp_solve_round(const int32_t* Wd, const int64_t* bl, int W, int64_t Ntot, int64_t w, int32_t* P,
                                    int64_t Pplane, int64_t* Pe, int64_t m, int L, const int64_t* xe, const int64_t* desc,
                                    int64_t ndesc, void* stream) {
  if (!Wd || !bl || W < 1 || !P || !Pe || m < 1 || L < 1 || L > kLMax || ndesc < 0 || ndesc > 0x7fffffff ||
      (ndesc && !desc))
    return SDPV_EINVAL;
  if (ndesc == 0) return SDPV_OK;
  grp_solve_round_kernel<<<(unsigned)ndesc, 256, 0, sdpv::as_stream(stream)>>>(Wd, bl, W, Ntot, w, P, Pplane, Pe, m, L,
                                                                                xe, desc);
  return sdpv::launch_status();
}

extern "C" int sdpv_grp_merge(int32_t* P, int64_t Pplane, int64_t* Pe, int64_t m, int L, const int64_t* desc,
                              int64_t ndesc, void* stream) {
  if (!P || !Pe || m < 1 || L < 1 || ndesc < 0 || ndesc > 0x7fffffff || (ndesc && !desc)) return SDPV_EINVAL;
  if (ndesc == 0) return SDPV_OK;
  grp_merge_kernel<<<(unsigned)ndesc, 256, 0, sdpv::as_stream(stream)>>>(P, Pplane, Pe, m, L, desc);
  return sdpv::launch_status();
}

extern "C" int sdpv_grp_tile_widen(const int32_t* Fa, int64_t Fplane, int L, int64_t e, int WL, int LF,
                                   const int64_t* fbase, int64_t ntiles, uint32_t* out, void* stream) {
  if (!Fa || !fbase || !out || L < 1 || WL <= L || LF < 2 || ntiles < 0 || ntiles > 0x7fffffff) return SDPV_EINVAL;
  if (ntiles == 0) return SDPV_OK;
  grp_tile_widen_kernel<<<(unsigned)ntiles, 256, 0, sdpv::as_stream(stream)>>>(Fa, Fplane, L, e, WL, LF, fbase, out);
  return sdpv::launch_status();
}

extern "C" int sdpv_grp_tile_narrow(const uint32_t* Lw, const uint32_t* Xw, int WL, int LF, int32_t* Fa, int64_t Fplane,
                                    int L, int64_t e, const int64_t* fbase, int32_t* Xa, int64_t Xplane,
                                    const int64_t* xidx, int64_t* xe, int64_t ntiles, void* stream) {
  if (!Lw || !Xw || !Fa || !fbase || !Xa || !xidx || !xe || L < 1 || WL <= L || LF < 2 || ntiles < 0 ||
      ntiles > 0x7fffffff)
    return SDPV_EINVAL;
  if (ntiles == 0) return SDPV_OK;
  grp_tile_narrow_kernel<<<(unsigned)ntiles, 256, 0, sdpv::as_stream(stream)>>>(Lw, Xw, WL, LF, Fa, Fplane, L, e, fbase,
                                                                                  Xa, Xplane, xidx, xe);
  return sdpv::launch_status();
}
