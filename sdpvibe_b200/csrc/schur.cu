// Schur-complement assembly of one chunk in one launch (sdpvibe/solver.py:634-652).
//
// From the pairings AXI = V^T X^-1 V and AY = V^T Y V of both parities ((2 nb, W, W), W = dim K) the
// reference composes S (nb, P, P), P = K dim (dim + 1) / 2, out of elementwise MPF products and sums over
// K x K sub-blocks.  Here one thread makes one lower entry (b, i, j) of S with the same operations in the
// same order:
//   dim 1:   S = AXI_0 AY_0 + AXI_1 AY_1                       (parities 0, 1: the fold)
//   dim > 1: row i in pair segment s_i = (c0, r0) at offset a, column j in s_j = (c1, r1) at offset bb
//            (segment s = c (c + 1) / 2 + r, pairs c >= r); per parity, with A = AXI, Y = AY and
//            [u, v] the entry (u K + a, v K + bb) of a pairing block:
//              el = ((A[c0,r1] Y[r0,c1] + A[r0,r1] Y[c0,c1]) + A[c0,c1] Y[r0,r1]) + A[r0,c1] Y[c0,r1]
//            then S = (el_0 + el_1) 2^-2
// each product and sum rounded as mpf_mul / mpf_add, so S is the composed result bit for bit; S is written
// at (i, j) and (j, i) (the reference copies its lower triangle up), and the diagonal entry of a padding
// row (xmask false) is set to one.
#include <cmath>

#include "common.cuh"
#include "mpcore.cuh"

namespace {
using namespace sdpv;

constexpr int kThreads = 128;

__device__ __forceinline__ void seg_of(int s, int& c, int& r) {
  c = 0;
  while ((c + 1) * (c + 2) / 2 <= s) c++;
  r = s - c * (c + 1) / 2;
}

template <int LMAX>
__device__ __forceinline__ void load_entry(const int32_t* __restrict__ M, const i64* __restrict__ eM, i64 plane,
                                           i64 idx, int L, u32* w, i64& e) {
  for (int k = 0; k < L; k++) w[k] = (u32)__ldg(M + (i64)k * plane + idx);
  e = __ldg(eM + idx);
}

template <int LMAX>
__global__ void __launch_bounds__(kThreads)
    schur_kernel(int L, i64 nb, int P, int K, int dim, const int32_t* __restrict__ A, const i64* __restrict__ eA,
                 const int32_t* __restrict__ Y, const i64* __restrict__ eY, const uint8_t* __restrict__ xmask,
                 const int32_t* __restrict__ onem, i64 onee, int32_t* __restrict__ S, i64* __restrict__ eS) {
  const i64 ntri = (i64)P * (P + 1) / 2;
  const i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nb * ntri) return;
  const i64 b = t / ntri;
  const int q = (int)(t - b * ntri);
  int i = (int)((sqrt(8.0 * q + 1.0) - 1.0) * 0.5);                // lower entry q -> (i, j), j <= i
  while ((i + 1) * (i + 2) / 2 <= q) i++;
  while (i * (i + 1) / 2 > q) i--;
  const int j = q - i * (i + 1) / 2;
  const int W = dim * K;
  const i64 plane = 2 * nb * (i64)W * W, splane = nb * (i64)P * P;
  u32 r[LMAX];
  i64 er;
  if (i == j && !xmask[b * P + i]) {
    for (int k = 0; k < L; k++) r[k] = (u32)onem[k];
    er = onee;
  } else if (dim == 1) {
    u32 x[LMAX], y[LMAX], m[2][LMAX];
    i64 ex, ey, em[2];
    for (int p = 0; p < 2; p++) {
      const i64 idx = ((p * nb + b) * W + i) * W + j;
      load_entry<LMAX>(A, eA, plane, idx, L, x, ex);
      load_entry<LMAX>(Y, eY, plane, idx, L, y, ey);
      mpf_mul_dev<LMAX>(x, ex, y, ey, L, m[p], em[p]);
    }
    mpf_add_dev<LMAX>(m[0], em[0], m[1], em[1], 1, L, r, er);
  } else {
    const int si = i / K, a = i - si * K, sj = j / K, bb = j - sj * K;
    int c0, r0, c1, r1;
    seg_of(si, c0, r0);
    seg_of(sj, c1, r1);
    u32 el[2][LMAX], x[LMAX], y[LMAX], tt[LMAX];
    i64 ee[2], ex, ey, et;
    for (int p = 0; p < 2; p++) {
      const i64 base = (p * nb + b) * (i64)W;
      // A[u, v] Y[w, z]: entry (u K + a, v K + bb) of AXI times entry (w K + a, z K + bb) of AY
      auto term = [&](int u, int v, int w, int z, u32* out, i64& eo) {
        load_entry<LMAX>(A, eA, plane, (base + u * K + a) * W + v * K + bb, L, x, ex);
        load_entry<LMAX>(Y, eY, plane, (base + w * K + a) * W + z * K + bb, L, y, ey);
        mpf_mul_dev<LMAX>(x, ex, y, ey, L, out, eo);
      };
      term(c0, r1, r0, c1, el[p], ee[p]);
      term(r0, r1, c0, c1, tt, et);
      mpf_add_dev<LMAX>(el[p], ee[p], tt, et, 1, L, el[p], ee[p]);
      term(c0, c1, r0, r1, tt, et);
      mpf_add_dev<LMAX>(el[p], ee[p], tt, et, 1, L, el[p], ee[p]);
      term(r0, c1, c0, r1, tt, et);
      mpf_add_dev<LMAX>(el[p], ee[p], tt, et, 1, L, el[p], ee[p]);
    }
    mpf_add_dev<LMAX>(el[0], ee[0], el[1], ee[1], 1, L, r, er);
    if (er != SDPV_EZ) er -= 2;
  }
  const i64 o1 = (b * P + i) * (i64)P + j, o2 = (b * P + j) * (i64)P + i;
  for (int k = 0; k < L; k++) {
    S[(i64)k * splane + o1] = (int32_t)r[k];
    S[(i64)k * splane + o2] = (int32_t)r[k];
  }
  eS[o1] = er;
  eS[o2] = er;
}

}  // namespace

extern "C" int sdpv_schur_assemble(int L, int64_t nb, int P, int K, int dim, const int32_t* AXI, const int64_t* eAXI,
                                   const int32_t* AY, const int64_t* eAY, const uint8_t* xmask, const int32_t* one_m,
                                   int64_t one_e, int32_t* S, int64_t* eS, void* stream) {
  if (L < 1 || L > 64 || nb < 0 || K < 1 || dim < 1 || P != K * dim * (dim + 1) / 2) return SDPV_EINVAL;
  const i64 n = nb * (i64)P * (P + 1) / 2;
  if (n == 0) return SDPV_OK;
  const unsigned grid = (unsigned)((n + kThreads - 1) / kThreads);
  cudaStream_t st = sdpv::as_stream(stream);
  if (L <= 16)
    schur_kernel<16><<<grid, kThreads, 0, st>>>(L, nb, P, K, dim, AXI, eAXI, AY, eAY, xmask, one_m, one_e, S, eS);
  else if (L <= 32)
    schur_kernel<32><<<grid, kThreads, 0, st>>>(L, nb, P, K, dim, AXI, eAXI, AY, eAY, xmask, one_m, one_e, S, eS);
  else
    schur_kernel<64><<<grid, kThreads, 0, st>>>(L, nb, P, K, dim, AXI, eAXI, AY, eAY, xmask, one_m, one_e, S, eS);
  return sdpv::launch_status();
}
