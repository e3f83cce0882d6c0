// Step-length eigenvalues on the GPU (FP64): batched symmetric eigenvalues by cyclic Jacobi.
//
// The step length needs lambda_min of M = L^-1 dM L^-T per block (sdpvibe/solver.py:1064-1093); the
// reference takes a float64 copy of M (scaled to O(1)) to the host and calls LAPACK.  Here the copy stays
// on the device: one CTA per block, the block in shared memory, rotations in the round-robin parallel
// order (n/2 disjoint (p, q) pairs per step: rows first, then columns, then the exact 2 x 2 update of the
// pivots), sweeps until the off-diagonal mass is below (eps ||A||_F)^2 / 4 or 40 sweeps.
//
// Error bound returned with each block: a rotation applied in float64 is an exact orthogonal similarity of
// a matrix perturbed by at most a few eps ||A||_F in each of the 2 (n - 1) rotations an entry takes per
// sweep, and the final off-diagonal part moves eigenvalues by at most its Frobenius norm (Weyl):
//   err = (6 n S + n + 2) eps ||A||_F + ||off(A_final)||_F   (S sweeps),
// a larger bound than LAPACK's (n + 2) eps ||A||_F; a block it does not resolve goes to the
// multiprecision refinement, as in the reference.
#include <cmath>

#include "common.cuh"

namespace {

constexpr int kThreads = 256;
constexpr int kNmax = 128;                 // blocks up to 128 x 128 (even padded size <= 128)

__global__ void __launch_bounds__(kThreads) jacobi_kernel(const double* __restrict__ A, int n, double* __restrict__ w,
                                                          double* __restrict__ err, int* __restrict__ sweeps_out) {
  extern __shared__ __align__(16) double sa[];          // np x np, row-major
  __shared__ double red[kThreads / 32];
  __shared__ double cs[kNmax / 2], sn[kNmax / 2], tt[kNmax / 2], dp[kNmax / 2], dq[kNmax / 2];
  __shared__ int pp[kNmax / 2], qq[kNmax / 2];
  __shared__ double s_norm, s_off;
  __shared__ int s_done;
  const int np = n + (n & 1);                            // an odd size gets an inert zero row / column
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const double* Ab = A + (size_t)blockIdx.x * n * n;
  for (int e = tid; e < np * np; e += kThreads) {
    const int i = e / np, j = e % np;
    sa[e] = (i < n && j < n) ? Ab[(size_t)i * n + j] : 0.0;
  }
  __syncthreads();
  // ||A||_F
  double part = 0.0;
  for (int e = tid; e < np * np; e += kThreads) part += sa[e] * sa[e];
  for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
  if (lane == 0) red[warp] = part;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int k = 0; k < kThreads / 32; k++) t += red[k];
    s_norm = sqrt(t);
    s_done = 0;
  }
  __syncthreads();
  const double eps = 2.220446049250313e-16;              // 2^-52
  const double tol = 0.25 * (eps * s_norm) * (eps * s_norm);
  const int half = np / 2;
  int sweep = 0;
  for (; sweep < 40 && !s_done; sweep++) {
    for (int r = 0; r < np - 1; r++) {
      // round-robin pairs: position 0 fixed, positions 1..np-1 rotated by r
      if (tid < half) {
        const int a = tid, b = np - 1 - tid;
        const int p0 = a == 0 ? 0 : 1 + (a - 1 + r) % (np - 1);
        const int q0 = 1 + (b - 1 + r) % (np - 1);
        const int p = p0 < q0 ? p0 : q0, q = p0 < q0 ? q0 : p0;
        const double apq = sa[p * np + q], app = sa[p * np + p], aqq = sa[q * np + q];
        double c = 1.0, s = 0.0, t = 0.0;
        if (apq != 0.0) {
          const double theta = (aqq - app) / (2.0 * apq);
          t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(1.0 + theta * theta));
          c = 1.0 / sqrt(1.0 + t * t);
          s = t * c;
        }
        pp[tid] = p;
        qq[tid] = q;
        cs[tid] = c;
        sn[tid] = s;
        tt[tid] = t * apq;                               // the pivots move by -/+ t a_pq
        dp[tid] = app;
        dq[tid] = aqq;
      }
      __syncthreads();
      for (int e = tid; e < half * np; e += kThreads) {  // rows p, q
        const int k = e / np, col = e % np;
        const int p = pp[k], q = qq[k];
        const double c = cs[k], s = sn[k];
        const double ap = sa[p * np + col], aq = sa[q * np + col];
        sa[p * np + col] = c * ap - s * aq;
        sa[q * np + col] = s * ap + c * aq;
      }
      __syncthreads();
      for (int e = tid; e < half * np; e += kThreads) {  // columns p, q
        const int k = e / np, row = e % np;
        const int p = pp[k], q = qq[k];
        const double c = cs[k], s = sn[k];
        const double ap = sa[row * np + p], aq = sa[row * np + q];
        sa[row * np + p] = c * ap - s * aq;
        sa[row * np + q] = s * ap + c * aq;
      }
      __syncthreads();
      if (tid < half && sn[tid] != 0.0) {                // the rotated 2 x 2 block exactly
        const int p = pp[tid], q = qq[tid];
        sa[p * np + p] = dp[tid] - tt[tid];
        sa[q * np + q] = dq[tid] + tt[tid];
        sa[p * np + q] = 0.0;
        sa[q * np + p] = 0.0;
      }
      __syncthreads();
    }
    // off-diagonal mass
    double off = 0.0;
    for (int e = tid; e < np * np; e += kThreads) {
      const int i = e / np, j = e % np;
      if (i != j) off += sa[e] * sa[e];
    }
    for (int o = 16; o; o >>= 1) off += __shfl_xor_sync(0xffffffffu, off, o);
    if (lane == 0) red[warp] = off;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
      for (int k = 0; k < kThreads / 32; k++) t += red[k];
      s_off = t;
      s_done = t <= tol;
    }
    __syncthreads();
  }
  // eigenvalues: the diagonal (without the inert padding entry), ascending by rank
  for (int i = tid; i < n; i += kThreads) {
    const double v = sa[i * np + i];
    int rank = 0;
    for (int j = 0; j < n; j++) {
      const double u = sa[j * np + j];
      rank += (u < v) || (u == v && j < i);
    }
    w[(size_t)blockIdx.x * n + rank] = v;
  }
  if (tid == 0) {
    err[blockIdx.x] = (6.0 * n * sweep + n + 2) * eps * s_norm + sqrt(s_off);
    if (sweeps_out) sweeps_out[blockIdx.x] = sweep;
  }
}

}  // namespace

extern "C" int sdpv_eig_sym_f64(const double* A, int64_t nb, int n, double* w, double* err, int* sweeps, void* stream) {
  if (nb < 0 || n < 1 || n > kNmax || nb > 0x7fffffff) return SDPV_EINVAL;
  if (nb == 0) return SDPV_OK;
  const int np = n + (n & 1);
  const size_t smem = (size_t)np * np * sizeof(double);
  static bool attr[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!attr[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(jacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)(kNmax * kNmax * sizeof(double)));
    if (e != cudaSuccess) return sdpv::set_cuda_error(e);
    attr[dev & 63] = true;
  }
  jacobi_kernel<<<(unsigned)nb, kThreads, smem, sdpv::as_stream(stream)>>>(A, n, w, err, sweeps);
  return sdpv::launch_status();
}
