// Column bookkeeping of the Gram accumulation (GramAcc.add, sdpvibe/mpf.py:556-579), one launch per chunk.
//
// Per column j, with the chunk's column top tp_j (sdpv_top_max; EZ for an all-zero column) and the running
// reference exponent E_j (EZ until the column has been seen):
//   live_j = tp_j > EZ/2,  known_j = E_j > EZ/2,  Tmax_j = max(Tmax_j, tp_j)
//   f = any_j (live_j and known_j and tp_j > E_j + HEAD)          (the partial sum must be flushed first)
//   rE_j = known_j ? E_j - NB : 0                                   (the flush's CRT exponents, old E)
//   E_j = (f and live_j and tp_j > E_j) ? tp_j : E_j;  then E_j = (live_j and E_j unknown) ? tp_j : E_j
//   target_j = E_j - NB                                             (the chunk's alignment exponents)
// and the flush count += f when the accumulator holds data.  One CTA; the any() is a block-wide OR.  The
// predicate f stays on the device: the flush (sdpv_crt_norm_if, sdpv_mpf_add_if, sdpv_zero_if) reads it,
// so the accumulation has no host decision and replays as one CUDA graph.
#include "common.cuh"

namespace {

constexpr int kThreads = 512;

__global__ void __launch_bounds__(kThreads) gram_columns_kernel(i64 N, const i64* __restrict__ tp, i64* __restrict__ E,
                                                                i64* __restrict__ Tmax, i64 head, i64 nbits,
                                                                int has_acc, i64* __restrict__ rE_old,
                                                                i64* __restrict__ target, int32_t* __restrict__ f_out,
                                                                i64* __restrict__ nflush) {
  const i64 half = SDPV_EZ / 2;
  bool flush = false;
  for (i64 j = threadIdx.x; j < N; j += kThreads) {
    const i64 t = tp[j], e = E[j];
    flush = flush || (t > half && e > half && t > e + head);
  }
  const bool f = __syncthreads_or(flush) != 0;
  for (i64 j = threadIdx.x; j < N; j += kThreads) {
    const i64 t = tp[j];
    i64 e = E[j];
    const bool live = t > half;
    if (t > Tmax[j]) Tmax[j] = t;
    rE_old[j] = e > half ? e - nbits : 0;
    if (f && live && t > e) e = t;
    if (live && !(e > half)) e = t;
    E[j] = e;
    target[j] = e - nbits;
  }
  if (threadIdx.x == 0) {
    *f_out = f ? 1 : 0;
    if (has_acc && f) *nflush += 1;
  }
}

__global__ void zero_if_kernel(uint4* __restrict__ p, i64 n16, const int32_t* __restrict__ pred) {
  if (*pred == 0) return;
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < n16; i += (i64)gridDim.x * blockDim.x)
    p[i] = make_uint4(0u, 0u, 0u, 0u);
}

}  // namespace

extern "C" int sdpv_gram_columns(int64_t N, const int64_t* tp, int64_t* E, int64_t* Tmax, int64_t head,
                                 int64_t nbits, int has_acc, int64_t* rE_old, int64_t* target, int32_t* f,
                                 int64_t* nflush, void* stream) {
  if (N < 0 || !tp || !E || !Tmax || !rE_old || !target || !f || !nflush) return SDPV_EINVAL;
  gram_columns_kernel<<<1, kThreads, 0, sdpv::as_stream(stream)>>>(N, tp, E, Tmax, head, nbits, has_acc, rE_old,
                                                                    target, f, nflush);
  return sdpv::launch_status();
}

extern "C" int sdpv_zero_if(void* p, int64_t nbytes, const int32_t* pred, void* stream) {
  if (!p || !pred || nbytes < 0 || (nbytes & 15) || (((uintptr_t)p) & 15)) return SDPV_EINVAL;
  if (nbytes == 0) return SDPV_OK;
  const i64 n16 = nbytes / 16;
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  i64 blocks = (n16 + 255) / 256;
  if (blocks > 4 * sms) blocks = 4 * sms;
  zero_if_kernel<<<(unsigned)blocks, 256, 0, sdpv::as_stream(stream)>>>(reinterpret_cast<uint4*>(p), n16, pred);
  return sdpv::launch_status();
}
