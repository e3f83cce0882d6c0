// Device error word and CUDA error bookkeeping.
#include <cstdio>
#include <cstring>
#include <mutex>

#include "common.cuh"

// One word per device that loads the library; kernels OR SDPV_ERRBIT_* into it.
__device__ unsigned g_sdpv_error_word;

namespace {
thread_local char g_last[512] = "";
constexpr int kMaxDev = 64;
unsigned* g_word_ptr[kMaxDev] = {};
std::mutex g_mu;
}  // namespace

namespace sdpv {

int set_cuda_error(cudaError_t e) {
  snprintf(g_last, sizeof(g_last), "%s: %s", cudaGetErrorName(e), cudaGetErrorString(e));
  return SDPV_ECUDA;
}

void set_message(const char* msg) { snprintf(g_last, sizeof(g_last), "%s", msg); }

unsigned* device_error_word() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= kMaxDev) return nullptr;
  std::lock_guard<std::mutex> g(g_mu);
  if (!g_word_ptr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_sdpv_error_word) != cudaSuccess) return nullptr;
    g_word_ptr[dev] = (unsigned*)p;
  }
  return g_word_ptr[dev];
}

EncodeTiledFn encode_tiled_fn() {
  static EncodeTiledFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (EncodeTiledFn)p;
  });
  return fn;
}

}  // namespace sdpv

extern "C" const char* sdpv_last_error(void) { return g_last; }

extern "C" int sdpv_get_error(unsigned* flags_host, void* stream) {
  if (!flags_host) return SDPV_EINVAL;
  unsigned* w = sdpv::device_error_word();
  if (!w) return SDPV_ECUDA;
  cudaStream_t s = sdpv::as_stream(stream);
  unsigned v = 0;
  cudaError_t e = cudaMemcpyAsync(&v, w, sizeof(v), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e == cudaSuccess && v) e = cudaMemsetAsync(w, 0, sizeof(unsigned), s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return sdpv::set_cuda_error(e);
  *flags_host = v;
  return SDPV_OK;
}

extern "C" int sdpv_device_status(void* stream) {
  unsigned v = 0;
  int st = sdpv_get_error(&v, stream);
  if (st != SDPV_OK) return st;
  if (v & SDPV_ERRBIT_TIMEOUT) return SDPV_ETIMEOUT;
  if (v & SDPV_ERRBIT_NOTSPD) return SDPV_ENOTSPD;
  if (v & SDPV_ERRBIT_OVERFLOW) return SDPV_EOVERFLOW;
  return SDPV_OK;
}

namespace {
// One warp waits on a shared-memory mbarrier expecting one arrival, with the pipelines' bounded wait
// shortened to limit_ns.  With arrive set lane 0 arrives first and the wait succeeds at once; without it
// nothing ever arrives, the wait gives up after limit_ns, sets the timeout bit and the kernel returns.
__global__ void wait_probe_kernel(u64 limit_ns, int arrive, unsigned* err) {
  __shared__ __align__(8) u64 bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_fence_init();
  }
  __syncwarp();
  if (arrive && threadIdx.x == 0) mbar_arrive(&bar);
  __syncwarp();
  if (threadIdx.x == 0) mbar_wait_ns(&bar, 0, err, limit_ns);
}
}  // namespace

extern "C" int sdpv_wait_probe(unsigned limit_us, int arrive, void* stream) {
  if (limit_us == 0 || limit_us > 2000000u) return SDPV_EINVAL;
  unsigned* err = sdpv::device_error_word();
  if (!err) return SDPV_ECUDA;
  wait_probe_kernel<<<1, 32, 0, sdpv::as_stream(stream)>>>((u64)limit_us * 1000ull, arrive, err);
  return sdpv::launch_status();
}
