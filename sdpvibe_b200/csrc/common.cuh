// Shared device/host helpers for the sm_100a kernels of libsdpv_b200.
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/sdpv_b200.h"

typedef uint32_t u32;
typedef uint64_t u64;
typedef int64_t i64;

#define SDPV_EZ (-(1LL << 40))  // exponent of zero (sdpvibe/mpf.py:21)

// ------------------------------------------------------------------ host side
namespace sdpv {

int set_cuda_error(cudaError_t e);         // records the text, returns SDPV_ECUDA
void set_message(const char* msg);         // records a diagnostic for sdpv_last_error
unsigned* device_error_word();             // this device's error word (no allocation)
int tune(int knob);                        // launch-shape knob (SDPV_TUNE_*), see tuning.cu
inline int launch_status() {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SDPV_OK : set_cuda_error(e);
}
inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }
// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link dependency).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn encode_tiled_fn();

// Device-side RNS tables of one limb count (see ctx.cu).
struct CtxDev {
  int L, n, E, W;
  int npad;          // moduli rounded up to 128 (MMA M of the decomposition)
  int kt;            // 128-byte K tiles of the byte-by-table product (ceil(4L/128))
  int npad16;        // moduli rounded up to 32 bytes (K of the CRT digit product, in 128-byte tiles)
  int Epad;          // CRT digits rounded up to 128 (N chunks of the digit product)
  int32_t* mods;     // (n)
  float* minv;       // (n) float(1/m)
  int32_t* c14;      // (n) 2^14 mod m
  int32_t* c1;       // (n) C1 (sdpvibe/rns.py:183)
  int32_t* c1m2;     // (n) C1 - C2 (top limb negative)
  int32_t* inv;      // (n) (M/m)^-1 mod m
  int32_t* md;       // (Epad) signed base-256 digits of M, zero padded
  uint8_t* tab;      // decomposition tables as swizzled SMEM images: [group][lo|hi][kt][128 rows][128 B]
  uint8_t* tabu;     // the same layout with unsigned digits of the canonical 256^j mod m (hi = t >> 7,
                     // lo = t & 127) and column 4L = (-2^(32L)) mod m against the sign byte
  uint8_t* ct;       // CRT digit table as swizzled SMEM images: [chunk][ktc][128 rows][128 B]
  int ktc;           // 128-byte K tiles of the CRT product (ceil(n/128))
};

}  // namespace sdpv

struct sdpv_ctx {
  sdpv::CtxDev d;
  int device;
  int32_t* mods_host;
};

// ------------------------------------------------------------------ device side
#define SDPV_WAIT_NS 2000000000ull  // a pipeline wait gives up after 2 s of wall-clock time

__device__ __forceinline__ u32 smem_u32(const void* p) { return (u32)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(u64* bar, u32 count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(u64* bar, u32 bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(u64* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(u64* bar, u32 phase) {
  u32 ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ u64 globaltimer_ns() {
  u64 t;
  asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait for the given phase parity; after limit_ns of wall-clock time it gives up, sets the
// timeout bit and returns false.
__device__ __forceinline__ bool mbar_wait_ns(u64* bar, u32 phase, unsigned* err, u64 limit_ns) {
  if (mbar_try_wait(bar, phase)) return true;
  const u64 t0 = globaltimer_ns();
  for (u32 it = 1;; it++) {
    if (mbar_try_wait(bar, phase)) return true;
    if ((it & 1023u) == 0 && globaltimer_ns() - t0 > limit_ns) break;
  }
  atomicOr(err, SDPV_ERRBIT_TIMEOUT);
  return false;
}
// The pipelines' wait: gives up after SDPV_WAIT_NS.
__device__ __forceinline__ bool mbar_wait(u64* bar, u32 phase, unsigned* err) {
  return mbar_wait_ns(bar, phase, err, SDPV_WAIT_NS);
}

__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// TMA: 4-D tiled load into shared memory, completion counted on an mbarrier.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, u64* bar, int c0, int c1, int c2,
                                            int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5, %6}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
      : "memory");
}
// Non-tensor bulk copy global -> shared (16-byte aligned addresses, size multiple of 16).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, u32 bytes, u64* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// ---- asynchronous global -> shared copies (no register round trip), grouped for multi-stage pipelines
// 4-byte copy; src_bytes = 0 writes zeros (used for out-of-range entries).
__device__ __forceinline__ void cp_async4(void* dst, const void* src, u32 src_bytes) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
               : "memory");
}
// 16-byte copy (both addresses 16-byte aligned); the bytes past src_bytes are written as zeros.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, u32 src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// TMA: 2-D tiled load into shared memory, completion counted on an mbarrier.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, u64* bar, int c0, int c1) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
      : "memory");
}
// TMA: 3-D tiled load into shared memory, completion counted on an mbarrier.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, u64* bar, int c0, int c1, int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], "
      "[%2];" ::"r"(smem_u32(dst)),
      "l"(map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2)
      : "memory");
}
// 3-D tiled store shared -> global (bulk-group completion).
__device__ __forceinline__ void tma_store_3d(const CUtensorMap* map, const void* src, int c0, int c1, int c2) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%2, %3, %4}], [%1];" ::"l"(map),
               "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2)
               : "memory");
}

// ---- TMA bulk tensor store shared -> global (2-D), bulk-group completion tracking
__device__ __forceinline__ void tma_store_2d(const CUtensorMap* map, const void* src, int c0, int c1) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%2, %3}], [%1];" ::"l"(map),
               "r"(smem_u32(src)), "r"(c0), "r"(c1)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bulk_wait_read() {   // smem sources of all but N groups may be reused
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
template <int N>
__device__ __forceinline__ void bulk_wait() {        // all but N groups complete
  asm volatile("cp.async.bulk.wait_group %0;" ::"n"(N) : "memory");
}

// ---- tcgen05 (5th-generation tensor cores, TMEM accumulators)
__device__ __forceinline__ void tmem_alloc(u32* dst_smem, u32 ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
               "r"(ncols));
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(u32 taddr, u32 ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, int8 x int8 -> int32, issued by one thread.
__device__ __forceinline__ void mma_i8(u32 tmem_d, u64 adesc, u64 bdesc, u32 idesc, u32 accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}
// Arrive on an mbarrier once all previously issued tcgen05.mma of this thread have completed.
__device__ __forceinline__ void mma_commit(u64* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Instruction descriptor: signed int8 A and B, int32 accumulator, both K-major, shape M x N.
__host__ __device__ constexpr u32 idesc_i8(int M, int N) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((u32)(N >> 3) << 17) | ((u32)(M >> 4) << 24);
}
// The same with unsigned 8-bit A and B (digit formats 0).
__host__ __device__ constexpr u32 idesc_u8(int M, int N) {
  return (2u << 4) | ((u32)(N >> 3) << 17) | ((u32)(M >> 4) << 24);
}
// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 bytes apart.
__device__ __forceinline__ u64 sdesc_sw128(u32 smem_addr) {
  u64 d = 0;
  d |= (u64)((smem_addr & 0x3FFFF) >> 4);       // start address
  d |= (u64)1 << 16;                            // leading byte offset (unused for swizzled K-major)
  d |= (u64)(1024 >> 4) << 32;                  // stride byte offset
  d |= (u64)1 << 46;                            // descriptor version (sm_100)
  d |= (u64)2 << 61;                            // SWIZZLE_128B
  return d;
}

// The same for K-major rows of rb = 32, 64 or 128 bytes (32-, 64- or 128-byte swizzle; 8-row groups 8 rb
// bytes apart).
__device__ __forceinline__ u64 sdesc_sw(u32 smem_addr, int rb) {
  u64 d = 0;
  d |= (u64)((smem_addr & 0x3FFFF) >> 4);
  d |= (u64)1 << 16;
  d |= (u64)((8 * rb) >> 4) << 32;
  d |= (u64)1 << 46;
  d |= (u64)(rb == 32 ? 6 : rb == 64 ? 4 : 2) << 61;
  return d;
}

// 32 lanes x 32 consecutive 32-bit columns (this warp's lane quarter) into registers.
__device__ __forceinline__ void tmem_ld32(u32 taddr, u32 (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]),
        "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
}
// 32 lanes x 16 consecutive 32-bit columns.
__device__ __forceinline__ void tmem_ld16(u32 taddr, u32 (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, "
      "[%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Byte offset of (row, 16-byte chunk) inside a K-major SWIZZLE_128B tile of 128-byte rows.
__host__ __device__ __forceinline__ u32 sw128_off(u32 row, u32 chunk) {
  return row * 128u + ((chunk ^ (row & 7u)) << 4);
}

// Exact x mod m in [0, m) for |x| < 2^31 and 2 < m < 2^15, with minv = float(1/m).
__device__ __forceinline__ int mod_exact(int x, int m, float minv) {
  int q = __float2int_rd(__int2float_rn(x) * minv);
  int r = x - q * m;
  r += (r < 0) ? m : 0;
  r -= (r >= m) ? m : 0;
  return r;
}
