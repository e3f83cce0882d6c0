// Host-side stand-ins for the CUDA built-ins used by SDPviBe's run-time-compiled kernel strings
// (sdpvibe/mpf.py:23-141 and sdpvibe/basecase.py:13-246), so that those strings compile with g++
// and run on the CPU as a checker.  TEST INFRASTRUCTURE ONLY: nothing in the product links this.
//
// Execution model: one thread block at a time.  Kernels that never synchronise run their threads
// serially; kernels that use __syncthreads/__syncwarp run one std::thread per CUDA thread, with a
// block-wide barrier and one barrier per warp, so `__shared__` (function-static here) is shared by
// the block exactly as on the GPU.
#pragma once
#include <algorithm>
#include <barrier>
#include <cmath>
#include <cstdint>
#include <cstddef>
#include <functional>
#include <memory>
#include <thread>
#include <vector>

struct sdpvref_dim { unsigned x = 0, y = 0, z = 0; };
inline thread_local sdpvref_dim threadIdx;
inline thread_local sdpvref_dim blockIdx;
inline sdpvref_dim blockDim;
inline sdpvref_dim gridDim;

#define __device__
#define __global__
#define __forceinline__ inline
#define __shared__ static

using std::max;
using std::min;

static inline int __clz(unsigned x) { return x ? __builtin_clz(x) : 32; }

struct sdpvref_block_sync {
  std::unique_ptr<std::barrier<>> block;
  std::vector<std::unique_ptr<std::barrier<>>> warps;
};
inline sdpvref_block_sync* sdpvref_sync = nullptr;

static inline void __syncthreads() { sdpvref_sync->block->arrive_and_wait(); }
static inline void __syncwarp() { sdpvref_sync->warps[threadIdx.x / 32]->arrive_and_wait(); }

// Run `body` for every thread of every block of a 1-D launch.
inline void sdpvref_run(unsigned grid, unsigned block, bool cooperative, const std::function<void()>& body) {
  gridDim.x = grid;
  blockDim.x = block;
  if (!cooperative) {
    for (unsigned b = 0; b < grid; b++)
      for (unsigned t = 0; t < block; t++) {
        blockIdx.x = b;
        threadIdx.x = t;
        body();
      }
    return;
  }
  for (unsigned b = 0; b < grid; b++) {
    sdpvref_block_sync s;
    s.block = std::make_unique<std::barrier<>>(block);
    for (unsigned w = 0; w < (block + 31) / 32; w++) {
      unsigned n = std::min(32u, block - 32 * w);
      s.warps.push_back(std::make_unique<std::barrier<>>(n));
    }
    sdpvref_sync = &s;
    std::vector<std::thread> th;
    th.reserve(block);
    for (unsigned t = 0; t < block; t++)
      th.emplace_back([&, b, t] {
        blockIdx.x = b;
        threadIdx.x = t;
        body();
      });
    for (auto& x : th) x.join();
    sdpvref_sync = nullptr;
  }
}
