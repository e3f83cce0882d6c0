// Launch-shape knobs of the kernels, set by the offline autotuner's table (sdpvibe_b200/autotune.py) or left
// at their defaults.  They change how work is cut into launches and items, never the results: every
// choice computes the same exact residues and rounds at the same points.
#include <atomic>

#include "common.cuh"

namespace {
// defaults: CRT CTAs per SM, narrow-item limit of the short side, block-packing limit, decomposition
// reducer warps, moduli group of the Python layer's contexts
std::atomic<int> g_knob[SDPV_TUNE_COUNT] = {{3}, {64}, {64}, {8}, {16}};
constexpr int kLo[SDPV_TUNE_COUNT] = {1, 0, 0, 8, 1};
constexpr int kHi[SDPV_TUNE_COUNT] = {4, 64, 64, 16, 16};
}  // namespace

namespace sdpv {
int tune(int knob) { return g_knob[knob].load(std::memory_order_relaxed); }
}  // namespace sdpv

extern "C" int sdpv_tune_set(int knob, int value) {
  if (knob < 0 || knob >= SDPV_TUNE_COUNT || value < kLo[knob] || value > kHi[knob]) return SDPV_EINVAL;
  if ((knob == SDPV_TUNE_NARROW_MAX || knob == SDPV_TUNE_PACK_MAX) && value % 16) return SDPV_EINVAL;
  if (knob == SDPV_TUNE_RES_WARPS && value % 8) return SDPV_EINVAL;
  if (knob == SDPV_TUNE_MOD_GROUP && (value & (value - 1))) return SDPV_EINVAL;
  g_knob[knob].store(value, std::memory_order_relaxed);
  return SDPV_OK;
}

extern "C" int sdpv_tune_get(int knob, int* value) {
  if (knob < 0 || knob >= SDPV_TUNE_COUNT || !value) return SDPV_EINVAL;
  *value = g_knob[knob].load(std::memory_order_relaxed);
  return SDPV_OK;
}
