// Tuning table lookup and the process-wide override used by the tuner.
#include "tuning.h"

#include <atomic>
#include <cmath>
#include <cstdlib>
#include <mutex>

#include "tuning_table.h"
#include "util.h"

namespace b200nufft {

namespace {

std::mutex g_override_mutex;
bool g_override_set = false;
b200nufft_tuning g_override{};
std::atomic<bool> g_fused_transforms{true};

int floor_log2(double v) { return v > 0.0 ? static_cast<int>(std::floor(std::log2(v))) : -16; }

}  // namespace

TuningKey tuning_key(int type, int dimensions, int precision, int width, int64_t fine_cells, int64_t points) {
  TuningKey k{};
  k.type = type;
  k.dimensions = dimensions;
  k.precision = precision;
  k.width = width;
  k.log2_cells = floor_log2(static_cast<double>(fine_cells));
  const double density = static_cast<double>(points > 0 ? points : 1) / static_cast<double>(fine_cells > 0 ? fine_cells : 1);
  int d = floor_log2(density);
  k.log2_density = d < -16 ? -16 : (d > 16 ? 16 : d);
  return k;
}

b200nufft_tuning default_tuning(int dimensions) {
  b200nufft_tuning t{};
  (void)dimensions;
  t.tile = 0;  // the plan's own default for its precision and width
  t.ctas_per_sm = 4;
  t.crowded_ctas_per_sm = 1;
  t.tensor_min_batch = 16;
  return t;
}

b200nufft_tuning tuning_for(const TuningKey& key) {
  b200nufft_tuning t = default_tuning(key.dimensions);
  int best = -1;
  int best_distance = 1 << 30;
  for (int i = 0; i < kTuningEntries; ++i) {
    const TuningEntry& e = kTuningTable[i];
    if (e.type != key.type || e.dimensions != key.dimensions || e.precision != key.precision || e.width != key.width) {
      continue;
    }
    const int distance = 4 * std::abs(e.log2_cells - key.log2_cells) + std::abs(e.log2_density - key.log2_density);
    if (distance < best_distance) {
      best_distance = distance;
      best = i;
    }
  }
  if (best >= 0) {
    const TuningEntry& e = kTuningTable[best];
    t.tile = e.tile;
    t.ctas_per_sm = e.ctas_per_sm;
    t.crowded_ctas_per_sm = e.crowded_ctas_per_sm;
    t.tensor_min_batch = e.tensor_min_batch;
  }
  std::lock_guard<std::mutex> lock(g_override_mutex);
  if (g_override_set) {
    if (g_override.tile > 0) t.tile = g_override.tile;
    if (g_override.ctas_per_sm > 0) t.ctas_per_sm = g_override.ctas_per_sm;
    if (g_override.crowded_ctas_per_sm > 0) t.crowded_ctas_per_sm = g_override.crowded_ctas_per_sm;
    if (g_override.tensor_min_batch > 0) t.tensor_min_batch = g_override.tensor_min_batch;
  }
  return t;
}

bool fused_fft_enabled() { return b200nufft::g_fused_transforms.load(); }

}  // namespace b200nufft

extern "C" int b200nufft_set_fused_transforms(int enable) {
  b200nufft::g_fused_transforms.store(enable != 0);
  return B200NUFFT_SUCCESS;
}

extern "C" int b200nufft_tuning_override(const b200nufft_tuning* tuning) {
  std::lock_guard<std::mutex> lock(b200nufft::g_override_mutex);
  if (tuning == nullptr) {
    b200nufft::g_override_set = false;
    return B200NUFFT_SUCCESS;
  }
  if (tuning->tile < 0 || tuning->ctas_per_sm < 0 || tuning->crowded_ctas_per_sm < 0 || tuning->tensor_min_batch < 0 ||
      (tuning->tile > 0 && (tuning->tile & (tuning->tile - 1)) != 0)) {
    b200nufft::set_last_error("tuning fields must be non-negative and the tile side a power of two");
    return B200NUFFT_INVALID_ARGUMENT;
  }
  b200nufft::g_override = *tuning;
  b200nufft::g_override_set = true;
  return B200NUFFT_SUCCESS;
}

extern "C" int b200nufft_tuning_lookup(int32_t type, int32_t dimensions, int32_t precision, int32_t width,
                                       int64_t fine_cells, int64_t point_count, b200nufft_tuning* out) {
  if (out == nullptr) {
    b200nufft::set_last_error("null output");
    return B200NUFFT_INVALID_ARGUMENT;
  }
  *out = b200nufft::tuning_for(
      b200nufft::tuning_key(type, dimensions, precision, width, fine_cells, point_count));
  return B200NUFFT_SUCCESS;
}
