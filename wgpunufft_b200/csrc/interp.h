// Host interface of the type-2 interpolation kernels (interp.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device.h"

namespace b200nufft {

struct InterpLaunch {
  const float* points;    // coordinates in bin (slot) order
  const void* windows;    // PreparedWindow per slot
  int64_t point_count;
  const uint32_t* perm;   // slot -> original point, in bin order
  const float2* fine;     // batch * fine_count
  int batch;
  float2* output;         // batch * point_count, input order
};

struct InterpLaunch64 {
  const double* points;   // coordinates in bin (slot) order
  int64_t point_count;
  const uint32_t* perm;
  const double2* fine;
  int batch;
  double2* output;
};

void interpolate_execute(const GridParams& g, const InterpLaunch& launch, cudaStream_t stream);

// Work items of the 2D bin interpolation kernels: the slots of every bin in
// parts of at most kInterpPartSlots, so that a bin holding many points
// (clustered points) is served by many CTAs instead of one. part_bin[p] is
// the bin of part p, part_start[b] the first part of bin b (bins + 1 words,
// the last one the number of parts).
constexpr uint32_t kInterpPartSlots = 512;
struct InterpParts {
  const uint32_t* part_bin;
  const uint32_t* part_start;
  int64_t upper_bound;  // launch width, at least the number of parts
};
// Launch width for `count` points in `bins` bins: every non-empty bin has at
// most n / kInterpPartSlots + 1 parts.
inline int64_t interp_parts_bound(int64_t count, uint64_t bins) {
  const int64_t nonempty = count < static_cast<int64_t>(bins) ? count : static_cast<int64_t>(bins);
  return nonempty + count / kInterpPartSlots + 1;
}
// parts: bins words of scratch; part_start: bins + 1 words; part_bin:
// interp_parts_bound(count, bins) words.
void interp_bin_parts(const uint32_t* offsets, uint64_t bins, uint32_t* parts, uint32_t* part_start,
                      uint32_t* part_bin, cudaStream_t stream);

// Batched 2D f32 interpolation over the type-2 bins (8 x 8 cells): the
// reachable fine-grid region of a bin is staged in shared memory for 32
// vectors at a time. Same values, bit for bit, as interpolate_execute.
struct InterpBinsLaunch {
  const void* windows;      // PreparedWindow per slot
  int64_t point_count;
  const uint32_t* perm;
  const uint32_t* offsets;  // bins + 1 slot offsets
  uint64_t bins;
  const float2* fine;
  int batch;
  float2* output;
  const uint32_t* inverse;  // slot of every point
  float2* staged;           // point_count x round_up(batch, 32), slot order
  InterpParts parts;
};
bool interpolate_bins_supported(const GridParams& g);
void interpolate_bins_execute(const GridParams& g, const InterpBinsLaunch& launch, cudaStream_t stream);
// Small batches: one CTA per bin, the bin's grid region staged in shared
// memory, outputs written in point order (inverse and staged unused).
void interpolate_region_execute(const GridParams& g, const InterpBinsLaunch& launch, cudaStream_t stream);
void interpolate_execute64(const GridParams& g, const InterpLaunch64& launch, cudaStream_t stream);
// output[b][i] = staged[inverse[i] * stride + b] for b < batch, i < count.
void unpermute_values(const float2* staged, int64_t stride, const uint32_t* inverse, int64_t count, int batch,
                      float2* output, cudaStream_t stream);
// 2D f64 plans on 4 x 4-cell bins: each bin's grid region staged in shared
// memory (same sums, bit for bit, as interpolate_execute64).
bool interpolate_region64_supported(const GridParams& g);
void interpolate_region64_execute(const GridParams& g, const InterpLaunch64& launch, const uint32_t* offsets,
                                  uint64_t bins, const InterpParts& parts, cudaStream_t stream);

}  // namespace b200nufft
