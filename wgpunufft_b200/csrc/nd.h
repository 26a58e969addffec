// Type-1 / type-2 kernels of plans with 4 to 8 dimensions (nd.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device.h"

namespace b200nufft {

constexpr int kNdMaxDimensions = 8;

// Fine-grid geometry and window of a plan with more than three dimensions.
struct NdParams {
  int32_t dimensions;
  int32_t width;
  int32_t f32;  // 1: f32 coordinates, values and window; 0: f64
  float half_width;
  float beta;
  double half_width64;
  FoldAxis axis[kNdMaxDimensions];
  FoldAxis64 axis64[kNdMaxDimensions];
  int64_t fine[kNdMaxDimensions];
  int64_t fine_count;
  const double* horner;  // f64 plans: device, rows x width
  int32_t horner_rows;
};

// Type 1: `batch` fine grids (fine_count cells of float2 or double2) from
// `count` points (point-major, f32 or f64) and their strengths
// (transform-major). `acc` holds 2 x batch x fine_count 64-bit words and
// `max_bits` batch words of scratch.
void nd_spread(const NdParams& p, const void* points, const void* strengths, int64_t count, int batch,
               unsigned long long* acc, unsigned long long* max_bits, void* fine, cudaStream_t stream);

// Type 2: `batch` outputs of `count` values (transform-major, original point
// order) gathered from the fine grids.
void nd_interpolate(const NdParams& p, const void* points, const void* fine, int64_t count, int batch,
                    void* output, cudaStream_t stream);

}  // namespace b200nufft
