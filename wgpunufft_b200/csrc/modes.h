// Host interface of the deconvolution kernels (modes.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace b200nufft {

struct ModeParams {
  int32_t dimensions;
  int32_t centered;  // centered mode order, else FFT order
  int64_t modes[8];
  int64_t fine[8];
  int64_t mode_count;
  int64_t fine_count;
};

void deconvolve_f32(const ModeParams& mp, int batch, const float2* fine, const float* amplitudes,
                    float2* output, cudaStream_t stream);
void predeconvolve_f32(const ModeParams& mp, int batch, const float2* input,
                       const float* amplitudes, float2* fine, cudaStream_t stream);
void deconvolve_f64(const ModeParams& mp, int batch, const double2* fine,
                    const double* amplitudes, double2* output, cudaStream_t stream);
void predeconvolve_f64(const ModeParams& mp, int batch, const double2* input,
                       const double* amplitudes, double2* fine, cudaStream_t stream);

}  // namespace b200nufft
