// Host interface of the deconvolution kernels (modes.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace b200nufft {

// Fine-grid index of mode storage index k along an axis of N modes and n
// cells (src/gpu_type1_nd.rs:642-652).
__host__ __device__ inline int64_t fine_index(int64_t k, int64_t N, int64_t n, bool centered) {
  if (centered) {
    const int64_t half = N / 2;
    return k < half ? n - (half - k) : k - half;
  }
  const int64_t nonnegative = (N + 1) / 2;
  return k < nonnegative ? k : n - (N - k);
}

// Mode storage index of fine-grid cell c, or -1 when no mode maps to it.
__host__ __device__ inline int64_t mode_index(int64_t c, int64_t N, int64_t n, bool centered) {
  if (centered) {
    const int64_t half = N / 2;
    if (c < N - half) return c + half;
    if (c >= n - half) return c - n + half;
    return -1;
  }
  const int64_t nonnegative = (N + 1) / 2;
  if (c < nonnegative) return c;
  if (c >= n - (N - nonnegative)) return c - n + N;
  return -1;
}

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
