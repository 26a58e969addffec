// Deconvolution around the fine-grid FFT.
//
// Type 1 truncates the transformed fine grid to the requested modes and
// scales every mode by its deconvolution amplitude prod_a 1/phi_hat_a(|k_a|)
// (the reference's deconvolution shader, src/gpu_type1_nd.rs:617-687). Type 2
// writes every fine-grid cell once: the deconvolved mode that maps to it, or
// zero, so the clearing pass of the reference (src/gpu_2d.rs:640-648, 896-957)
// is fused into the scatter.
#include <cuda_runtime.h>

#include "device.h"
#include "modes.h"

namespace b200nufft {

namespace {

// Index: uint32_t when every mode and cell index fits (32-bit divisions are
// far cheaper than 64-bit ones), else int64_t.
template <typename Real, typename Complex, typename Index>
__global__ void deconvolve_kernel(ModeParams mp, int batch, const Complex* __restrict__ fine,
                                  const Real* __restrict__ amplitudes,
                                  Complex* __restrict__ output) {
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= mp.mode_count) return;
  Index rest = static_cast<Index>(k);
  int64_t flat = 0, stride = 1;
  for (int a = 0; a < mp.dimensions; ++a) {
    const Index n = static_cast<Index>(mp.modes[a]);
    const int64_t index = rest % n;
    rest /= n;
    flat += fine_index(index, mp.modes[a], mp.fine[a], mp.centered) * stride;
    stride *= mp.fine[a];
  }
  const Real amplitude = amplitudes[k];
  for (int b = 0; b < batch; ++b) {
    const Complex v = fine[static_cast<int64_t>(b) * mp.fine_count + flat];
    Complex o;
    o.x = v.x * amplitude;
    o.y = v.y * amplitude;
    output[static_cast<int64_t>(b) * mp.mode_count + k] = o;
  }
}

template <typename Real, typename Complex, typename Index>
__global__ void predeconvolve_kernel(ModeParams mp, int batch, const Complex* __restrict__ input,
                                     const Real* __restrict__ amplitudes,
                                     Complex* __restrict__ fine) {
  const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= mp.fine_count) return;
  Index rest = static_cast<Index>(c);
  int64_t flat = 0, stride = 1;
  bool mapped = true;
  for (int a = 0; a < mp.dimensions; ++a) {
    const Index n = static_cast<Index>(mp.fine[a]);
    const int64_t cell = rest % n;
    rest /= n;
    const int64_t index = mode_index(cell, mp.modes[a], mp.fine[a], mp.centered);
    mapped = mapped && index >= 0;
    flat += index * stride;
    stride *= mp.modes[a];
  }
  const Real amplitude = mapped ? amplitudes[flat] : Real(0);
  for (int b = 0; b < batch; ++b) {
    Complex o;
    o.x = Real(0);
    o.y = Real(0);
    if (mapped) {
      const Complex v = input[static_cast<int64_t>(b) * mp.mode_count + flat];
      o.x = v.x * amplitude;
      o.y = v.y * amplitude;
    }
    fine[static_cast<int64_t>(b) * mp.fine_count + c] = o;
  }
}

bool narrow(const ModeParams& mp) {
  return mp.fine_count < (int64_t(1) << 31) && mp.mode_count < (int64_t(1) << 31);
}

template <typename Real, typename Complex>
void deconvolve_any(const ModeParams& mp, int batch, const Complex* fine, const Real* amplitudes, Complex* output,
                    cudaStream_t stream) {
  const unsigned blocks = static_cast<unsigned>((mp.mode_count + 255) / 256);
  if (narrow(mp)) {
    deconvolve_kernel<Real, Complex, uint32_t><<<blocks, 256, 0, stream>>>(mp, batch, fine, amplitudes, output);
  } else {
    deconvolve_kernel<Real, Complex, int64_t><<<blocks, 256, 0, stream>>>(mp, batch, fine, amplitudes, output);
  }
  note_launch();
}

template <typename Real, typename Complex>
void predeconvolve_any(const ModeParams& mp, int batch, const Complex* input, const Real* amplitudes,
                       Complex* fine, cudaStream_t stream) {
  const unsigned blocks = static_cast<unsigned>((mp.fine_count + 255) / 256);
  if (narrow(mp)) {
    predeconvolve_kernel<Real, Complex, uint32_t><<<blocks, 256, 0, stream>>>(mp, batch, input, amplitudes, fine);
  } else {
    predeconvolve_kernel<Real, Complex, int64_t><<<blocks, 256, 0, stream>>>(mp, batch, input, amplitudes, fine);
  }
  note_launch();
}

}  // namespace

void deconvolve_f32(const ModeParams& mp, int batch, const float2* fine, const float* amplitudes,
                    float2* output, cudaStream_t stream) {
  deconvolve_any<float, float2>(mp, batch, fine, amplitudes, output, stream);
}

void predeconvolve_f32(const ModeParams& mp, int batch, const float2* input,
                       const float* amplitudes, float2* fine, cudaStream_t stream) {
  predeconvolve_any<float, float2>(mp, batch, input, amplitudes, fine, stream);
}

void deconvolve_f64(const ModeParams& mp, int batch, const double2* fine,
                    const double* amplitudes, double2* output, cudaStream_t stream) {
  deconvolve_any<double, double2>(mp, batch, fine, amplitudes, output, stream);
}

void predeconvolve_f64(const ModeParams& mp, int batch, const double2* input,
                       const double* amplitudes, double2* fine, cudaStream_t stream) {
  predeconvolve_any<double, double2>(mp, batch, input, amplitudes, fine, stream);
}

}  // namespace b200nufft
