// Deconvolution around the fine-grid FFT.
//
// Type 1 truncates the transformed fine grid to the requested modes and
// scales every mode by its deconvolution amplitude prod_a 1/phi_hat_a(|k_a|)
// (the reference's deconvolution shader, src/gpu_type1_nd.rs:617-687). Type 2
// writes every fine-grid cell once: the deconvolved mode that maps to it, or
// zero, so the clearing pass of the reference (src/gpu_2d.rs:640-648, 896-957)
// is fused into the scatter.
#include <cuda_runtime.h>

#include <algorithm>

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

// Grids of at least kRowsMinRows rows of at least kRowsMinCells cells along
// axis 0: a CTA per row, its mode offset along the other axes found once, so
// a thread does no division; the threads stride along the row.
constexpr int kRowsMinCells = 64;
constexpr int64_t kRowsMinRows = 1024;

template <typename Real, typename Complex, typename Index>
__global__ void __launch_bounds__(256) predeconvolve_rows_kernel(ModeParams mp, int batch,
                                                                 const Complex* __restrict__ input,
                                                                 const Real* __restrict__ amplitudes,
                                                                 Complex* __restrict__ fine) {
  __shared__ int64_t row_flat;
  __shared__ int row_mapped;
  const Index row = static_cast<Index>(blockIdx.x);
  if (threadIdx.x == 0) {
    Index rest = row;
    int64_t flat = 0, stride = mp.modes[0];
    bool mapped = true;
    for (int a = 1; a < mp.dimensions; ++a) {
      const Index n = static_cast<Index>(mp.fine[a]);
      const int64_t cell = rest % n;
      rest /= n;
      const int64_t index = mode_index(cell, mp.modes[a], mp.fine[a], mp.centered);
      mapped = mapped && index >= 0;
      flat += index * stride;
      stride *= mp.modes[a];
    }
    row_flat = flat;
    row_mapped = mapped ? 1 : 0;
  }
  __syncthreads();
  const int64_t n0 = mp.fine[0];
  const int64_t row_start = n0 * static_cast<int64_t>(row);
  for (int64_t x = threadIdx.x; x < n0; x += blockDim.x) {
    const int64_t index = mode_index(x, mp.modes[0], n0, mp.centered);
    const bool mapped = row_mapped != 0 && index >= 0;
    const int64_t flat = row_flat + index;
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
      fine[static_cast<int64_t>(b) * mp.fine_count + row_start + x] = o;
    }
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
  // Enough rows to fill the GPU (1D grids are one row).
  if (mp.fine[0] >= kRowsMinCells && mp.fine_count / mp.fine[0] >= kRowsMinRows) {
    const unsigned rows = static_cast<unsigned>(mp.fine_count / mp.fine[0]);
    const int threads = static_cast<int>(std::min<int64_t>(256, (mp.fine[0] + 31) / 32 * 32));
    if (narrow(mp)) {
      predeconvolve_rows_kernel<Real, Complex, uint32_t><<<rows, threads, 0, stream>>>(mp, batch, input, amplitudes,
                                                                                       fine);
    } else {
      predeconvolve_rows_kernel<Real, Complex, int64_t><<<rows, threads, 0, stream>>>(mp, batch, input, amplitudes,
                                                                                      fine);
    }
    note_launch();
    return;
  }
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
