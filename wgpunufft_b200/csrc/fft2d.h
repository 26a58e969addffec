// Host interface of the fused 2D f32 transforms (fft2d.cu): the fine-grid
// FFT of 2D f32 plans whose fine axes are powers of two, computed in shared
// memory one fine row or a few mode columns per CTA and pruned to the modes,
// with the fold of the spreading tiles fused into the row transforms (type
// 1), the deconvolution into the column transforms (type 1) and the
// predeconvolution into the column transforms (type 2).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "device.h"
#include "modes.h"
#include "spread.h"

namespace b200nufft {

// Fine-grid lengths the fused transforms take: powers of two from 2^6 to 2^12.
constexpr int kFft2dMinLog2 = 6;
constexpr int kFft2dMaxLog2 = 12;

struct Fft2dParams {
  int32_t log2n[2];          // fine-grid lengths 2^log2n[a]
  int32_t modes[2];          // modes per axis
  int32_t centered;          // centered mode order, else FFT order
  int32_t sign;              // exponent sign of the transform (+1 or -1)
  const float2* twiddle[2];  // fft2d_twiddles(2^log2n[a], sign), device
};

// Whether a 2D f32 plan with these fine-grid lengths and modes takes the fused transforms.
bool fft2d_supported(int dimensions, const int64_t* fine, const int64_t* modes);

// The twiddles exp(sign 2 pi i m / n) of an n-point transform in the order
// its passes read them, computed in double and rounded to float.
std::vector<float2> fft2d_twiddles(int64_t n, int sign);

// Bytes of the row-transformed intermediate of `batch` vectors.
size_t fft2d_rows_bytes(const Fft2dParams& fp, int batch);

// Type 1: the fold of the padded tiles into every fine row and its
// transform along axis 0, kept modes only, into `rows` (stage fold), then
// the transforms along axis 1 with the deconvolution into `output` (stage
// fft).
void fft2d_type1(const SpreadParams& sp, const Fft2dParams& fp, int batch, const float2* scratch,
                 const uint32_t* part_start, int64_t part_limit, const int2* candidates, const float* amplitudes,
                 float2* rows, float2* output, cudaStream_t stream, StageTimer* timer);

// Type 2: the predeconvolved modes transformed along axis 1 into `rows`
// (stage predeconvolution), then along axis 0 into every cell of the fine
// grid (stage fft).
void fft2d_type2(const Fft2dParams& fp, int batch, const float2* input, const float* amplitudes, float2* rows,
                 float2* fine, cudaStream_t stream, StageTimer* timer);

}  // namespace b200nufft
