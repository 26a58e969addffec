// Host interface of the fused fine-grid transforms (fused_fft.cu): the
// fine-grid FFT of 2D and 3D f32 plans whose fine axes are powers of two,
// one axis per pass, each pass pruned to the kept modes, with the fold of
// the spreading tiles fused into the pass along axis 0 and the
// deconvolution into the last pass (type 1), or the predeconvolution into
// the first pass (type 2).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "device.h"
#include "spread.h"

namespace b200nufft {

// Fine-grid lengths the fused transforms take: powers of two from 2^6 to 2^12.
constexpr int kFusedFftMinLog2 = 6;
constexpr int kFusedFftMaxLog2 = 12;

struct FusedFftParams {
  int32_t dims;              // 2 or 3
  int32_t log2n[3];          // fine-grid lengths 2^log2n[a]
  int32_t modes[3];          // modes per axis
  int32_t centered;          // centered mode order, else FFT order
  int32_t sign;              // exponent sign of the transform (+1 or -1)
  const float2* twiddle[3];  // fused_fft_twiddles(2^log2n[a], sign), device
};

// Whether an f32 plan with these fine-grid lengths and modes takes the fused transforms.
bool fused_fft_supported(int dimensions, const int64_t* fine, const int64_t* modes);

// The twiddles exp(sign 2 pi i m / n) of an n-point transform in the order
// its passes read them, computed in double and rounded to float.
std::vector<float2> fused_fft_twiddles(int64_t n, int sign);

// Bytes of the buffer of the pass along axis 0 (`rows` below) for `batch`
// vectors: every fine position of the other axes times m0. 3D plans also
// take a `spare` buffer of n2 m1 m0 entries per vector (the fine grid serves).
size_t fused_fft_buffer_bytes(const FusedFftParams& fp, int batch);

// Type 1: the fold of the padded tiles into every fine row and its
// transform along axis 0, kept modes only, into `rows` (stage fold), then
// the passes along the other axes (through `spare` in 3D), the last scaled
// by the deconvolution amplitudes into `output` (stage fft). With scratch
// null the rows come from the fine grid already folded into `spare` (the
// pass along axis 0 is then timed in stage fft).
void fused_fft_type1(const SpreadParams& sp, const FusedFftParams& fp, int batch, const float2* scratch,
                     const uint32_t* part_start, int64_t part_limit, const int2* candidates, const float* amplitudes,
                     float2* rows, float2* spare, float2* output, cudaStream_t stream, StageTimer* timer);

// Type 2: the predeconvolved modes transformed along the last axis (stage
// predeconvolution), then along the others down to axis 0, into every cell
// of the fine grid (stage fft). 3D passes go through `spare`, which may be
// the fine grid itself (it is read before the last pass writes `fine`).
void fused_fft_type2(const FusedFftParams& fp, int batch, const float2* input, const float* amplitudes, float2* rows,
                     float2* spare, float2* fine, cudaStream_t stream, StageTimer* timer);

}  // namespace b200nufft
