// Conversions between the reference's Df64 storage and native f64.
//
// A Df64 scalar is a pair of floats (hi, lo) whose sum is the value
// (the reference's DoubleFloat, two f32 words per scalar). B200 has native
// f64, so Df64 plans convert their inputs to f64, run the f64 pipeline, and
// convert the outputs back: hi = the value rounded to f32, lo = the rest
// rounded to f32.
#include <cuda_runtime.h>

#include "device.h"

namespace b200nufft {

namespace {

__global__ void df64_to_f64_kernel(const float2* __restrict__ pairs, int64_t count,
                                   double* __restrict__ out) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float2 p = pairs[i];
  out[i] = static_cast<double>(p.x) + static_cast<double>(p.y);
}

__global__ void f64_to_df64_kernel(const double* __restrict__ values, int64_t count,
                                   float2* __restrict__ pairs) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const double v = values[i];
  const float hi = __double2float_rn(v);
  const float lo = __double2float_rn(v - static_cast<double>(hi));
  pairs[i] = make_float2(hi, lo);
}

}  // namespace

void df64_to_f64(const float* pairs, int64_t count, double* out, cudaStream_t stream) {
  if (count <= 0) return;
  df64_to_f64_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, stream>>>(
      reinterpret_cast<const float2*>(pairs), count, out);
  note_launch();
}

void f64_to_df64(const double* values, int64_t count, float* pairs, cudaStream_t stream) {
  if (count <= 0) return;
  f64_to_df64_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, stream>>>(
      values, count, reinterpret_cast<float2*>(pairs));
  note_launch();
}

}  // namespace b200nufft
