// Device side of the host-array C interface: host arrays are copied to the
// device as they are, then checked and converted to the plan's storage here
// (f32, f64, or Df64 pairs), so the host touches each array only through its
// copy. Checks follow capi/src/plan.rs:524-545: type-1/2 coordinates must not
// be NaN nor lie beyond 3 pi (after rounding to f32 for f32 plans), type-3
// coordinates and all input values must be finite; the smallest offending
// element index is reported.
#include "capi_io.h"

#include <cstring>

namespace b200nufft {

namespace {

constexpr double kThreePi = 3.0 * 3.14159265358979323846;

// Order-preserving 64-bit keys of doubles, for atomic minima and maxima.
__device__ __forceinline__ unsigned long long order_key(double v) {
  const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(v));
  return (bits >> 63) ? ~bits : (bits | 0x8000000000000000ull);
}

template <typename In>
__device__ __forceinline__ double load_scalar(const In* p) {
  return static_cast<double>(*p);
}

// Rounds a host value to the plan's storage and returns the value the plan
// computes with (f32 plans see the f32 rounding).
__device__ __forceinline__ double stored_value(double v, int precision) {
  return precision == B200NUFFT_PRECISION_F32 ? static_cast<double>(static_cast<float>(v)) : v;
}

__device__ __forceinline__ void store_scalar(void* out, int64_t index, double v, int precision) {
  if (precision == B200NUFFT_PRECISION_F32) {
    static_cast<float*>(out)[index] = static_cast<float>(v);
  } else if (precision == B200NUFFT_PRECISION_F64) {
    static_cast<double*>(out)[index] = v;
  } else {
    const float hi = static_cast<float>(v);
    static_cast<float2*>(out)[index] = make_float2(hi, static_cast<float>(v - static_cast<double>(hi)));
  }
}

template <typename In>
__global__ void gather_points_kernel(const In* __restrict__ in, int64_t axis_stride, int64_t point_stride,
                                     int dim, int64_t count, int precision, int check, void* __restrict__ out,
                                     unsigned long long* __restrict__ first_bad,
                                     unsigned long long* __restrict__ bounds) {
  const int64_t total = count * dim;
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int64_t i = e / dim;
    const int a = static_cast<int>(e - i * dim);
    const double v = stored_value(load_scalar(in + a * axis_stride + i * point_stride), precision);
    const bool bad = check == 0 ? (isnan(v) || fabs(v) > kThreePi) : !isfinite(v);
    if (bad) atomicMin(first_bad, static_cast<unsigned long long>(e));
    store_scalar(out, e, v, precision);
    if (bounds != nullptr && !bad) {
      atomicMin(&bounds[2 * a], order_key(v));
      atomicMax(&bounds[2 * a + 1], order_key(v));
    }
  }
}

template <typename In>
__global__ void convert_values_kernel(const In* __restrict__ in, int64_t count, int precision, void* __restrict__ out,
                                      unsigned long long* __restrict__ first_bad) {
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < count;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const double v = load_scalar(in + e);
    if (!isfinite(v)) atomicMin(first_bad, static_cast<unsigned long long>(e));
    if (out != nullptr) store_scalar(out, e, v, precision);
  }
}

template <typename Out>
__global__ void convert_back_kernel(const void* __restrict__ in, int64_t count, int precision, Out* __restrict__ out) {
  for (int64_t e = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < count;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    double v;
    if (precision == B200NUFFT_PRECISION_F32) {
      v = static_cast<const float*>(in)[e];
    } else if (precision == B200NUFFT_PRECISION_F64) {
      v = static_cast<const double*>(in)[e];
    } else {
      const float2 p = static_cast<const float2*>(in)[e];
      v = static_cast<double>(p.x) + static_cast<double>(p.y);
    }
    out[e] = static_cast<Out>(v);
  }
}

unsigned grid_for(int64_t count) {
  const int64_t blocks = (count + 255) / 256;
  return static_cast<unsigned>(blocks < 148 * 16 ? (blocks > 0 ? blocks : 1) : 148 * 16);
}

}  // namespace

void capi_gather_points(HostScalar in, const void* src, int64_t axis_stride, int64_t point_stride, int dim,
                        int64_t count, int precision, int check, void* out, unsigned long long* first_bad,
                        unsigned long long* bounds, cudaStream_t stream) {
  if (count <= 0) return;
  const unsigned grid = grid_for(count * dim);
  if (in == HostScalar::F32) {
    gather_points_kernel<float><<<grid, 256, 0, stream>>>(static_cast<const float*>(src), axis_stride, point_stride,
                                                          dim, count, precision, check, out, first_bad, bounds);
  } else {
    gather_points_kernel<double><<<grid, 256, 0, stream>>>(static_cast<const double*>(src), axis_stride,
                                                           point_stride, dim, count, precision, check, out,
                                                           first_bad, bounds);
  }
  note_launch();
}

void capi_convert_values(HostScalar in, const void* src, int64_t count, int precision, void* out,
                         unsigned long long* first_bad, cudaStream_t stream) {
  if (count <= 0) return;
  const unsigned grid = grid_for(count);
  if (in == HostScalar::F32) {
    convert_values_kernel<float><<<grid, 256, 0, stream>>>(static_cast<const float*>(src), count, precision, out,
                                                           first_bad);
  } else {
    convert_values_kernel<double><<<grid, 256, 0, stream>>>(static_cast<const double*>(src), count, precision, out,
                                                            first_bad);
  }
  note_launch();
}

void capi_convert_back(int precision, const void* src, int64_t count, HostScalar out, void* dst,
                       cudaStream_t stream) {
  if (count <= 0) return;
  const unsigned grid = grid_for(count);
  if (out == HostScalar::F32) {
    convert_back_kernel<float><<<grid, 256, 0, stream>>>(src, count, precision, static_cast<float*>(dst));
  } else {
    convert_back_kernel<double><<<grid, 256, 0, stream>>>(src, count, precision, static_cast<double*>(dst));
  }
  note_launch();
}

double capi_key_value(unsigned long long key) {
  const unsigned long long bits = (key >> 63) ? (key & 0x7FFFFFFFFFFFFFFFull) : ~key;
  double v;
  std::memcpy(&v, &bits, sizeof(v));
  return v;
}

}  // namespace b200nufft
