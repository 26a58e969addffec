// Device-side checks and conversions of the host-array C interface (capi_io.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device.h"

namespace b200nufft {

enum class HostScalar { F32, F64 };

// Point-major coordinates in the plan's storage (precision), from element
// (point i, axis a) at src[a * axis_stride + i * point_stride]. check 0:
// type-1/2 coordinates (not NaN, |x| <= 3 pi after rounding to the storage);
// check 1: finite. The smallest offending element index (i * dim + a) is
// folded into *first_bad with atomicMin; when `bounds` is given, the
// per-axis minimum and maximum are folded into bounds[2a], bounds[2a + 1] as
// order-preserving keys (capi_key_value decodes them).
void capi_gather_points(HostScalar in, const void* src, int64_t axis_stride, int64_t point_stride, int dim,
                        int64_t count, int precision, int check, void* out, unsigned long long* first_bad,
                        unsigned long long* bounds, cudaStream_t stream);

// `count` scalars checked for finiteness and, when `out` is given, converted
// to the plan's storage.
void capi_convert_values(HostScalar in, const void* src, int64_t count, int precision, void* out,
                         unsigned long long* first_bad, cudaStream_t stream);

// `count` scalars of the plan's storage converted to the host scalar type.
void capi_convert_back(int precision, const void* src, int64_t count, HostScalar out, void* dst,
                       cudaStream_t stream);

double capi_key_value(unsigned long long key);

}  // namespace b200nufft
