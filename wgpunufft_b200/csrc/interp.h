// Host interface of the type-2 interpolation kernels (interp.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device.h"

namespace b200nufft {

struct InterpLaunch {
  const float* points;    // coordinates in bin (slot) order
  int64_t point_count;
  const uint32_t* perm;   // slot -> original point, in bin order
  const float2* fine;     // batch * fine_count
  int batch;
  float2* output;         // batch * point_count, input order
};

void interpolate_execute(const GridParams& g, const InterpLaunch& launch, cudaStream_t stream);

}  // namespace b200nufft
