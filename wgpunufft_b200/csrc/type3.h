// Type-3 plans (the NufftType3Plan mirror).
#pragma once

#include <cuda_runtime.h>

#include "device.h"

namespace b200nufft {

class Type3Plan {
 public:
  explicit Type3Plan(const b200nufft_type3_config& config);
  void set_points(int64_t source_count, const void* sources, int64_t target_count,
                  const void* targets, cudaStream_t stream);
  void execute(int64_t active_batch, const void* strengths, void* output, cudaStream_t stream);
  void info(b200nufft_type3_info* out) const;
};

}  // namespace b200nufft
