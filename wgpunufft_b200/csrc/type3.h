// Type-3 plans (the NufftType3Plan mirror, src/type3.rs, src/gpu_type3.rs).
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "device.h"
#include "es_kernel.h"
#include "plan.h"

namespace b200nufft {

// Per-axis rescaling of a type-3 plan (NufftType3AxisMetadata, src/type3.rs:225-286).
struct Type3Axis {
  double source_half_width;
  double source_center;
  double target_half_width;
  double target_center;
  int64_t outer;        // outer grid length nf
  double grid_spacing;  // h = 2 pi / nf
  double source_scale;  // gamma: x' = (x - C) / gamma
};

// The constants of the pre- and post-phase kernels.
struct Type3Params {
  int32_t dimensions;
  int32_t isign;
  double source_center[3];
  double source_inv_scale[3];
  double target_center[3];
  double target_scale[3];  // h * gamma
  int32_t quadrature_count;
  double nodes[18];        // positive Gauss-Legendre nodes times w/2
  double weights[18];      // 2 (w/2) weight phi(node)
};

class Type3Plan {
 public:
  explicit Type3Plan(const b200nufft_type3_config& config);
  void set_points(int64_t source_count, const void* sources, int64_t target_count,
                  const void* targets, cudaStream_t stream);
  void execute(int64_t active_batch, const void* strengths, void* output, cudaStream_t stream);
  void info(b200nufft_type3_info* out) const;

 private:
  int dim_ = 1;
  int64_t batch_ = 1;
  double eps_ = 1e-9;
  int isign_ = 1;
  double sigma_ = 2.0;
  int precision_ = B200NUFFT_PRECISION_F64;
  int device_ = 0;
  EsKernel kernel_;
  std::vector<Type3Axis> axes_;
  Type3Params params_{};
  std::unique_ptr<NufftPlan> outer_;
  std::unique_ptr<NufftPlan> inner_;
  int64_t source_count_ = -1;
  int64_t target_count_ = 0;
  DeviceBuffer rescaled_sources_, source_factors_, rescaled_targets_, target_factors_;
  DeviceBuffer prephased_, outer_grid_, interpolated_;
  DeviceBuffer sources64_, targets64_, strengths64_, output64_;
};

}  // namespace b200nufft
