// extern "C" entry points of include/b200_nufft.h.
#include <cstring>
#include <exception>
#include <new>

#include "plan.h"
#include "type3.h"
#include "util.h"

using b200nufft::NufftFailure;

struct b200nufft_plan_s {
  b200nufft::NufftPlan impl;
  b200nufft_plan_s(const b200nufft_config& c, bool with_device) : impl(c, with_device) {}
};

struct b200nufft_type3_plan_s {
  b200nufft::Type3Plan impl;
  explicit b200nufft_type3_plan_s(const b200nufft_type3_config& c) : impl(c) {}
};

b200nufft::NufftPlan* b200nufft_plan_impl(b200nufft_plan plan) { return &plan->impl; }

namespace {

template <typename F>
int guarded(F&& body) {
  try {
    body();
    return B200NUFFT_SUCCESS;
  } catch (const NufftFailure& failure) {
    b200nufft::set_last_error(failure.message);
    return failure.code;
  } catch (const std::bad_alloc&) {
    b200nufft::set_last_error("host allocation failed");
    return B200NUFFT_INTERNAL;
  } catch (const std::exception& e) {
    b200nufft::set_last_error(std::string("internal error: ") + e.what());
    return B200NUFFT_INTERNAL;
  } catch (...) {
    b200nufft::set_last_error("internal error");
    return B200NUFFT_INTERNAL;
  }
}

template <typename P>
void require(P* plan) {
  if (!plan) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null plan"};
}

}  // namespace

extern "C" {

void b200nufft_default_config(b200nufft_config* config) {
  if (!config) return;
  std::memset(config, 0, sizeof(*config));
  config->type = 1;
  config->dimensions = 1;
  config->n_modes[0] = 1;
  config->batch = 1;
  config->eps = 1e-6;
  config->isign = 1;
  config->mode_order = B200NUFFT_MODE_ORDER_CENTERED;
  config->sigma = 2.0;
  config->precision = B200NUFFT_PRECISION_F32;
  config->device = -1;
}

int b200nufft_plan_create(const b200nufft_config* config, b200nufft_plan* plan) {
  return guarded([&] {
    if (!config || !plan) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null argument"};
    *plan = nullptr;
    *plan = new b200nufft_plan_s(*config, true);
  });
}

int b200nufft_plan_create_host(const b200nufft_config* config, b200nufft_plan* plan) {
  return guarded([&] {
    if (!config || !plan) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null argument"};
    *plan = nullptr;
    *plan = new b200nufft_plan_s(*config, false);
  });
}

int b200nufft_plan_choose_geometry(b200nufft_plan plan, int64_t point_count, int32_t* geometry) {
  return guarded([&] {
    require(plan);
    if (!geometry) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null result"};
    *geometry = plan->impl.choose_geometry(point_count);
  });
}

void b200nufft_plan_destroy(b200nufft_plan plan) { delete plan; }

int b200nufft_plan_get_info(b200nufft_plan plan, b200nufft_plan_info* info) {
  return guarded([&] {
    require(plan);
    if (!info) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null info"};
    plan->impl.info(info);
  });
}

int b200nufft_plan_kernel_fourier_coefficients(b200nufft_plan plan, int32_t axis, double* values,
                                               int64_t capacity, int64_t* count) {
  return guarded([&] {
    require(plan);
    if (axis < 0 || axis >= plan->impl.dimensions()) {
      throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "axis out of range"};
    }
    const auto& v = plan->impl.phi_hat(axis);
    if (count) *count = static_cast<int64_t>(v.size());
    if (values) {
      const int64_t n = std::min<int64_t>(capacity, static_cast<int64_t>(v.size()));
      std::memcpy(values, v.data(), static_cast<size_t>(n) * sizeof(double));
    }
  });
}

int b200nufft_required_point_bytes(b200nufft_plan plan, int64_t point_count, uint64_t* bytes) {
  return guarded([&] {
    require(plan);
    if (!bytes) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null result"};
    *bytes = plan->impl.required_point_bytes(point_count);
  });
}

int b200nufft_required_input_bytes(b200nufft_plan plan, int64_t point_count, int64_t active_batch,
                                   uint64_t* bytes) {
  return guarded([&] {
    require(plan);
    if (!bytes) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null result"};
    *bytes = plan->impl.required_input_bytes(point_count, active_batch);
  });
}

int b200nufft_required_output_bytes(b200nufft_plan plan, int64_t point_count, int64_t active_batch,
                                    uint64_t* bytes) {
  return guarded([&] {
    require(plan);
    if (!bytes) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null result"};
    *bytes = plan->impl.required_output_bytes(point_count, active_batch);
  });
}

int b200nufft_set_points(b200nufft_plan plan, int64_t point_count, const void* points, void* stream) {
  return guarded([&] {
    require(plan);
    plan->impl.set_points(point_count, points, static_cast<cudaStream_t>(stream));
  });
}

int b200nufft_execute(b200nufft_plan plan, int64_t active_batch, const void* input, void* output,
                      void* stream) {
  return guarded([&] {
    require(plan);
    plan->impl.execute(active_batch, input, output, static_cast<cudaStream_t>(stream));
  });
}

int b200nufft_encode(b200nufft_plan plan, int64_t active_batch, int64_t point_count,
                     const void* points, const void* input, void* output, void* stream) {
  return guarded([&] {
    require(plan);
    plan->impl.set_points(point_count, points, static_cast<cudaStream_t>(stream));
    plan->impl.execute(active_batch, input, output, static_cast<cudaStream_t>(stream));
  });
}

int b200nufft_copy_bin_order(b200nufft_plan plan, uint32_t* permutation, uint32_t* bin_offsets,
                             void* stream) {
  return guarded([&] {
    require(plan);
    plan->impl.copy_bin_order(permutation, bin_offsets, static_cast<cudaStream_t>(stream));
  });
}

int b200nufft_copy_prepared_slots(b200nufft_plan plan, int32_t* starts, float* offsets,
                                  void* stream) {
  return guarded([&] {
    require(plan);
    plan->impl.copy_prepared_slots(starts, offsets, static_cast<cudaStream_t>(stream));
  });
}

int b200nufft_plan_synchronize(b200nufft_plan plan, void* stream) {
  return guarded([&] {
    require(plan);
    plan->impl.synchronize(static_cast<cudaStream_t>(stream));
  });
}

int b200nufft_plan_stage_timing(b200nufft_plan plan, int32_t enable) {
  return guarded([&] {
    require(plan);
    plan->impl.timer().enable(enable != 0);
  });
}

int b200nufft_plan_stage_report(b200nufft_plan plan, b200nufft_stage_report* report) {
  return guarded([&] {
    require(plan);
    if (!report) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null report"};
    plan->impl.timer().report(report);
  });
}

int b200nufft_type3_plan_create(const b200nufft_type3_config* config, b200nufft_type3_plan* plan) {
  return guarded([&] {
    if (!config || !plan) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null argument"};
    *plan = nullptr;
    *plan = new b200nufft_type3_plan_s(*config);
  });
}

void b200nufft_type3_plan_destroy(b200nufft_type3_plan plan) { delete plan; }

int b200nufft_type3_get_info(b200nufft_type3_plan plan, b200nufft_type3_info* info) {
  return guarded([&] {
    require(plan);
    if (!info) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null info"};
    plan->impl.info(info);
  });
}

int b200nufft_type3_set_points(b200nufft_type3_plan plan, int64_t source_count, const void* sources,
                               int64_t target_count, const void* targets, void* stream) {
  return guarded([&] {
    require(plan);
    plan->impl.set_points(source_count, sources, target_count, targets,
                          static_cast<cudaStream_t>(stream));
  });
}

int b200nufft_type3_execute(b200nufft_type3_plan plan, int64_t active_batch, const void* strengths,
                            void* output, void* stream) {
  return guarded([&] {
    require(plan);
    plan->impl.execute(active_batch, strengths, output, static_cast<cudaStream_t>(stream));
  });
}

const char* b200nufft_last_error(void) { return b200nufft::last_error(); }

const char* b200nufft_version(void) { return "0.1.0"; }

uint64_t b200nufft_launch_count(void) { return b200nufft::launch_count(); }

}  // extern "C"
