// Many independent type-1 problems in one persistent spreading launch
// (b200nufft_batch_*).
//
// The reference runs every plan on its own (src/plan.rs), and bounds long
// dispatches by splitting them (src/gpu_dispatch.rs:30-116). Here the
// problems of a batch -- 2D and 3D f32 type-1 plans of one window width,
// each with its own grid, point set and strengths -- are spread by one
// launch whose CTAs pull (problem, tile part) items from a device counter,
// so that small problems fill the GPU together instead of one after another.
// Each problem's fold, FFT and deconvolution then run on one of several
// streams forked from the caller's and joined back to it. Every problem's
// padded tiles, and so its modes, are the bits of its own execution.
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <vector>

#include "plan.h"
#include "util.h"

namespace b200nufft {

namespace {

constexpr int kBatchStreams = 8;

class BatchExecutor {
 public:
  BatchExecutor(NufftPlan* const* plans, int count) : plans_(plans, plans + count) {
    if (count <= 0 || count > kMaxBatchProblems) {
      throw NufftFailure{B200NUFFT_INVALID_ARGUMENT,
                         "a batch holds 1 to " + std::to_string(kMaxBatchProblems) + " plans"};
    }
    device_ = plans_[0]->device();
    width_ = plans_[0]->kernel().width;
    for (NufftPlan* p : plans_) {
      if (p == nullptr) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null plan"};
      if (p->type() != 1 || p->precision() != B200NUFFT_PRECISION_F32 || (p->dimensions() != 2 && p->dimensions() != 3)) {
        throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "a batch takes 2D and 3D f32 type-1 plans"};
      }
      if (p->kernel().width != width_) {
        throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "the plans of a batch share one window width (one eps)"};
      }
      if (p->device() != device_) throw NufftFailure{B200NUFFT_GPU_DEVICE_MISMATCH, "the plans of a batch share one device"};
    }
    check_cuda(cudaSetDevice(device_), "select batch device");
    for (int k = 0; k < kBatchStreams; ++k) {
      cudaStream_t s;
      check_cuda(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "batch stream");
      streams_.push_back(s);
      cudaEvent_t e;
      check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "batch event");
      joins_.push_back(e);
    }
    check_cuda(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming), "batch event");
  }

  ~BatchExecutor() {
    cudaSetDevice(device_);
    cudaDeviceSynchronize();
    for (cudaStream_t s : streams_) cudaStreamDestroy(s);
    for (cudaEvent_t e : joins_) cudaEventDestroy(e);
    cudaEventDestroy(fork_);
  }

  void execute(const void* const* strengths, void* const* outputs, cudaStream_t stream) {
    check_cuda(cudaSetDevice(device_), "select batch device");
    if (strengths == nullptr || outputs == nullptr) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null arrays"};
    refresh();
    BatchStrengths ptrs{};
    for (size_t p = 0; p < plans_.size(); ++p) {
      if (plans_[p]->points_set_count() > 0 && (strengths[p] == nullptr || outputs[p] == nullptr)) {
        throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null strengths or output of problem " + std::to_string(p)};
      }
      ptrs.ptr[p] = static_cast<const float2*>(strengths[p]);
    }
    batch_spread(static_cast<const BatchProblem*>(problems_.get()), ptrs, static_cast<int>(plans_.size()), width_,
                 has_2d_, has_3d_, shared_bytes_, static_cast<uint32_t*>(work_.get()), stream);
    check_cuda(cudaEventRecord(fork_, stream), "batch fork");
    for (cudaStream_t s : streams_) check_cuda(cudaStreamWaitEvent(s, fork_, 0), "batch fork wait");
    for (size_t p = 0; p < plans_.size(); ++p) plans_[p]->finish_batch(outputs[p], streams_[p % streams_.size()]);
    for (size_t k = 0; k < streams_.size(); ++k) {
      check_cuda(cudaEventRecord(joins_[k], streams_[k]), "batch join");
      check_cuda(cudaStreamWaitEvent(stream, joins_[k], 0), "batch join wait");
    }
    check_cuda(cudaGetLastError(), "batch launch");
  }

 private:
  // The device descriptors: rebuilt on the host every execution (a plan's
  // own executions can grow its scratch buffer, set_points replaces its point
  // set) and uploaded when they differ from the last upload. The upload is
  // synchronous, so the first execution after set_points must not be
  // captured in a graph.
  void refresh() {
    std::vector<BatchProblem> host(plans_.size());
    size_t shared = 0;
    bool has_2d = false, has_3d = false;
    for (size_t p = 0; p < plans_.size(); ++p) {
      if (!plans_[p]->batch_problem(&host[p])) {
        throw NufftFailure{B200NUFFT_GPU_EXECUTION_UNAVAILABLE,
                           "problem " + std::to_string(p) + " has no point set (b200nufft_set_points)"};
      }
      shared = std::max(shared, spread_shared_bytes(host[p].sp));
      has_2d = has_2d || plans_[p]->dimensions() == 2;
      has_3d = has_3d || plans_[p]->dimensions() == 3;
    }
    const size_t bytes = host.size() * sizeof(BatchProblem);
    if (uploaded_.size() == host.size() && std::memcmp(uploaded_.data(), host.data(), bytes) == 0) return;
    void* d = problems_.reserve(bytes, "batch descriptors");
    check_cuda(cudaMemcpy(d, host.data(), bytes, cudaMemcpyHostToDevice), "upload batch descriptors");
    work_.reserve((plans_.size() + 2) * sizeof(uint32_t), "batch work list");
    uploaded_ = std::move(host);
    shared_bytes_ = shared;
    has_2d_ = has_2d;
    has_3d_ = has_3d;
  }

  std::vector<NufftPlan*> plans_;
  std::vector<BatchProblem> uploaded_;
  int device_ = 0;
  int width_ = 0;
  bool has_2d_ = false, has_3d_ = false;
  size_t shared_bytes_ = 0;
  DeviceBuffer problems_, work_;
  std::vector<cudaStream_t> streams_;
  std::vector<cudaEvent_t> joins_;
  cudaEvent_t fork_ = nullptr;
};

}  // namespace

}  // namespace b200nufft

struct b200nufft_batch_s {
  std::unique_ptr<b200nufft::BatchExecutor> impl;
};

// The plan handle's layout is defined in api.cpp.
b200nufft::NufftPlan* b200nufft_plan_impl(b200nufft_plan plan);

extern "C" int b200nufft_batch_create(const b200nufft_plan* plans, int32_t count, b200nufft_batch* batch) {
  try {
    if (plans == nullptr || batch == nullptr) throw b200nufft::NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null argument"};
    std::vector<b200nufft::NufftPlan*> impls;
    for (int32_t i = 0; i < count; ++i) impls.push_back(plans[i] ? b200nufft_plan_impl(plans[i]) : nullptr);
    auto* b = new b200nufft_batch_s;
    try {
      b->impl = std::make_unique<b200nufft::BatchExecutor>(impls.data(), count);
    } catch (...) {
      delete b;
      throw;
    }
    *batch = b;
    return B200NUFFT_SUCCESS;
  } catch (const b200nufft::NufftFailure& failure) {
    b200nufft::set_last_error(failure.message);
    return failure.code;
  } catch (...) {
    b200nufft::set_last_error("internal error");
    return B200NUFFT_INTERNAL;
  }
}

extern "C" void b200nufft_batch_destroy(b200nufft_batch batch) { delete batch; }

extern "C" int b200nufft_batch_execute(b200nufft_batch batch, const void* const* strengths, void* const* outputs,
                                       void* stream) {
  try {
    if (batch == nullptr) throw b200nufft::NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null batch"};
    batch->impl->execute(strengths, outputs, static_cast<cudaStream_t>(stream));
    return B200NUFFT_SUCCESS;
  } catch (const b200nufft::NufftFailure& failure) {
    b200nufft::set_last_error(failure.message);
    return failure.code;
  } catch (...) {
    b200nufft::set_last_error("internal error");
    return B200NUFFT_INTERNAL;
  }
}
