// CUDA-event stage timing of a plan (b200nufft_plan_stage_timing).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "status.h"

namespace b200nufft {

enum Stage {
  kStageBinKeys = 0,
  kStageDigitScan,
  kStageRadixPasses,
  kStageBinOffsets,
  kStageTileParts,
  kStageStrengthScale,
  kStageSpread,
  kStageFold,
  kStageFft,
  kStageDeconvolution,
  kStagePredeconvolution,
  kStageInterpolation,
};

class StageTimer {
 public:
  ~StageTimer() { clear(); }
  void enable(bool on) { enabled_ = on; }
  bool enabled() const { return enabled_; }

  // Records the start of `stage` on `stream`; a no-op unless enabled.
  void begin(int stage, cudaStream_t stream) {
    if (!enabled_) return;
    Pair p{stage, nullptr, nullptr};
    cudaEventCreate(&p.start);
    cudaEventCreate(&p.stop);
    cudaEventRecord(p.start, stream);
    pairs_.push_back(p);
    open_ = true;
  }

  void end(cudaStream_t stream) {
    if (!enabled_ || !open_) return;
    cudaEventRecord(pairs_.back().stop, stream);
    open_ = false;
  }

  // Sums the elapsed time of every recorded pair per stage; the caller has
  // synchronized the streams they were recorded on.
  void report(b200nufft_stage_report* out) {
    for (int s = 0; s < B200NUFFT_STAGE_COUNT; ++s) {
      out->milliseconds[s] = 0.0;
      out->launches[s] = 0;
    }
    for (const Pair& p : pairs_) {
      float ms = 0.0f;
      if (cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess) {
        out->milliseconds[p.stage] += ms;
        out->launches[p.stage] += 1;
      }
    }
    clear();
  }

  void clear() {
    for (const Pair& p : pairs_) {
      cudaEventDestroy(p.start);
      cudaEventDestroy(p.stop);
    }
    pairs_.clear();
    open_ = false;
  }

 private:
  struct Pair {
    int stage;
    cudaEvent_t start;
    cudaEvent_t stop;
  };
  bool enabled_ = false;
  bool open_ = false;
  std::vector<Pair> pairs_;
};

// Times one stage for the lifetime of the scope.
class StageScope {
 public:
  StageScope(StageTimer* timer, int stage, cudaStream_t stream) : timer_(timer), stream_(stream) {
    if (timer_) timer_->begin(stage, stream_);
  }
  ~StageScope() {
    if (timer_) timer_->end(stream_);
  }

 private:
  StageTimer* timer_;
  cudaStream_t stream_;
};

}  // namespace b200nufft
