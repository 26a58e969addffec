// Type-1 / type-2 plans (the NufftPlan mirror) as the C++ host sees them.
#pragma once

#include <cufft.h>

#include <algorithm>
#include <map>
#include <memory>
#include <vector>

#include "device.h"
#include "es_kernel.h"
#include "fused_fft.h"
#include "interp.h"
#include "layout.h"
#include "modes.h"
#include "nd.h"
#include "spread.h"
#include "tc_interp.h"
#include "tc_spread.h"

namespace b200nufft {

class NufftPlan {
 public:
  // Without a device only the host-side metadata is built (the reference's
  // NufftPlan::type1 / type2 plans without GPU resources, src/plan.rs:449-455).
  explicit NufftPlan(const b200nufft_config& config, bool with_device = true);
  ~NufftPlan();

  void set_points(int64_t count, const void* points, cudaStream_t stream);
  void execute(int64_t active_batch, const void* input, void* output, cudaStream_t stream);
  // Type-1 plans: spreads the strengths of the remembered points onto `grid`
  // (active_batch fine grids of the plan's precision), with no FFT and no
  // deconvolution (Type1GpuPlanNd::encode_spread_batch, src/gpu_type1_nd.rs:477).
  void spread_to(int64_t active_batch, const void* strengths, void* grid, cudaStream_t stream);
  int64_t fine_count() const { return fine_count_; }
  void info(b200nufft_plan_info* out) const;
  int choose_geometry(int64_t point_count) const;
  const std::vector<double>& phi_hat(int axis) const { return phi_hat_[axis]; }
  uint64_t required_point_bytes(int64_t count) const;
  uint64_t required_input_bytes(int64_t count, int64_t active_batch) const;
  uint64_t required_output_bytes(int64_t count, int64_t active_batch) const;
  void copy_bin_order(uint32_t* permutation, uint32_t* bin_offsets, cudaStream_t stream);
  void copy_prepared_slots(int32_t* starts, float* offsets, cudaStream_t stream);
  // Waits for the plan's work on `stream` and reports a device wait that gave up.
  void synchronize(cudaStream_t stream);
  // Persistent execution of many problems (batch.cpp): this plan's spreading
  // descriptor for one vector (false when the plan cannot join: not a 2D or
  // 3D f32 type-1 plan with points set), and the rest of its execution once
  // the batch has spread its tiles: fold, FFT, deconvolution.
  bool batch_problem(BatchProblem* out);
  void finish_batch(void* output, cudaStream_t stream);
  // Points of the last set_points (-1 before the first).
  int64_t points_set_count() const { return point_count_; }
  StageTimer& timer() { return timer_; }

  int type() const { return type_; }
  int dimensions() const { return dim_; }
  int precision() const { return precision_; }
  int64_t batch() const { return batch_; }
  int64_t mode_count() const { return mode_count_; }
  int device() const { return device_; }
  const std::vector<int64_t>& fine_shape() const { return fine_; }
  const EsKernel& kernel() const { return kernel_; }

 private:
  void make_current() const;
  void validate_active_batch(int64_t active_batch) const;
  void configure_bins(int geometry);
  void configure_type2_bins();
  void configure_tiles();
  // Smallest active batch on the tensor cores: 1 when the configuration
  // forces them, else the tuned threshold (at least kTcMinBatch).
  int64_t tensor_min_batch() const {
    return tc_min_batch_ == 1 ? 1 : std::max<int64_t>(tc_min_batch_, tuned_.tensor_min_batch);
  }
  // The reference's bin order of a type-1 point set (ref_perm_, ref_keys_,
  // ref_offsets_): its points outside the fold's reach back in bin 0.
  void reference_order(cudaStream_t stream);
  cufftHandle fft_for(int batch);
  void run_fft(void* fine, int batch, int direction, cudaStream_t stream);
  void execute_f32(int batch, const void* input, void* output, uint64_t out_bytes,
                   cudaStream_t stream);
  void execute_f64(int batch, const void* input, void* output, uint64_t in_bytes,
                   uint64_t out_bytes, cudaStream_t stream);
  // Plans of 4 to 8 dimensions: generic spreading / interpolation and an FFT
  // over groups of up to three axes.
  void execute_nd(int batch, const void* input, void* output, void* fine, int direction, cudaStream_t stream);
  void spread_nd(int batch, const void* strengths, void* grid, cudaStream_t stream);
  void run_fft_nd(void* fine, int batch, int direction, cudaStream_t stream);
  size_t scalar_bytes() const;

  int type_ = 1;
  int dim_ = 1;
  int64_t modes_[8] = {1, 1, 1, 1, 1, 1, 1, 1};
  int64_t batch_ = 1;
  double eps_ = 1e-6;
  int isign_ = 1;
  int mode_order_ = 0;
  double sigma_ = 2.0;
  int precision_ = B200NUFFT_PRECISION_F32;
  int device_ = 0;
  EsKernel kernel_;
  EsHornerTable horner_;
  std::vector<int64_t> fine_;
  std::vector<std::vector<double>> phi_hat_;
  SpreadLayout layout_;
  int64_t mode_count_ = 1;
  int64_t fine_count_ = 1;
  GridParams grid_{};
  ModeParams modes_params_{};
  SpreadParams spread_{};

  bool has_device_ = true;
  StageTimer timer_;
  DeviceBuffer amplitudes_;
  DeviceBuffer horner_device_;
  // Df64 plans: f64 copies of the caller's double-float coordinates and values.
  DeviceBuffer points64_, input64_, output64_;
  DeviceBuffer fine_grid_;
  std::map<int, cufftHandle> ffts_;
  // 2D and 3D f32 plans with power-of-two fine axes: the fused transforms
  // (fused_fft.cu), their twiddle tables and the buffer of the pass along
  // axis 0 (the fine grid serves as the second buffer of 3D plans).
  bool fused_fft_active_ = false;
  FusedFftParams fused_fft_{};
  DeviceBuffer fused_fft_twiddles_, fused_fft_rows_;
  // Type 1: the fold runs inside the fused pass along axis 0, for fewer than
  // eight vectors (batches fold eight vectors per thread, sharing the tile
  // lookups, and keep cuFFT) on grids above kWarpFoldCells cells (smaller
  // ones keep the warp fold of crowded tiles).
  bool fused_fold(int batch) const { return fused_fft_active_ && fine_count_ > kWarpFoldCells && batch < 8; }
  // Plans of 4 to 8 dimensions.
  NdParams nd_{};
  DeviceBuffer nd_acc_;                       // 64-bit integer fine grids of type 1
  std::map<int64_t, cufftHandle> nd_ffts_;    // by first axis of the group and batch

  // Remembered points and their bin order.
  int64_t point_count_ = -1;
  const void* points_ = nullptr;
  int geometry_ = -1;
  uint64_t bins_ = 0;
  uint32_t* perm_ = nullptr;
  uint32_t* sorted_keys_ = nullptr;
  DeviceBuffer keys_a_, keys_b_, vals_a_, vals_b_, hist_, status_, counters_, offsets_;
  DeviceBuffer sorted_points_;
  DeviceBuffer valid_mask_;  // type-1 plans: points within the fold's reach, caller order
  DeviceBuffer ref_perm_, ref_keys_, ref_offsets_;  // type-1 plans: the reference's order, on request
  DeviceBuffer part_cap_;    // type-1 plans: records per part, sized on the device
  DeviceBuffer windows_;  // f32 plans: PreparedWindow per slot
  DeviceBuffer inverse_;  // batched 2D f32 type-2 plans: slot of every point
  // 2D type-2 plans: the bins' slots in parts of at most kInterpPartSlots
  // (work items of the bin interpolation kernels).
  DeviceBuffer interp_parts_, interp_part_start_, interp_part_bin_;
  int64_t interp_parts_bound_ = 0;
  void prepare_interp_parts(const uint32_t* offsets, cudaStream_t stream);
  InterpParts interp_parts() const;
  DeviceBuffer staged_;   // batched 2D f32 type-2 plans: values in slot order
  // 3D type-2 plans: the interpolation's point order (support starts'
  // (z, y) rows, 8-cell x segments), in which the sorted coordinates (and the
  // prepared windows of f32 plans) are kept; the reference's bin order stays
  // in perm_.
  bool rows_order_ = false;
  DeviceBuffer rows_perm_, rows_offsets_;
  const uint32_t* interp_perm() const {
    return rows_order_ ? static_cast<const uint32_t*>(rows_perm_.get()) : perm_;
  }
  // The bins of that order (one cell along y and z, 8 along x) and their count.
  GridParams rows_grid(uint64_t* bins) const;
  // Copies a sort's permutation into rows_perm_ (the sort buffers are reused).
  void keep_rows_order(const uint32_t* order, int64_t count, cudaStream_t stream);
  // The reference's bin order (perm_, offsets_, sorted_keys_) of a point set
  // kept in the row order is sorted only when it is asked for: the
  // interpolation does not read it.
  bool bin_order_pending_ = false;
  DeviceBuffer unsorted_;  // the coordinates back in the caller's order, for that sort
  void finish_bin_order(cudaStream_t stream);
  SortBuffers sort_buffers(int64_t count);

  // Spreading state.
  DeviceBuffer parts_, part_start_, max_bits_, scratch_, candidates_;
  DeviceBuffer warp_segments_;     // 3D f32: segment table of the warp spreader
  int32_t warp_layout_key_[4] = {};  // width and padded tile of that table
  int64_t part_upper_bound_ = 0;
  std::vector<int2> host_candidates_;
  int64_t candidate_tile_[3] = {0, 0, 0};
  int32_t dest_fold_ = 0;  // SpreadParams::dest_fold of the kept candidate table

  // Tensor-core spreading (2D f32 type-1 plans of batch >= kTcMinBatch):
  // enabled by the configuration, active when the chosen bins allow it.
  bool tc_enabled_ = false;
  bool tc_active_ = false;
  int64_t tc_min_batch_ = kTcMinBatch;  // smallest active batch run on the tensor cores
  b200nufft_tuning tuned_{0, 4, 1, kTcMinBatch};  // the tuning of the last point set
  DeviceBuffer tc_weights_, tc_inverse_, tc_tile_chunks_, tc_tile_chunk_start_, tc_chunks_;
  DeviceBuffer tc_parts_, tc_part_start_, tc_packed_;
  int64_t tc_part_upper_bound_ = 0;

  // Tensor-core interpolation (2D f32 type-2 plans of batch >= kTcMinBatch):
  // the points ordered by exact support start in bins of 8 x 1 cells, their
  // window records, the slot of every point and the chunk tables.
  bool tc2_enabled_ = false;
  bool tc2_active_ = false;
  GridParams tc2_grid_{};
  DeviceBuffer tc2_offsets_, tc2_weights_, tc2_inverse_, tc2_tile_chunks_, tc2_tile_chunk_start_, tc2_chunks_;
  DeviceBuffer tc2_parts_, tc2_part_start_;
  DeviceBuffer tc2_vector_max_;  // batch words: largest grid magnitude of every vector
  int64_t tc2_part_upper_bound_ = 0;
};

}  // namespace b200nufft
