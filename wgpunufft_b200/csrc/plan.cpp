// Type-1 / type-2 plan: creation (src/plan.rs:658-694), point preparation
// (src/plan.rs:890-925) and execution (src/plan.rs:931-977, 1183-1229).
#include "plan.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

#include "fused_fft.h"
#include "tuning.h"
#include "util.h"

namespace b200nufft {

namespace {

constexpr double kTwoPi = 6.28318530717958647692;
// Records of one spreading subproblem, at most.
constexpr int32_t kPartCap = 4096;
// Padded tile bytes a spreading CTA may hold, so that two fit on an SM.
constexpr int64_t kTileBytesTarget = 100 * 1024;
// Points one plan can bin: look-back words hold 30-bit counts.
constexpr int64_t kMaxPoints = (int64_t(1) << 30) - 1;
// Active batches from which 2D f32 type-2 plans stage bin regions in shared memory.
constexpr int kInterpBinsMinBatch = 8;

int64_t mode_for_storage_index(int order, int64_t index, int64_t length) {
  // src/direct.rs:120-131
  if (order == B200NUFFT_MODE_ORDER_CENTERED) return index - length / 2;
  return index < (length + 1) / 2 ? index : index - length;
}

int64_t pow2_ceil(int64_t v) {
  int64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

int ilog2(int64_t v) {
  int s = 0;
  while ((int64_t(1) << s) < v) ++s;
  return s;
}

// config.rs:252-284: an F32 plan whose rounding, amplified by deconvolution,
// would miss the tolerance by far is rejected.
void validate_f32_rounding(const int64_t* modes, int dim, double eps, double sigma,
                           const std::vector<std::vector<double>>& coefficients) {
  double estimate = static_cast<double>(std::numeric_limits<float>::epsilon()) / 2.0;
  for (int a = 0; a < dim; ++a) {
    const auto& axis = coefficients[a];
    if (axis.empty()) continue;
    const double center = axis[0];
    const int64_t half = modes[a] / 2;
    double sum = 0.0;
    for (int64_t index = 0; index < modes[a]; ++index) {
      const int64_t magnitude = index > half ? index - half : half - index;
      const double value =
          magnitude < static_cast<int64_t>(axis.size()) ? std::fabs(axis[magnitude]) : 0.0;
      sum += value > 0.0 ? (center / value) * (center / value)
                         : std::numeric_limits<double>::infinity();
    }
    estimate *= std::sqrt(sum / static_cast<double>(modes[a]));
  }
  if (estimate > 10.0 * eps && estimate > 1.0e-5) {
    throw NufftFailure{B200NUFFT_F32_TOLERANCE_UNREACHABLE,
                       "f32 rounding amplified by the deconvolution (estimated error " +
                           std::to_string(estimate) + ") misses eps " + std::to_string(eps) +
                           " at sigma " + std::to_string(sigma) +
                           "; use sigma = 2, a larger tolerance, or f64"};
  }
}

}  // namespace

NufftPlan::NufftPlan(const b200nufft_config& c, bool with_device) : has_device_(with_device) {
  if (c.type != 1 && c.type != 2) {
    throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "plan type must be 1 or 2"};
  }
  type_ = c.type;
  if (c.batch <= 0) {
    throw NufftFailure{B200NUFFT_INVALID_BATCH, "batch must be at least one"};
  }
  if (c.dimensions < 1 || c.dimensions > 8) {
    throw NufftFailure{B200NUFFT_INVALID_DIMENSIONS, "dimensions must lie in 1..8"};
  }
  if (c.dimensions > B200NUFFT_MAX_DIMENSIONS) {
    throw NufftFailure{B200NUFFT_GPU_DIMENSIONS_UNSUPPORTED,
                       "GPU plans support 1 to 8 dimensions"};
  }
  dim_ = c.dimensions;
  batch_ = c.batch;
  mode_count_ = 1;
  for (int a = 0; a < dim_; ++a) {
    if (c.n_modes[a] <= 0) {
      throw NufftFailure{B200NUFFT_ZERO_MODE, "axis " + std::to_string(a) + " has no modes"};
    }
    modes_[a] = c.n_modes[a];
    if (mode_count_ > std::numeric_limits<int64_t>::max() / modes_[a]) {
      throw NufftFailure{B200NUFFT_LENGTH_OVERFLOW, "total Fourier mode count"};
    }
    mode_count_ *= modes_[a];
  }
  if (mode_count_ > std::numeric_limits<int64_t>::max() / batch_) {
    throw NufftFailure{B200NUFFT_LENGTH_OVERFLOW, "batched Fourier mode count"};
  }
  eps_ = c.eps;
  isign_ = c.isign >= 0 ? 1 : -1;
  if (c.mode_order != B200NUFFT_MODE_ORDER_CENTERED && c.mode_order != B200NUFFT_MODE_ORDER_FFT) {
    throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "mode order must be 0 (centered) or 1 (FFT)"};
  }
  mode_order_ = c.mode_order;
  sigma_ = c.sigma == 0.0 ? 2.0 : c.sigma;
  precision_ = c.precision == 0 ? B200NUFFT_PRECISION_F32 : c.precision;
  if (precision_ != B200NUFFT_PRECISION_F32 && precision_ != B200NUFFT_PRECISION_F64 &&
      precision_ != B200NUFFT_PRECISION_DF64) {
    throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "precision must be F64 (1), DF64 (2) or F32 (3)"};
  }
  kernel_ = EsKernel::for_tolerance(eps_, sigma_);
  if (c.spread_method < B200NUFFT_SPREAD_AUTO || c.spread_method > B200NUFFT_SPREAD_TENSOR_CORES) {
    throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "spread method must be 0 (auto), 1 (CUDA cores) or 2 (tensor cores)"};
  }
  const bool f32 = precision_ == B200NUFFT_PRECISION_F32;
  const bool tc1_qualifies = type_ == 1 && dim_ == 2 && f32 && kernel_.width <= kTcMaxWidth;
  const bool tc2_qualifies = type_ == 2 && dim_ == 2 && f32 && kernel_.width <= kTi2MaxWidth;
  if (c.spread_method == B200NUFFT_SPREAD_TENSOR_CORES && !tc1_qualifies && !tc2_qualifies) {
    throw NufftFailure{B200NUFFT_INVALID_ARGUMENT,
                       "tensor cores need a 2D f32 plan with a window of at most 8 points (type 1) or 7 (type 2)"};
  }
  const bool tc_requested = (c.spread_method == B200NUFFT_SPREAD_AUTO && batch_ >= kTcMinBatch) ||
                            c.spread_method == B200NUFFT_SPREAD_TENSOR_CORES;
  tc_enabled_ = tc1_qualifies && tc_requested;
  tc2_enabled_ = tc2_qualifies && tc_requested;
  tc_min_batch_ = c.spread_method == B200NUFFT_SPREAD_TENSOR_CORES ? 1 : kTcMinBatch;
  fine_count_ = 1;
  for (int a = 0; a < dim_; ++a) {
    const uint64_t n = select_fine_grid_size(static_cast<uint64_t>(modes_[a]), sigma_, kernel_.width);
    fine_.push_back(static_cast<int64_t>(n));
  }
  const bool horner = precision_ != B200NUFFT_PRECISION_F32;
  if (horner) horner_ = EsHornerTable::fit(kernel_);
  for (int a = 0; a < dim_; ++a) {
    phi_hat_.push_back(centered_fourier_coefficients(kernel_, static_cast<size_t>(fine_[a]),
                                                     horner ? &horner_ : nullptr));
  }
  if (precision_ == B200NUFFT_PRECISION_F32) {
    validate_f32_rounding(modes_, dim_, eps_, sigma_, phi_hat_);
    // src/gpu_type1_nd.rs:68-73: support indices must stay exact in f32.
    const int64_t maximum = (int64_t(1) << 24) - kernel_.width;
    for (int a = 0; a < dim_; ++a) {
      if (fine_[a] > maximum) {
        throw NufftFailure{B200NUFFT_GPU_FINE_GRID_INDEX_UNSUPPORTED,
                           "fine-grid axis of " + std::to_string(fine_[a]) +
                               " cells exceeds the f32-exact maximum " + std::to_string(maximum)};
      }
    }
  }
  for (int a = 0; a < dim_; ++a) {
    if (fine_count_ > std::numeric_limits<int64_t>::max() / fine_[a]) {
      throw NufftFailure{B200NUFFT_LENGTH_OVERFLOW, "fine-grid element count"};
    }
    fine_count_ *= fine_[a];
  }
  if (dim_ <= 3) layout_ = SpreadLayout::for_grid(kernel_.width, fine_,
                                   precision_ == B200NUFFT_PRECISION_F32 ? LayoutPrecision::F32
                                   : precision_ == B200NUFFT_PRECISION_F64 ? LayoutPrecision::F64
                                                                           : LayoutPrecision::Df64);

  // Deconvolution amplitudes prod_a 1 / phi_hat_a(|k_a|), divided in f64 in
  // axis order and, for f32 plans, rounded once (mode_amplitudes_nd and
  // mode_amplitudes_nd_f64, src/gpu_nd.rs:910-990).
  std::vector<double> amplitudes(static_cast<size_t>(mode_count_));
  for (int64_t flat = 0; flat < mode_count_; ++flat) {
    int64_t rest = flat;
    double amplitude = 1.0;
    for (int a = 0; a < dim_; ++a) {
      const int64_t index = rest % modes_[a];
      rest /= modes_[a];
      const int64_t mode = mode_for_storage_index(mode_order_, index, modes_[a]);
      const double coefficient = phi_hat_[a][static_cast<size_t>(mode < 0 ? -mode : mode)];
      if (!std::isfinite(coefficient) || coefficient == 0.0) {
        throw NufftFailure{B200NUFFT_INVALID_KERNEL_FOURIER_COEFFICIENT,
                           "kernel Fourier coefficient of mode " + std::to_string(mode) +
                               " is zero or not finite"};
      }
      amplitude /= coefficient;
    }
    if (precision_ == B200NUFFT_PRECISION_F32 && !std::isfinite(static_cast<float>(amplitude))) {
      throw NufftFailure{B200NUFFT_INVALID_KERNEL_FOURIER_COEFFICIENT,
                         "deconvolution amplitude overflows f32"};
    }
    if (!std::isfinite(amplitude)) {
      throw NufftFailure{B200NUFFT_INVALID_KERNEL_FOURIER_COEFFICIENT,
                         "deconvolution amplitude is not finite"};
    }
    amplitudes[static_cast<size_t>(flat)] = amplitude;
  }
  if (!with_device) return;
  int current = 0;
  check_cuda(cudaGetDevice(&current), "current device");
  device_ = c.device < 0 ? current : c.device;
  make_current();
  if (precision_ == B200NUFFT_PRECISION_F32) {
    std::vector<float> rounded(amplitudes.begin(), amplitudes.end());
    void* amp = amplitudes_.reserve(rounded.size() * sizeof(float), "deconvolution amplitudes");
    check_cuda(cudaMemcpy(amp, rounded.data(), rounded.size() * sizeof(float), cudaMemcpyHostToDevice),
               "upload deconvolution amplitudes");
  } else {
    void* amp = amplitudes_.reserve(amplitudes.size() * sizeof(double), "deconvolution amplitudes");
    check_cuda(cudaMemcpy(amp, amplitudes.data(), amplitudes.size() * sizeof(double),
                          cudaMemcpyHostToDevice),
               "upload deconvolution amplitudes");
    void* table = horner_device_.reserve(horner_.coefficients.size() * sizeof(double), "Horner table");
    check_cuda(cudaMemcpy(table, horner_.coefficients.data(),
                          horner_.coefficients.size() * sizeof(double), cudaMemcpyHostToDevice),
               "upload Horner table");
  }

  std::memset(&grid_, 0, sizeof(grid_));
  grid_.dimensions = dim_;
  grid_.width = kernel_.width;
  grid_.half_width = static_cast<float>(kernel_.half_width());
  grid_.beta = static_cast<float>(kernel_.beta);
  grid_.fine_count = fine_count_;
  grid_.half_width64 = kernel_.half_width();
  grid_.horner = horner ? static_cast<const double*>(horner_device_.get()) : nullptr;
  grid_.horner_rows = horner ? horner_.coefficient_count : 0;
  if (!horner && kernel_.width + 3 <= kHornerRows32 && kernel_.width <= kHornerWidth32) {
    // f32 plans: the same panels rounded to f32, bottom-aligned in w + 3 rows.
    const EsHornerTable table = EsHornerTable::fit(kernel_);
    const int rows = table.coefficient_count;
    const int first = kHornerRows32 - rows;
    for (int r = 0; r < rows; ++r) {
      for (int j = 0; j < kernel_.width; ++j) {
        grid_.horner32[first + r][j] = static_cast<float>(table.coefficients[r * kernel_.width + j]);
      }
    }
  }
  if (dim_ > 3) {
    // Plans of 4 to 8 dimensions: fold constants for every axis, no bins.
    nd_.dimensions = dim_;
    nd_.width = kernel_.width;
    nd_.f32 = precision_ == B200NUFFT_PRECISION_F32 ? 1 : 0;
    nd_.half_width = static_cast<float>(kernel_.half_width());
    nd_.beta = static_cast<float>(kernel_.beta);
    nd_.half_width64 = kernel_.half_width();
    nd_.fine_count = fine_count_;
    nd_.horner = grid_.horner;
    nd_.horner_rows = grid_.horner_rows;
    for (int a = 0; a < dim_; ++a) {
      const double scale = static_cast<double>(fine_[a]) / kTwoPi;
      FoldAxis& axis = nd_.axis[a];
      axis.scale_hi = static_cast<float>(scale);
      axis.scale_lo = static_cast<float>(scale - static_cast<double>(axis.scale_hi));
      axis.origin = static_cast<float>(fine_[a] / 2);
      axis.length_f = static_cast<float>(fine_[a]);
      axis.length = static_cast<int32_t>(fine_[a]);
      nd_.axis64[a].scale = scale;
      nd_.axis64[a].origin = static_cast<double>(fine_[a] / 2);
      nd_.axis64[a].length = static_cast<double>(fine_[a]);
      nd_.fine[a] = fine_[a];
    }
  }
  for (int a = 0; a < std::min(dim_, 3); ++a) {
    const double scale = static_cast<double>(fine_[a]) / kTwoPi;
    FoldAxis& axis = grid_.axis[a];
    axis.scale_hi = static_cast<float>(scale);
    axis.scale_lo = static_cast<float>(scale - static_cast<double>(axis.scale_hi));
    axis.origin = static_cast<float>(fine_[a] / 2);
    axis.length_f = static_cast<float>(fine_[a]);
    axis.length = static_cast<int32_t>(fine_[a]);
    grid_.axis64[a].scale = scale;
    grid_.axis64[a].origin = static_cast<double>(fine_[a] / 2);
    grid_.axis64[a].length = static_cast<double>(fine_[a]);
    grid_.fine[a] = fine_[a];
  }
  std::memset(&modes_params_, 0, sizeof(modes_params_));
  modes_params_.dimensions = dim_;
  modes_params_.centered = mode_order_ == B200NUFFT_MODE_ORDER_CENTERED ? 1 : 0;
  modes_params_.mode_count = mode_count_;
  modes_params_.fine_count = fine_count_;
  for (int a = 0; a < dim_; ++a) {
    modes_params_.modes[a] = modes_[a];
    modes_params_.fine[a] = fine_[a];
  }
  fine_grid_.reserve(static_cast<size_t>(batch_) * fine_count_ * 2 * scalar_bytes(), "fine grid");
  // 2D and 3D f32 plans with power-of-two fine axes: the fused transforms and
  // their twiddle tables, of the plan's exponent sign (isign >= 0: +1).
  fused_fft_active_ = precision_ == B200NUFFT_PRECISION_F32 && fused_fft_enabled() &&
                      fused_fft_supported(dim_, fine_.data(), modes_);
  if (fused_fft_active_) {
    std::memset(&fused_fft_, 0, sizeof(fused_fft_));
    fused_fft_.dims = dim_;
    fused_fft_.sign = isign_ >= 0 ? 1 : -1;
    fused_fft_.centered = modes_params_.centered;
    size_t offsets[3] = {0, 0, 0};
    std::vector<float2> tables;
    for (int a = 0; a < dim_; ++a) {
      int k = 0;
      while ((int64_t{1} << k) < fine_[a]) ++k;
      fused_fft_.log2n[a] = k;
      fused_fft_.modes[a] = static_cast<int32_t>(modes_[a]);
      const std::vector<float2> t = fused_fft_twiddles(fine_[a], fused_fft_.sign);
      offsets[a] = tables.size();
      tables.insert(tables.end(), t.begin(), t.end());
    }
    float2* dev = static_cast<float2*>(fused_fft_twiddles_.reserve(tables.size() * sizeof(float2), "twiddles"));
    check_cuda(cudaMemcpy(dev, tables.data(), tables.size() * sizeof(float2), cudaMemcpyHostToDevice),
               "upload twiddles");
    for (int a = 0; a < dim_; ++a) fused_fft_.twiddle[a] = dev + offsets[a];
  }
  counters_.reserve(8 * sizeof(uint32_t), "sort tickets");
  check_cuda(cudaMemset(counters_.get(), 0, 8 * sizeof(uint32_t)), "clear sort tickets");
  hist_.reserve(4 * 256 * sizeof(uint32_t), "digit histograms");
  max_bits_.reserve(static_cast<size_t>(batch_) * sizeof(uint64_t), "strength maxima");
}

NufftPlan::~NufftPlan() {
  if (!has_device_) return;
  cudaSetDevice(device_);
  cudaDeviceSynchronize();
  for (auto& entry : ffts_) cufftDestroy(entry.second);
  for (auto& entry : nd_ffts_) cufftDestroy(entry.second);
}

void NufftPlan::make_current() const { check_cuda(cudaSetDevice(device_), "select plan device"); }

size_t NufftPlan::scalar_bytes() const {
  return precision_ == B200NUFFT_PRECISION_F32 ? 4 : 8;
}

void NufftPlan::validate_active_batch(int64_t active_batch) const {
  if (active_batch <= 0 || active_batch > batch_) {
    throw NufftFailure{B200NUFFT_INVALID_BATCH, "active batch " + std::to_string(active_batch) +
                                                    " outside 1.." + std::to_string(batch_)};
  }
}

uint64_t NufftPlan::required_point_bytes(int64_t count) const {
  if (count < 0) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "negative point count"};
  const size_t coord = precision_ == B200NUFFT_PRECISION_F32 ? 4 : 8;
  return static_cast<uint64_t>(count) * dim_ * coord;
}

uint64_t NufftPlan::required_input_bytes(int64_t count, int64_t active_batch) const {
  validate_active_batch(active_batch);
  const uint64_t elements = type_ == 1 ? static_cast<uint64_t>(count) : static_cast<uint64_t>(mode_count_);
  return elements * active_batch * 2 * (precision_ == B200NUFFT_PRECISION_F32 ? 4 : 8);
}

uint64_t NufftPlan::required_output_bytes(int64_t count, int64_t active_batch) const {
  validate_active_batch(active_batch);
  const uint64_t elements = type_ == 1 ? static_cast<uint64_t>(mode_count_) : static_cast<uint64_t>(count);
  return elements * active_batch * 2 * (precision_ == B200NUFFT_PRECISION_F32 ? 4 : 8);
}

void NufftPlan::configure_bins(int geometry) {
  const BinGeometry& g = layout_.geometries[static_cast<size_t>(geometry)];
  uint64_t stride = 1;
  for (int a = 0; a < dim_; ++a) {
    grid_.axis[a].shift = ilog2(g.side[a]);
    grid_.axis[a].bins = static_cast<uint32_t>(g.bins[a]);
    grid_.axis[a].stride = static_cast<uint32_t>(stride);
    stride *= static_cast<uint64_t>(g.bins[a]);
  }
  bins_ = stride;
}

void NufftPlan::configure_type2_bins() {
  // f32: interpolation bins of 8 cells per axis in 1D and 2D and 4 in 3D
  // (src/gpu.rs:19, src/gpu_2d.rs:22, src/gpu_3d.rs:25). f64 and Df64: the
  // rank-generic bins of type2_bin_shape (src/gpu_nd.rs:566-586), 4 cells per
  // axis, doubled from the last axis backwards while above 2^24 bins.
  int64_t sides[3] = {1, 1, 1};
  if (precision_ == B200NUFFT_PRECISION_F32) {
    for (int a = 0; a < dim_; ++a) sides[a] = dim_ == 3 ? 4 : 8;
  } else {
    for (int a = 0; a < dim_; ++a) sides[a] = 4;
    auto count = [&]() {
      int64_t total = 1;
      for (int a = 0; a < dim_; ++a) total *= (fine_[a] + sides[a] - 1) / sides[a];
      return total;
    };
    int axis = dim_;
    while (count() > (int64_t(1) << 24)) {
      axis = axis == 0 ? dim_ - 1 : axis - 1;
      sides[axis] *= 2;
    }
  }
  uint64_t stride = 1;
  for (int a = 0; a < dim_; ++a) {
    const int64_t side = sides[a];
    const int64_t bins = (fine_[a] + side - 1) / side;
    grid_.axis[a].shift = ilog2(side);
    grid_.axis[a].bins = static_cast<uint32_t>(bins);
    grid_.axis[a].stride = static_cast<uint32_t>(stride);
    stride *= static_cast<uint64_t>(bins);
  }
  bins_ = stride;
}

void NufftPlan::configure_tiles() {
  SpreadParams& sp = spread_;
  int64_t kept_candidate_base[3];
  int32_t kept_candidate_count[3];
  for (int a = 0; a < 3; ++a) {
    kept_candidate_base[a] = sp.candidate_base[a];
    kept_candidate_count[a] = sp.candidate_count[a];
  }
  std::memset(&sp, 0, sizeof(sp));
  sp.grid = grid_;
  const int w = kernel_.width;
  const b200nufft_tuning tuning = tuned_;
  int64_t tile[3] = {1, 1, 1};
  if (dim_ == 1) tile[0] = 1024;
  // 2D f32 register runs (w <= 7) slide along the rows of 64 x 64 tiles:
  // a thread's range of consecutive records then spans more starts of a row.
  const bool runs2d = dim_ == 2 && precision_ == B200NUFFT_PRECISION_F32 && 2 * w * w * 4 < 400;
  if (dim_ == 2) tile[0] = tile[1] = runs2d ? 64 : 32;
  if (dim_ == 3) tile[0] = tile[1] = tile[2] = 16;
  if (tuning.tile > 0) {
    for (int a = 0; a < dim_; ++a) tile[a] = tuning.tile;
  }
  for (int a = 0; a < dim_; ++a) tile[a] = std::min(tile[a], pow2_ceil(fine_[a]));
  // The tensor-core spreader needs one-cell bin rows, column bins of at most
  // 8 cells, and its own tile shape (16 cells x 22 - w rows).
  tc_active_ = tc_enabled_ && grid_.axis[1].shift == 0 && grid_.axis[0].shift <= 3;
  if (tc_active_) {
    tile[0] = kTcTileX;
    tile[1] = tc_tile_rows(w);
  }
  auto padded_bytes = [&]() {
    int64_t cells = 1;
    for (int a = 0; a < dim_; ++a) cells *= tile[a] + w - 1;
    return cells * 16;
  };
  while (!tc_active_ && padded_bytes() > kTileBytesTarget) {
    int largest = dim_ - 1;
    for (int a = dim_ - 1; a >= 0; --a) {
      if (tile[a] > tile[largest]) largest = a;
    }
    if (tile[largest] == 1) break;
    tile[largest] /= 2;
  }
  sp.tile_count = 1;
  sp.padded_cells = 1;
  int64_t tiles_per_bin = 1;
  int64_t rows = 1;
  for (int a = 0; a < dim_; ++a) {
    sp.tile[a] = static_cast<int32_t>(tile[a]);
    sp.pad[a] = static_cast<int32_t>(tile[a] + w - 1);
    sp.ntiles[a] = static_cast<int32_t>((fine_[a] + tile[a] - 1) / tile[a]);
    sp.tile_count *= sp.ntiles[a];
    sp.padded_cells *= sp.pad[a];
    const int64_t side = int64_t(1) << grid_.axis[a].shift;
    if (side > tile[a]) tiles_per_bin *= side / tile[a];
    if (a > 0) rows *= std::max<int64_t>(1, tile[a] / side);
  }
  for (int a = dim_; a < 3; ++a) {
    sp.tile[a] = 1;
    sp.pad[a] = 1;
    sp.ntiles[a] = 1;
  }
  if (rows > kMaxTileRows) {
    throw NufftFailure{B200NUFFT_INTERNAL, "spreading tile spans too many bin rows"};
  }
  // 3D f32 tiles of widths 5 to 8: the shared-memory pitches and the segment
  // table of the warp spreader (uploaded when the tile shape changes).
  if (dim_ == 3 && precision_ == B200NUFFT_PRECISION_F32 && w >= kWarpMinWidth && w <= kWarpMaxWidth) {
    uint32_t table[32 * warp_max_rounds()];
    int32_t pitch0 = 0, pitch01 = 0;
    if (spread_warp_layout(w, sp.pad, pitch0, pitch01, table)) {
      const int32_t key[4] = {w, sp.pad[0], sp.pad[1], sp.pad[2]};
      const size_t bytes = sizeof(uint32_t) * 32 * warp_rounds(w);
      if (std::memcmp(key, warp_layout_key_, sizeof(key)) != 0) {
        void* dst = warp_segments_.reserve(bytes, "warp segment table");
        check_cuda(cudaMemcpy(dst, table, bytes, cudaMemcpyHostToDevice), "upload warp segment table");
        std::memcpy(warp_layout_key_, key, sizeof(key));
      }
      sp.pitch0 = pitch0;
      sp.pitch01 = pitch01;
      sp.span = pitch01 * sp.pad[2];
      sp.warp_segments = static_cast<const uint32_t*>(warp_segments_.get());
    }
  }
  // Parts of at most kPartCap records (f64), fewer for small point sets so that
  // about four CTAs per SM have work. On one-cell bins holding eight or more
  // points per cell, consecutive records share their start: parts sized for
  // one CTA per SM give every thread runs several times longer, and the
  // warps' flushes, which would otherwise all land on the same few windows,
  // fall on more cells and come less often.
  // (Register runs are taken in 1D, and in 2D while the 2 w^2 accumulators
  // fit: spread_run in spread.cu.)
  const int64_t real_bytes = precision_ == B200NUFFT_PRECISION_F32 ? 4 : 8;
  const bool runs = dim_ == 1 || (dim_ == 2 && 2 * w * w * real_bytes < 400);
  bool one_cell_bins = true;
  for (int a = 0; a < dim_; ++a) one_cell_bins = one_cell_bins && grid_.axis[a].shift == 0;
  const bool crowded = runs && one_cell_bins && point_count_ >= 8 * grid_.fine_count;
  const int64_t spread_ctas = (crowded ? tuning.crowded_ctas_per_sm : tuning.ctas_per_sm) * int64_t{148};
  int64_t cap = (std::max<int64_t>(point_count_, 1) + spread_ctas - 1) / spread_ctas;
  // 3D parts stay within the 2048 records that crowded tiles bucket in shared
  // memory; 1D and 2D f32 parts take up to 16384 records, so that a thread's
  // register runs can reach 64 records in crowded tiles.
  const int64_t part_cap = dim_ == 3 ? 2048 : (precision_ == B200NUFFT_PRECISION_F32 ? 16384 : kPartCap);
  cap = std::min<int64_t>(part_cap, std::max<int64_t>(256, (cap + 255) / 256 * 256));
  sp.part_cap = static_cast<int32_t>(cap);
  // The device sizes the parts from the points within reach (the others sort
  // after every bin), so that such points change no part; the host bounds the
  // parts for any count up to point_count_: valid / cap(valid) is at most
  // 4 x 148, or point_count_ / part_cap once the cap saturates.
  const int64_t most_ctas = std::max(tuning.ctas_per_sm, tuning.crowded_ctas_per_sm) * int64_t{148};
  int64_t records_per_cap = most_ctas;
  if (type_ == 1) {
    sp.part_cap_device = static_cast<int32_t*>(part_cap_.reserve(sizeof(int32_t), "part cap"));
    sp.cap_ctas = tuning.ctas_per_sm * 148;
    sp.cap_ctas_crowded = tuning.crowded_ctas_per_sm * 148;
    sp.cap_max = static_cast<int32_t>(part_cap);
    sp.crowded_points = runs && one_cell_bins ? 8 * grid_.fine_count : std::numeric_limits<int64_t>::max();
    sp.cap_bins = bins_;
    records_per_cap = std::max<int64_t>(most_ctas, (std::max<int64_t>(point_count_, 0) + part_cap - 1) / part_cap);
  }
  const int64_t part_bound = type_ == 1 ? sp.tile_count + tiles_per_bin * records_per_cap + 1
                                        : sp.tile_count + (std::max<int64_t>(point_count_, 0) * tiles_per_bin +
                                                           sp.part_cap - 1) / sp.part_cap + 1;
  // Candidate (tile, local) pairs of every coordinate of every axis: tile t
  // covers cells (t * tile + l) mod n for l < pad. They depend on the grid
  // and tile shape only, so later point sets reuse them.
  if (!host_candidates_.empty() && candidate_tile_[0] == tile[0] && candidate_tile_[1] == tile[1] &&
      candidate_tile_[2] == tile[2]) {
    for (int a = 0; a < 3; ++a) {
      sp.candidate_base[a] = kept_candidate_base[a];
      sp.candidate_count[a] = kept_candidate_count[a];
    }
    sp.dest_fold = dest_fold_;
    part_upper_bound_ = part_bound;
    return;
  }
  host_candidates_.clear();
  for (int a = 0; a < 3; ++a) candidate_tile_[a] = tile[a];
  bool dest_fold = dim_ == 3 && tile[0] == 16 && tile[1] == 16 && tile[2] % 4 == 0;
  for (int a = 0; a < dim_; ++a) {
    const int64_t n = fine_[a];
    std::vector<std::vector<int2>> lists(static_cast<size_t>(n));
    for (int64_t t = 0; t < sp.ntiles[a]; ++t) {
      for (int64_t l = 0; l < sp.pad[a]; ++l) {
        const int64_t cell = (t * tile[a] + l) % n;
        lists[static_cast<size_t>(cell)].push_back(make_int2(static_cast<int>(t), static_cast<int>(l)));
      }
    }
    size_t most = 1;
    for (const auto& list : lists) most = std::max(most, list.size());
    // The destination-tile fold walks, per axis, the candidates of the
    // tile's first cell in their order: every cell of the tile must list an
    // ordered part of them, each tile once.
    dest_fold = dest_fold && most <= 2;
    for (int64_t t = 0; dest_fold && t < sp.ntiles[a]; ++t) {
      const auto& first = lists[static_cast<size_t>(t * tile[a])];
      if (first.size() == 2 && first[0].x == first[1].x) dest_fold = false;
      for (int64_t c = t * tile[a]; dest_fold && c < std::min<int64_t>((t + 1) * tile[a], n); ++c) {
        size_t at = 0;
        for (const int2& e : lists[static_cast<size_t>(c)]) {
          while (at < first.size() && first[at].x != e.x) ++at;
          if (at == first.size()) {
            dest_fold = false;
            break;
          }
          ++at;
        }
      }
    }
    sp.candidate_base[a] = static_cast<int64_t>(host_candidates_.size());
    sp.candidate_count[a] = static_cast<int32_t>(most);
    for (const auto& list : lists) {
      for (size_t k = 0; k < most; ++k) {
        host_candidates_.push_back(k < list.size() ? list[k] : make_int2(-1, -1));
      }
    }
  }
  dest_fold_ = dest_fold ? 1 : 0;
  sp.dest_fold = dest_fold_;
  void* cand = candidates_.reserve(host_candidates_.size() * sizeof(int2), "fold candidates");
  check_cuda(cudaMemcpy(cand, host_candidates_.data(), host_candidates_.size() * sizeof(int2),
                        cudaMemcpyHostToDevice),
             "upload fold candidates");
  spread_.grid = grid_;
  part_upper_bound_ = part_bound;
}

int NufftPlan::choose_geometry(int64_t point_count) const {
  if (type_ != 1) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "type-2 plans bin in one geometry"};
  if (point_count < 0) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "negative point count"};
  if (dim_ > 3) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "plans of more than three dimensions do not bin"};
  return layout_.choose_geometry(point_count);
}

void NufftPlan::prepare_interp_parts(const uint32_t* offsets, cudaStream_t stream) {
  interp_parts_bound_ = interp_parts_bound(point_count_, bins_);
  uint32_t* parts = static_cast<uint32_t*>(interp_parts_.reserve(bins_ * sizeof(uint32_t), "bin parts"));
  uint32_t* part_start =
      static_cast<uint32_t*>(interp_part_start_.reserve((bins_ + 1) * sizeof(uint32_t), "bin part offsets"));
  uint32_t* part_bin = static_cast<uint32_t*>(
      interp_part_bin_.reserve(static_cast<size_t>(interp_parts_bound_) * sizeof(uint32_t), "part bins"));
  interp_bin_parts(offsets, bins_, parts, part_start, part_bin, stream);
}

InterpParts NufftPlan::interp_parts() const {
  InterpParts p;
  p.part_bin = static_cast<const uint32_t*>(interp_part_bin_.get());
  p.part_start = static_cast<const uint32_t*>(interp_part_start_.get());
  p.upper_bound = interp_parts_bound_;
  return p;
}

void NufftPlan::set_points(int64_t count, const void* points, cudaStream_t stream) {
  if (!has_device_) {
    throw NufftFailure{B200NUFFT_GPU_EXECUTION_UNAVAILABLE,
                       "the plan was created without device resources"};
  }
  make_current();
  if (count < 0) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "negative point count"};
  if (count > kMaxPoints) {
    throw NufftFailure{B200NUFFT_LENGTH_OVERFLOW, "more than 2^30 - 1 points in one point set"};
  }
  if (count > 0 && points == nullptr) {
    throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null point buffer"};
  }
  point_count_ = count;
  points_ = points;
  tuned_ = tuning_for(tuning_key(type_, dim_, precision_, kernel_.width, fine_count_, count));
  if (dim_ > 3) {
    // No bins: the coordinates are kept (in f64 for Df64 plans) as given.
    const size_t coords = static_cast<size_t>(std::max<int64_t>(count, 1)) * dim_;
    if (precision_ == B200NUFFT_PRECISION_F32) {
      void* kept = sorted_points_.reserve(coords * sizeof(float), "coordinates");
      if (count > 0) {
        check_cuda(cudaMemcpyAsync(kept, points, static_cast<size_t>(count) * dim_ * sizeof(float),
                                   cudaMemcpyDeviceToDevice, stream),
                   "keep coordinates");
      }
    } else {
      void* kept = sorted_points_.reserve(coords * sizeof(double), "coordinates");
      if (count > 0 && precision_ == B200NUFFT_PRECISION_DF64) {
        df64_to_f64(static_cast<const float*>(points), count * dim_, static_cast<double*>(kept), stream);
      } else if (count > 0) {
        check_cuda(cudaMemcpyAsync(kept, points, static_cast<size_t>(count) * dim_ * sizeof(double),
                                   cudaMemcpyDeviceToDevice, stream),
                   "keep coordinates");
      }
    }
    check_cuda(cudaGetLastError(), "set points launch");
    return;
  }
  if (type_ == 1) {
    geometry_ = layout_.choose_geometry(count);
    configure_bins(geometry_);
  } else {
    geometry_ = -1;
    configure_type2_bins();
  }
  bin_order_pending_ = false;
  SortBuffers buf = sort_buffers(count);
  // Type-1 plans sort the points outside the fold's reach after every bin
  // (one more offset word) and mark the others in valid_mask_.
  const bool valid_first = type_ == 1;
  uint32_t* offsets = static_cast<uint32_t*>(
      offsets_.reserve((bins_ + (valid_first ? 2 : 1)) * sizeof(uint32_t), "bin offsets"));
  uint32_t* valid_mask = valid_first ? static_cast<uint32_t*>(valid_mask_.reserve(
                                           static_cast<size_t>((std::max<int64_t>(count, 1) + 31) / 32) * sizeof(uint32_t),
                                           "reach mask"))
                                     : nullptr;
  const size_t sorted_bytes = static_cast<size_t>(std::max<int64_t>(count, 1)) * dim_ * scalar_bytes();
  if (precision_ == B200NUFFT_PRECISION_F32) {
    tc2_active_ = tc2_enabled_ && tc_interp_supported(grid_);
    if (tc2_active_ && count > 0) {
      // The tensor-core order first (its permutation is consumed at once),
      // then the reference's type-2 bins in the same sort buffers.
      uint64_t bins2 = 0;
      tc2_grid_ = tc_interp_bins(grid_, &bins2);
      uint32_t* offsets2 =
          static_cast<uint32_t*>(tc2_offsets_.reserve((bins2 + 1) * sizeof(uint32_t), "tensor-core bin offsets"));
      uint32_t* perm2 = nullptr;
      uint32_t* keys2 = nullptr;
      sort_points(static_cast<const float*>(points), count, tc2_grid_, KeyKind::SupportStart, bins2, buf, offsets2,
                  &perm2, &keys2, stream, &timer_);
      StageScope scope(&timer_, kStageTileParts, stream);
      const int64_t tiles = tc_interp_tiles(grid_);
      const int64_t chunk_bound = tc_interp_chunk_bound(grid_, count);
      Ti2Prepare p;
      p.points = static_cast<const float*>(points);
      p.count = count;
      p.perm = perm2;
      p.offsets = offsets2;
      p.weights = static_cast<TcWeights*>(tc2_weights_.reserve(static_cast<size_t>(count) * sizeof(TcWeights),
                                                                "tensor-core window records"));
      p.inverse = static_cast<uint32_t*>(tc2_inverse_.reserve(static_cast<size_t>(count) * sizeof(uint32_t),
                                                               "tensor-core point slots"));
      p.tile_count = tiles;
      p.tile_chunks = static_cast<uint32_t*>(tc2_tile_chunks_.reserve(tiles * sizeof(uint32_t), "tile chunks"));
      p.tile_chunk_start = static_cast<uint32_t*>(
          tc2_tile_chunk_start_.reserve((tiles + 1) * sizeof(uint32_t), "tile chunk offsets"));
      p.chunks = static_cast<Ti2Chunk*>(tc2_chunks_.reserve(chunk_bound * sizeof(Ti2Chunk), "chunk table"));
      p.parts = static_cast<uint32_t*>(tc2_parts_.reserve(tiles * sizeof(uint32_t), "tensor-core parts"));
      p.part_start = static_cast<uint32_t*>(
          tc2_part_start_.reserve((tiles + 1) * sizeof(uint32_t), "tensor-core part offsets"));
      tc_interp_prepare(tc2_grid_, p, stream);
      tc2_part_upper_bound_ = tiles + chunk_bound / kTi2ChunksPerPart + 1;
      tc2_vector_max_.reserve(static_cast<size_t>(std::max<int64_t>(batch_, 1)) * sizeof(uint32_t), "vector maxima");
    }
    // 3D type 2: the interpolation takes the points in the order of their
    // support starts' (z, y) rows and 8-cell segments of x, so that a warp's
    // 32 points gather from few grid rows; only that order is sorted here
    // (its permutation kept), the reference's bins when they are asked for.
    rows_order_ = type_ == 2 && dim_ == 3 && count > 0;
    if (rows_order_) {
      uint64_t stride = 0;
      const GridParams rows = rows_grid(&stride);
      uint32_t* rows_offsets = static_cast<uint32_t*>(rows_offsets_.reserve((stride + 1) * sizeof(uint32_t),
                                                                           "row-order offsets"));
      uint32_t* order = nullptr;
      uint32_t* keys = nullptr;
      sort_points(static_cast<const float*>(points), count, rows, KeyKind::SupportStart, stride, buf, rows_offsets,
                  &order, &keys, stream, &timer_);
      keep_rows_order(order, count, stream);
      bin_order_pending_ = true;
    } else if (valid_first) {
      sort_points_valid_first(static_cast<const float*>(points), count, grid_, bins_, buf, offsets, valid_mask,
                              &perm_, &sorted_keys_, stream, &timer_);
    } else {
      sort_points(static_cast<const float*>(points), count, grid_, KeyKind::ApproximateCell, bins_, buf, offsets,
                  &perm_, &sorted_keys_, stream, &timer_);
    }
    float* sorted = static_cast<float*>(sorted_points_.reserve(sorted_bytes, "sorted coordinates"));
    gather_sorted_points(static_cast<const float*>(points), interp_perm(), count, dim_, sorted, stream,
                         &timer_);
    // The spreader and interpolator read each point's window start and offset.
    void* windows = windows_.reserve(static_cast<size_t>(std::max<int64_t>(count, 1)) * prepared_window_bytes(dim_),
                                     "prepared windows");
    StageScope scope(&timer_, kStageBinOffsets, stream);
    prepare_windows(sorted, count, grid_, windows, stream);
    if (type_ == 2 && dim_ == 2 && batch_ >= kInterpBinsMinBatch) {
      void* inverse = inverse_.reserve(static_cast<size_t>(std::max<int64_t>(count, 1)) * sizeof(uint32_t),
                                       "point slots");
      invert_permutation(perm_, count, static_cast<uint32_t*>(inverse), stream);
    }
    if (type_ == 2 && dim_ == 2) prepare_interp_parts(offsets, stream);
  } else {
    const double* points64 = static_cast<const double*>(points);
    if (precision_ == B200NUFFT_PRECISION_DF64 && count > 0) {
      double* converted = static_cast<double*>(points64_.reserve(sorted_bytes, "f64 coordinates"));
      df64_to_f64(static_cast<const float*>(points), count * dim_, converted, stream);
      points64 = converted;
    }
    // 3D type 2: the interpolation's row order alone, as for f32 plans.
    rows_order_ = type_ == 2 && dim_ == 3 && count > 0;
    if (rows_order_) {
      uint64_t stride = 0;
      const GridParams rows = rows_grid(&stride);
      uint32_t* rows_offsets = static_cast<uint32_t*>(rows_offsets_.reserve((stride + 1) * sizeof(uint32_t),
                                                                           "row-order offsets"));
      uint32_t* order = nullptr;
      uint32_t* keys = nullptr;
      sort_points64(points64, count, rows, stride, buf, rows_offsets, &order, &keys, stream, &timer_, nullptr);
      keep_rows_order(order, count, stream);
      bin_order_pending_ = true;
    } else {
      sort_points64(points64, count, grid_, bins_, buf, offsets, &perm_, &sorted_keys_, stream,
                    &timer_, valid_mask);
    }
    double* sorted = static_cast<double*>(sorted_points_.reserve(sorted_bytes, "sorted coordinates"));
    gather_sorted_points64(points64, interp_perm(), count, dim_, sorted, stream, &timer_);
    if (type_ == 2 && dim_ == 2) {
      StageScope scope(&timer_, kStageBinOffsets, stream);
      prepare_interp_parts(offsets, stream);
    }
  }
  if (type_ == 1) {
    configure_tiles();
    parts_.reserve(static_cast<size_t>(spread_.tile_count) * sizeof(uint32_t), "tile parts");
    part_start_.reserve(static_cast<size_t>(spread_.tile_count + 1) * sizeof(uint32_t),
                        "tile part offsets");
    spread_count_parts(spread_, offsets, static_cast<uint32_t*>(parts_.get()),
                       static_cast<uint32_t*>(part_start_.get()), stream, &timer_);
    if (tc_active_) {
      const int64_t tiles = spread_.tile_count;
      const int64_t chunk_bound = tc_chunk_bound(spread_, count);
      TcPrepare p;
      p.sorted_points = static_cast<const float*>(sorted_points_.get());
      p.count = count;
      p.perm = perm_;
      p.offsets = offsets;
      p.weights = static_cast<TcWeights*>(
          tc_weights_.reserve(static_cast<size_t>(std::max<int64_t>(count, 1)) * sizeof(TcWeights), "point windows"));
      p.inverse = static_cast<uint32_t*>(
          tc_inverse_.reserve(static_cast<size_t>(std::max<int64_t>(count, 1)) * sizeof(uint32_t), "point slots"));
      p.tile_chunks = static_cast<uint32_t*>(tc_tile_chunks_.reserve(tiles * sizeof(uint32_t), "tile chunks"));
      p.tile_chunk_start = static_cast<uint32_t*>(
          tc_tile_chunk_start_.reserve((tiles + 1) * sizeof(uint32_t), "tile chunk offsets"));
      p.chunks = static_cast<TcChunk*>(tc_chunks_.reserve(chunk_bound * sizeof(TcChunk), "chunk table"));
      p.parts = static_cast<uint32_t*>(tc_parts_.reserve(tiles * sizeof(uint32_t), "tensor-core parts"));
      p.part_start = static_cast<uint32_t*>(
          tc_part_start_.reserve((tiles + 1) * sizeof(uint32_t), "tensor-core part offsets"));
      tc_prepare(spread_, p, stream, &timer_);
      tc_part_upper_bound_ = tiles + chunk_bound / kTcChunksPerPart + 1;
    }
  }
  check_cuda(cudaGetLastError(), "set points launch");
}

cufftHandle NufftPlan::fft_for(int batch) {
  auto found = ffts_.find(batch);
  if (found != ffts_.end()) return found->second;
  int n[3];
  for (int a = 0; a < dim_; ++a) n[a] = static_cast<int>(fine_[dim_ - 1 - a]);
  cufftHandle handle;
  const cufftType kind = precision_ == B200NUFFT_PRECISION_F32 ? CUFFT_C2C : CUFFT_Z2Z;
  const cufftResult r = cufftPlanMany(&handle, dim_, n, nullptr, 1, static_cast<int>(fine_count_),
                                      nullptr, 1, static_cast<int>(fine_count_), kind, batch);
  if (r != CUFFT_SUCCESS) {
    throw NufftFailure{B200NUFFT_FFT_SHAPE_UNSUPPORTED,
                       "cuFFT plan creation failed with code " + std::to_string(static_cast<int>(r))};
  }
  ffts_[batch] = handle;
  return handle;
}

void NufftPlan::run_fft(void* fine, int batch, int direction, cudaStream_t stream) {
  StageScope scope(&timer_, kStageFft, stream);
  cufftHandle h = fft_for(batch);
  cufftSetStream(h, stream);
  const cufftResult r =
      precision_ == B200NUFFT_PRECISION_F32
          ? cufftExecC2C(h, static_cast<cufftComplex*>(fine), static_cast<cufftComplex*>(fine), direction)
          : cufftExecZ2Z(h, static_cast<cufftDoubleComplex*>(fine),
                         static_cast<cufftDoubleComplex*>(fine), direction);
  if (r != CUFFT_SUCCESS) {
    throw NufftFailure{B200NUFFT_FFT_EXECUTION_FAILED,
                       "cuFFT execution failed with code " + std::to_string(static_cast<int>(r))};
  }
}

void NufftPlan::execute(int64_t active_batch, const void* input, void* output, cudaStream_t stream) {
  if (!has_device_) {
    throw NufftFailure{B200NUFFT_GPU_EXECUTION_UNAVAILABLE,
                       "the plan was created without device resources"};
  }
  make_current();
  validate_active_batch(active_batch);
  if (point_count_ < 0) {
    throw NufftFailure{B200NUFFT_GPU_EXECUTION_UNAVAILABLE,
                       "call b200nufft_set_points (or b200nufft_encode) before executing"};
  }
  const uint64_t in_bytes = required_input_bytes(point_count_, active_batch);
  const uint64_t out_bytes = required_output_bytes(point_count_, active_batch);
  // Empty buffers (zero points) may be null.
  if ((output == nullptr && out_bytes > 0) || (input == nullptr && in_bytes > 0)) {
    throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null input or output buffer"};
  }
  if (out_bytes == 0) return;
  const char* in_lo = static_cast<const char*>(input);
  const char* out_lo = static_cast<const char*>(output);
  if (input && in_bytes && out_bytes && in_lo < out_lo + out_bytes && out_lo < in_lo + in_bytes) {
    throw NufftFailure{B200NUFFT_GPU_BUFFER_ALIAS_UNSUPPORTED, "input and output overlap"};
  }
  const int batch = static_cast<int>(active_batch);
  if (precision_ == B200NUFFT_PRECISION_F32) {
    execute_f32(batch, input, output, out_bytes, stream);
  } else {
    execute_f64(batch, input, output, in_bytes, out_bytes, stream);
  }
  check_cuda(cudaGetLastError(), "execute launch");
}

void NufftPlan::execute_f32(int batch, const void* input, void* output, uint64_t out_bytes,
                            cudaStream_t stream) {
  float2* fine = static_cast<float2*>(fine_grid_.get());
  const int direction = isign_ >= 0 ? CUFFT_INVERSE : CUFFT_FORWARD;
  if (dim_ > 3) {
    execute_nd(batch, input, output, fine, direction, stream);
    return;
  }
  if (type_ == 1) {
    if (point_count_ == 0) {
      check_cuda(cudaMemsetAsync(output, 0, out_bytes, stream), "zero type-1 output");
      return;
    }
    if (tc_active_ && batch >= tensor_min_batch()) {
      const int64_t groups = (batch + kTcVectors - 1) / kTcVectors;
      TcLaunch t;
      t.strengths = static_cast<const float2*>(input);
      t.count = point_count_;
      t.batch = batch;
      t.inverse = static_cast<const uint32_t*>(tc_inverse_.get());
      t.weights = static_cast<const TcWeights*>(tc_weights_.get());
      t.chunks = static_cast<const TcChunk*>(tc_chunks_.get());
      t.tile_chunk_start = static_cast<const uint32_t*>(tc_tile_chunk_start_.get());
      t.part_start = static_cast<const uint32_t*>(tc_part_start_.get());
      t.part_upper_bound = tc_part_upper_bound_;
      t.packed = static_cast<float*>(tc_packed_.reserve(
          static_cast<size_t>(groups) * point_count_ * kTcRows * sizeof(float), "packed strengths"));
      t.scratch = static_cast<float2*>(scratch_.reserve(static_cast<size_t>(tc_part_upper_bound_) * groups *
                                                            kTcVectors * spread_.padded_cells * sizeof(float2),
                                                        "spreading tiles"));
      t.candidates = static_cast<const int2*>(candidates_.get());
      t.fine = fine;
      t.error_flag = static_cast<uint32_t*>(counters_.get()) + 7;
      tc_spread_execute(spread_, t, stream, &timer_);
      run_fft(fine, batch, direction, stream);
      StageScope scope(&timer_, kStageDeconvolution, stream);
      deconvolve_f32(modes_params_, batch, fine, static_cast<const float*>(amplitudes_.get()),
                     static_cast<float2*>(output), stream);
      return;
    }
    const size_t scratch_bytes = static_cast<size_t>(part_upper_bound_) * batch *
                                 spread_.padded_cells * sizeof(float2);
    SpreadLaunch l;
    l.points = static_cast<const float*>(sorted_points_.get());
    l.windows = windows_.get();
    l.strengths = static_cast<const float2*>(input);
    l.point_count = point_count_;
    l.batch = batch;
    l.perm = perm_;
    l.offsets = static_cast<const uint32_t*>(offsets_.get());
    l.part_start = static_cast<const uint32_t*>(part_start_.get());
    l.part_upper_bound = part_upper_bound_;
    l.max_bits = static_cast<uint32_t*>(max_bits_.get());
    l.scratch = static_cast<float2*>(scratch_.reserve(scratch_bytes, "spreading tiles"));
    l.candidates = static_cast<const int2*>(candidates_.get());
    l.fine = fine;
    l.valid_mask = static_cast<const uint32_t*>(valid_mask_.get());
    if (fused_fold(batch)) {
      // 2D: the fold runs inside the pass along axis 0. 3D: the fold kernel
      // (a thread per cell: the crowded tiles' long part lists overlap
      // better) folds into the fine grid, which that pass reads.
      if (dim_ == 2) l.fine = nullptr;
      spread_execute(spread_, l, stream, &timer_);
      float2* rows = static_cast<float2*>(
          fused_fft_rows_.reserve(fused_fft_buffer_bytes(fused_fft_, batch), "transformed rows"));
      fused_fft_type1(spread_, fused_fft_, batch, dim_ == 2 ? l.scratch : nullptr, l.part_start,
                      l.part_upper_bound, l.candidates, static_cast<const float*>(amplitudes_.get()), rows, fine,
                      static_cast<float2*>(output), stream, &timer_);
      return;
    }
    spread_execute(spread_, l, stream, &timer_);
    run_fft(fine, batch, direction, stream);
    StageScope scope(&timer_, kStageDeconvolution, stream);
    deconvolve_f32(modes_params_, batch, fine, static_cast<const float*>(amplitudes_.get()),
                   static_cast<float2*>(output), stream);
  } else {
    if (fused_fft_active_) {
      float2* rows = static_cast<float2*>(
          fused_fft_rows_.reserve(fused_fft_buffer_bytes(fused_fft_, batch), "transformed rows"));
      fused_fft_type2(fused_fft_, batch, static_cast<const float2*>(input), static_cast<const float*>(amplitudes_.get()),
                      rows, fine, fine, stream, &timer_);
    } else {
      {
        StageScope scope(&timer_, kStagePredeconvolution, stream);
        predeconvolve_f32(modes_params_, batch, static_cast<const float2*>(input),
                          static_cast<const float*>(amplitudes_.get()), fine, stream);
      }
      run_fft(fine, batch, direction, stream);
    }
    if (tc2_active_ && batch >= tensor_min_batch()) {
      const int64_t groups = (batch + kTi2Vectors - 1) / kTi2Vectors;
      Ti2Launch t;
      t.fine = fine;
      t.batch = batch;
      t.count = point_count_;
      t.weights = static_cast<const TcWeights*>(tc2_weights_.get());
      t.chunks = static_cast<const Ti2Chunk*>(tc2_chunks_.get());
      t.tile_chunk_start = static_cast<const uint32_t*>(tc2_tile_chunk_start_.get());
      t.part_start = static_cast<const uint32_t*>(tc2_part_start_.get());
      t.part_upper_bound = tc2_part_upper_bound_;
      t.inverse = static_cast<const uint32_t*>(tc2_inverse_.get());
      t.staged = static_cast<float2*>(staged_.reserve(
          static_cast<size_t>(point_count_) * groups * kTi2Vectors * sizeof(float2), "staged type-2 values"));
      t.output = static_cast<float2*>(output);
      t.vector_max = static_cast<uint32_t*>(tc2_vector_max_.get());
      t.error_flag = static_cast<uint32_t*>(counters_.get()) + 7;
      StageScope scope(&timer_, kStageInterpolation, stream);
      tc_interp_execute(tc2_grid_, t, stream);
      return;
    }
    if (dim_ == 2 && batch >= kInterpBinsMinBatch && interpolate_bins_supported(grid_)) {
      InterpBinsLaunch b;
      b.windows = windows_.get();
      b.point_count = point_count_;
      b.perm = perm_;
      b.offsets = static_cast<const uint32_t*>(offsets_.get());
      b.bins = bins_;
      b.fine = fine;
      b.batch = batch;
      b.output = static_cast<float2*>(output);
      b.inverse = static_cast<const uint32_t*>(inverse_.get());
      b.staged = static_cast<float2*>(staged_.reserve(
          static_cast<size_t>(std::max<int64_t>(point_count_, 1)) * ((batch + 31) / 32 * 32) * sizeof(float2),
          "staged type-2 values"));
      b.parts = interp_parts();
      StageScope scope(&timer_, kStageInterpolation, stream);
      interpolate_bins_execute(grid_, b, stream);
      return;
    }
    if (dim_ == 2 && interpolate_bins_supported(grid_)) {
      InterpBinsLaunch b{};
      b.windows = windows_.get();
      b.point_count = point_count_;
      b.perm = perm_;
      b.offsets = static_cast<const uint32_t*>(offsets_.get());
      b.bins = bins_;
      b.fine = fine;
      b.batch = batch;
      b.output = static_cast<float2*>(output);
      b.parts = interp_parts();
      StageScope scope(&timer_, kStageInterpolation, stream);
      interpolate_region_execute(grid_, b, stream);
      return;
    }
    InterpLaunch l;
    l.points = static_cast<const float*>(sorted_points_.get());
    l.windows = windows_.get();
    l.point_count = point_count_;
    l.perm = interp_perm();
    l.fine = fine;
    l.batch = batch;
    l.output = static_cast<float2*>(output);
    StageScope scope(&timer_, kStageInterpolation, stream);
    interpolate_execute(grid_, l, stream);
  }
}

void NufftPlan::execute_f64(int batch, const void* input, void* output, uint64_t in_bytes,
                            uint64_t out_bytes, cudaStream_t stream) {
  double2* fine = static_cast<double2*>(fine_grid_.get());
  const int direction = isign_ >= 0 ? CUFFT_INVERSE : CUFFT_FORWARD;
  // Df64 values arrive as (hi, lo) float pairs per scalar; the pipeline runs
  // in f64 on converted copies.
  const bool df64 = precision_ == B200NUFFT_PRECISION_DF64;
  const double2* in = static_cast<const double2*>(input);
  double2* out = static_cast<double2*>(output);
  if (df64) {
    double* converted = static_cast<double*>(input64_.reserve(std::max<uint64_t>(in_bytes, 16), "f64 input"));
    if (in_bytes) df64_to_f64(static_cast<const float*>(input), static_cast<int64_t>(in_bytes / 8), converted, stream);
    in = reinterpret_cast<const double2*>(converted);
    out = static_cast<double2*>(output64_.reserve(std::max<uint64_t>(out_bytes, 16), "f64 output"));
  }
  if (dim_ > 3) {
    execute_nd(batch, in, out, fine, direction, stream);
  } else if (type_ == 1) {
    if (point_count_ == 0) {
      check_cuda(cudaMemsetAsync(output, 0, out_bytes, stream), "zero type-1 output");
      return;
    }
    const size_t scratch_bytes = static_cast<size_t>(part_upper_bound_) * batch *
                                 spread_.padded_cells * sizeof(double2);
    SpreadLaunch64 l;
    l.points = static_cast<const double*>(sorted_points_.get());
    l.strengths = in;
    l.point_count = point_count_;
    l.batch = batch;
    l.perm = perm_;
    l.offsets = static_cast<const uint32_t*>(offsets_.get());
    l.part_start = static_cast<const uint32_t*>(part_start_.get());
    l.part_upper_bound = part_upper_bound_;
    l.max_bits = static_cast<unsigned long long*>(max_bits_.get());
    l.scratch = static_cast<double2*>(scratch_.reserve(scratch_bytes, "spreading tiles"));
    l.candidates = static_cast<const int2*>(candidates_.get());
    l.fine = fine;
    l.valid_mask = static_cast<const uint32_t*>(valid_mask_.get());
    spread_execute64(spread_, l, stream, &timer_);
    run_fft(fine, batch, direction, stream);
    StageScope scope(&timer_, kStageDeconvolution, stream);
    deconvolve_f64(modes_params_, batch, fine, static_cast<const double*>(amplitudes_.get()), out,
                   stream);
  } else {
    {
      StageScope scope(&timer_, kStagePredeconvolution, stream);
      predeconvolve_f64(modes_params_, batch, in, static_cast<const double*>(amplitudes_.get()),
                        fine, stream);
    }
    run_fft(fine, batch, direction, stream);
    InterpLaunch64 l;
    l.points = static_cast<const double*>(sorted_points_.get());
    l.point_count = point_count_;
    l.perm = interp_perm();
    l.fine = fine;
    l.batch = batch;
    l.output = out;
    StageScope scope(&timer_, kStageInterpolation, stream);
    // Staged regions pay off for one vector and wide windows (measured: w 13
    // 1.5x faster; w 10 even; batches of 16 slower, whose window weights the
    // thread-per-point kernel reuses across vectors).
    if (batch == 1 && kernel_.width >= 11 && interpolate_region64_supported(grid_)) {
      interpolate_region64_execute(grid_, l, static_cast<const uint32_t*>(offsets_.get()), bins_, interp_parts(),
                                   stream);
    } else {
      interpolate_execute64(grid_, l, stream);
    }
  }
  if (df64 && out_bytes) {
    f64_to_df64(reinterpret_cast<const double*>(out), static_cast<int64_t>(out_bytes / 8),
                static_cast<float*>(output), stream);
  }
}

void NufftPlan::spread_nd(int batch, const void* strengths, void* grid, cudaStream_t stream) {
  StageScope scope(&timer_, kStageSpread, stream);
  auto* acc = static_cast<unsigned long long*>(
      nd_acc_.reserve(static_cast<size_t>(batch) * fine_count_ * 2 * sizeof(unsigned long long), "integer fine grid"));
  nd_spread(nd_, sorted_points_.get(), strengths, point_count_, batch, acc,
            static_cast<unsigned long long*>(max_bits_.get()), grid, stream);
}

void NufftPlan::execute_nd(int batch, const void* input, void* output, void* fine, int direction,
                           cudaStream_t stream) {
  const bool f32 = precision_ == B200NUFFT_PRECISION_F32;
  if (type_ == 1) {
    spread_nd(batch, input, fine, stream);
    run_fft_nd(fine, batch, direction, stream);
    StageScope scope(&timer_, kStageDeconvolution, stream);
    if (f32) {
      deconvolve_f32(modes_params_, batch, static_cast<const float2*>(fine),
                     static_cast<const float*>(amplitudes_.get()), static_cast<float2*>(output), stream);
    } else {
      deconvolve_f64(modes_params_, batch, static_cast<const double2*>(fine),
                     static_cast<const double*>(amplitudes_.get()), static_cast<double2*>(output), stream);
    }
    return;
  }
  {
    StageScope scope(&timer_, kStagePredeconvolution, stream);
    if (f32) {
      predeconvolve_f32(modes_params_, batch, static_cast<const float2*>(input),
                        static_cast<const float*>(amplitudes_.get()), static_cast<float2*>(fine), stream);
    } else {
      predeconvolve_f64(modes_params_, batch, static_cast<const double2*>(input),
                        static_cast<const double*>(amplitudes_.get()), static_cast<double2*>(fine), stream);
    }
  }
  run_fft_nd(fine, batch, direction, stream);
  StageScope scope(&timer_, kStageInterpolation, stream);
  nd_interpolate(nd_, sorted_points_.get(), fine, point_count_, batch, output, stream);
}

// The d-dimensional transform as transforms over groups of up to three
// consecutive axes: the first group batched over everything else, each later
// group batched over the cells of the axes before it (element stride
// `inner`) and run once per block of the axes after it.
void NufftPlan::run_fft_nd(void* fine, int batch, int direction, cudaStream_t stream) {
  StageScope scope(&timer_, kStageFft, stream);
  const bool f32 = precision_ == B200NUFFT_PRECISION_F32;
  const size_t element = 2 * scalar_bytes();
  int64_t inner = 1;
  for (int a0 = 0; a0 < dim_; a0 += 3) {
    const int a1 = std::min(dim_, a0 + 3);
    const int rank = a1 - a0;
    int64_t span = 1, outer = batch;
    for (int a = a0; a < a1; ++a) span *= fine_[a];
    for (int a = a1; a < dim_; ++a) outer *= fine_[a];
    const int64_t key = static_cast<int64_t>(a0) * (int64_t(1) << 32) + batch;
    auto found = nd_ffts_.find(key);
    cufftHandle h;
    if (found != nd_ffts_.end()) {
      h = found->second;
    } else {
      if (inner * span > std::numeric_limits<int32_t>::max() || outer > std::numeric_limits<int32_t>::max()) {
        throw NufftFailure{B200NUFFT_FFT_SHAPE_UNSUPPORTED, "fine grid too large for the grouped FFT"};
      }
      int n[3];
      for (int r = 0; r < rank; ++r) n[r] = static_cast<int>(fine_[a1 - 1 - r]);
      const cufftType kind = f32 ? CUFFT_C2C : CUFFT_Z2Z;
      cufftResult r;
      if (a0 == 0) {
        r = cufftPlanMany(&h, rank, n, nullptr, 1, static_cast<int>(span), nullptr, 1, static_cast<int>(span), kind,
                          static_cast<int>(outer));
      } else {
        r = cufftPlanMany(&h, rank, n, n, static_cast<int>(inner), 1, n, static_cast<int>(inner), 1, kind,
                          static_cast<int>(inner));
      }
      if (r != CUFFT_SUCCESS) {
        throw NufftFailure{B200NUFFT_FFT_SHAPE_UNSUPPORTED,
                           "cuFFT plan creation failed with code " + std::to_string(static_cast<int>(r))};
      }
      nd_ffts_[key] = h;
    }
    cufftSetStream(h, stream);
    const int64_t blocks = a0 == 0 ? 1 : outer;
    for (int64_t o = 0; o < blocks; ++o) {
      char* base = static_cast<char*>(fine) + static_cast<size_t>(o * inner * span) * element;
      const cufftResult r =
          f32 ? cufftExecC2C(h, reinterpret_cast<cufftComplex*>(base), reinterpret_cast<cufftComplex*>(base), direction)
              : cufftExecZ2Z(h, reinterpret_cast<cufftDoubleComplex*>(base),
                             reinterpret_cast<cufftDoubleComplex*>(base), direction);
      if (r != CUFFT_SUCCESS) {
        throw NufftFailure{B200NUFFT_FFT_EXECUTION_FAILED,
                           "cuFFT execution failed with code " + std::to_string(static_cast<int>(r))};
      }
    }
    inner *= span;
  }
}

void NufftPlan::spread_to(int64_t active_batch, const void* strengths, void* grid,
                          cudaStream_t stream) {
  if (!has_device_ || type_ != 1) {
    throw NufftFailure{B200NUFFT_GPU_EXECUTION_UNAVAILABLE, "spreading needs a type-1 GPU plan"};
  }
  make_current();
  validate_active_batch(active_batch);
  if (point_count_ < 0) {
    throw NufftFailure{B200NUFFT_GPU_EXECUTION_UNAVAILABLE, "no point set"};
  }
  const int batch = static_cast<int>(active_batch);
  if (point_count_ == 0) {
    check_cuda(cudaMemsetAsync(grid, 0, static_cast<size_t>(batch) * fine_count_ * 2 * scalar_bytes(),
                               stream),
               "zero spread grid");
    return;
  }
  if (dim_ > 3) {
    spread_nd(batch, strengths, grid, stream);
    check_cuda(cudaGetLastError(), "spread launch");
    return;
  }
  if (precision_ == B200NUFFT_PRECISION_F32) {
    SpreadLaunch l;
    l.points = static_cast<const float*>(sorted_points_.get());
    l.windows = windows_.get();
    l.strengths = static_cast<const float2*>(strengths);
    l.point_count = point_count_;
    l.batch = batch;
    l.perm = perm_;
    l.offsets = static_cast<const uint32_t*>(offsets_.get());
    l.part_start = static_cast<const uint32_t*>(part_start_.get());
    l.part_upper_bound = part_upper_bound_;
    l.max_bits = static_cast<uint32_t*>(max_bits_.get());
    l.scratch = static_cast<float2*>(scratch_.reserve(
        static_cast<size_t>(part_upper_bound_) * batch * spread_.padded_cells * sizeof(float2),
        "spreading tiles"));
    l.candidates = static_cast<const int2*>(candidates_.get());
    l.fine = static_cast<float2*>(grid);
    l.valid_mask = static_cast<const uint32_t*>(valid_mask_.get());
    spread_execute(spread_, l, stream, &timer_);
  } else {
    SpreadLaunch64 l;
    l.points = static_cast<const double*>(sorted_points_.get());
    l.strengths = static_cast<const double2*>(strengths);
    l.point_count = point_count_;
    l.batch = batch;
    l.perm = perm_;
    l.offsets = static_cast<const uint32_t*>(offsets_.get());
    l.part_start = static_cast<const uint32_t*>(part_start_.get());
    l.part_upper_bound = part_upper_bound_;
    l.max_bits = static_cast<unsigned long long*>(max_bits_.get());
    l.scratch = static_cast<double2*>(scratch_.reserve(
        static_cast<size_t>(part_upper_bound_) * batch * spread_.padded_cells * sizeof(double2),
        "spreading tiles"));
    l.candidates = static_cast<const int2*>(candidates_.get());
    l.fine = static_cast<double2*>(grid);
    l.valid_mask = static_cast<const uint32_t*>(valid_mask_.get());
    spread_execute64(spread_, l, stream, &timer_);
  }
  check_cuda(cudaGetLastError(), "spread launch");
}

GridParams NufftPlan::rows_grid(uint64_t* bins) const {
  // Bins of one cell along y and z and 8 cells along x: sorted by these
  // keys, the points come in the order of their support starts' (z, y)
  // rows and 8-cell x segments.
  GridParams rows = grid_;
  uint64_t stride = 1;
  for (int a = 0; a < 3; ++a) {
    const int shift = a == 0 ? std::min(3, ilog2(fine_[0])) : 0;
    rows.axis[a].shift = shift;
    rows.axis[a].bins = static_cast<uint32_t>((fine_[a] + (int64_t{1} << shift) - 1) >> shift);
    rows.axis[a].stride = static_cast<uint32_t>(stride);
    stride *= rows.axis[a].bins;
  }
  *bins = stride;
  return rows;
}

void NufftPlan::keep_rows_order(const uint32_t* order, int64_t count, cudaStream_t stream) {
  uint32_t* kept = static_cast<uint32_t*>(rows_perm_.reserve(static_cast<size_t>(count) * sizeof(uint32_t),
                                                             "row-order permutation"));
  check_cuda(cudaMemcpyAsync(kept, order, static_cast<size_t>(count) * sizeof(uint32_t), cudaMemcpyDeviceToDevice,
                             stream),
             "keep row order");
}

SortBuffers NufftPlan::sort_buffers(int64_t count) {
  const size_t words = static_cast<size_t>(std::max<int64_t>(count, 1)) * sizeof(uint32_t);
  SortBuffers buf;
  buf.keys_a = static_cast<uint32_t*>(keys_a_.reserve(words, "bin keys"));
  buf.keys_b = static_cast<uint32_t*>(keys_b_.reserve(words, "bin keys"));
  buf.vals_a = static_cast<uint32_t*>(vals_a_.reserve(words, "point permutation"));
  buf.vals_b = static_cast<uint32_t*>(vals_b_.reserve(words, "point permutation"));
  buf.hist = static_cast<uint32_t*>(hist_.get());
  buf.status = static_cast<uint32_t*>(status_.reserve(sort_status_bytes(count), "look-back words"));
  buf.counters = static_cast<uint32_t*>(counters_.get());
  return buf;
}

void NufftPlan::finish_bin_order(cudaStream_t stream) {
  if (!bin_order_pending_) return;
  // The same sort as set_points' (stable, so ties keep the caller's order),
  // on the coordinates put back in the caller's order from the row order.
  const int64_t count = point_count_;
  SortBuffers buf = sort_buffers(count);
  uint32_t* offsets = static_cast<uint32_t*>(offsets_.get());
  const uint32_t* rows = static_cast<const uint32_t*>(rows_perm_.get());
  if (precision_ == B200NUFFT_PRECISION_F32) {
    float* coords = static_cast<float*>(unsorted_.reserve(static_cast<size_t>(count) * 3 * sizeof(float),
                                                           "coordinates in the caller's order"));
    scatter_points3(static_cast<const float*>(sorted_points_.get()), rows, count, coords, stream);
    sort_points(coords, count, grid_, KeyKind::ApproximateCell, bins_, buf, offsets, &perm_, &sorted_keys_,
                stream, &timer_);
  } else {
    double* coords = static_cast<double*>(unsorted_.reserve(static_cast<size_t>(count) * 3 * sizeof(double),
                                                             "coordinates in the caller's order"));
    scatter_points3(static_cast<const double*>(sorted_points_.get()), rows, count, coords, stream);
    sort_points64(coords, count, grid_, bins_, buf, offsets, &perm_, &sorted_keys_, stream, &timer_, nullptr);
  }
  check_cuda(cudaGetLastError(), "bin order launch");
  bin_order_pending_ = false;
}

void NufftPlan::copy_bin_order(uint32_t* permutation, uint32_t* bin_offsets, cudaStream_t stream) {
  make_current();
  if (dim_ > 3) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "plans of more than three dimensions do not bin"};
  if (point_count_ < 0) {
    throw NufftFailure{B200NUFFT_GPU_EXECUTION_UNAVAILABLE, "no point set"};
  }
  finish_bin_order(stream);
  const uint32_t* order = perm_;
  const uint32_t* offsets = static_cast<const uint32_t*>(offsets_.get());
  if (type_ == 1) {
    // Type-1 points outside the fold's reach were sorted after every bin:
    // the reference's order holds them in bin 0.
    reference_order(stream);
    order = static_cast<const uint32_t*>(ref_perm_.get());
    offsets = static_cast<const uint32_t*>(ref_offsets_.get());
  }
  if (permutation && point_count_ > 0) {
    check_cuda(cudaMemcpyAsync(permutation, order, point_count_ * sizeof(uint32_t),
                               cudaMemcpyDeviceToDevice, stream),
               "copy permutation");
  }
  if (bin_offsets) {
    check_cuda(cudaMemcpyAsync(bin_offsets, offsets, (bins_ + 1) * sizeof(uint32_t),
                               cudaMemcpyDeviceToDevice, stream),
               "copy bin offsets");
  }
}

void NufftPlan::reference_order(cudaStream_t stream) {
  const size_t words = static_cast<size_t>(std::max<int64_t>(point_count_, 1));
  uint32_t* ref_perm = static_cast<uint32_t*>(ref_perm_.reserve(words * sizeof(uint32_t), "reference order"));
  uint32_t* ref_keys = static_cast<uint32_t*>(ref_keys_.reserve(words * sizeof(uint32_t), "reference keys"));
  uint32_t* ref_offsets =
      static_cast<uint32_t*>(ref_offsets_.reserve((bins_ + 1) * sizeof(uint32_t), "reference bin offsets"));
  reference_bin_order(perm_, sorted_keys_, static_cast<const uint32_t*>(offsets_.get()), point_count_, bins_,
                      ref_perm, ref_keys, ref_offsets, stream);
}

void NufftPlan::copy_prepared_slots(int32_t* starts, float* offsets, cudaStream_t stream) {
  if (dim_ > 3) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "plans of more than three dimensions do not bin"};
  make_current();
  if (point_count_ < 0 || type_ != 1) {
    throw NufftFailure{B200NUFFT_GPU_EXECUTION_UNAVAILABLE, "no type-1 point set"};
  }
  if (!starts || !offsets) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null buffer"};
  reference_order(stream);
  prepare_reference_slots(static_cast<const float*>(points_), point_count_, grid_,
                          static_cast<const uint32_t*>(ref_perm_.get()), static_cast<const uint32_t*>(ref_keys_.get()),
                          starts, offsets, stream);
}

bool NufftPlan::batch_problem(BatchProblem* out) {
  if (!has_device_ || type_ != 1 || precision_ != B200NUFFT_PRECISION_F32 || (dim_ != 2 && dim_ != 3) ||
      point_count_ < 0) {
    return false;
  }
  make_current();
  std::memset(out, 0, sizeof(*out));
  out->sp = spread_;
  out->windows = windows_.get();
  out->perm = perm_;
  out->offsets = static_cast<const uint32_t*>(offsets_.get());
  out->part_start = static_cast<const uint32_t*>(part_start_.get());
  out->valid_mask = static_cast<const uint32_t*>(valid_mask_.get());
  out->point_count = point_count_;
  out->max_bits = static_cast<uint32_t*>(max_bits_.get());
  out->scratch = static_cast<float2*>(scratch_.reserve(
      static_cast<size_t>(std::max<int64_t>(part_upper_bound_, 1)) * spread_.padded_cells * sizeof(float2),
      "spreading tiles"));
  return true;
}

void NufftPlan::finish_batch(void* output, cudaStream_t stream) {
  make_current();
  float2* fine = static_cast<float2*>(fine_grid_.get());
  if (point_count_ == 0) {
    check_cuda(cudaMemsetAsync(output, 0, static_cast<size_t>(mode_count_) * sizeof(float2), stream),
               "zero type-1 output");
    return;
  }
  SpreadLaunch l{};
  l.batch = 1;
  l.part_start = static_cast<const uint32_t*>(part_start_.get());
  l.part_upper_bound = part_upper_bound_;
  l.scratch = static_cast<float2*>(scratch_.get());
  l.candidates = static_cast<const int2*>(candidates_.get());
  l.fine = fine;
  if (fused_fold(1)) {
    float2* rows = static_cast<float2*>(
        fused_fft_rows_.reserve(fused_fft_buffer_bytes(fused_fft_, 1), "transformed rows"));
    if (dim_ == 3) {
      StageScope scope(&timer_, kStageFold, stream);
      spread_fold(spread_, l, stream);
    }
    fused_fft_type1(spread_, fused_fft_, 1, dim_ == 2 ? l.scratch : nullptr, l.part_start, l.part_upper_bound,
                    l.candidates, static_cast<const float*>(amplitudes_.get()), rows, fine,
                    static_cast<float2*>(output), stream, &timer_);
    check_cuda(cudaGetLastError(), "batch finish launch");
    return;
  }
  {
    StageScope scope(&timer_, kStageFold, stream);
    spread_fold(spread_, l, stream);
  }
  run_fft(fine, 1, isign_ >= 0 ? CUFFT_INVERSE : CUFFT_FORWARD, stream);
  StageScope scope(&timer_, kStageDeconvolution, stream);
  deconvolve_f32(modes_params_, 1, fine, static_cast<const float*>(amplitudes_.get()), static_cast<float2*>(output),
                 stream);
  check_cuda(cudaGetLastError(), "batch finish launch");
}

void NufftPlan::synchronize(cudaStream_t stream) {
  make_current();
  check_cuda(cudaStreamSynchronize(stream), "synchronize");
  uint32_t flag = 0;
  check_cuda(cudaMemcpy(&flag, static_cast<uint32_t*>(counters_.get()) + 7, sizeof(uint32_t),
                        cudaMemcpyDeviceToHost),
             "read device flags");
  if (flag != 0) {
    cudaMemset(static_cast<uint32_t*>(counters_.get()) + 7, 0, sizeof(uint32_t));
    throw NufftFailure{B200NUFFT_DEVICE_TIMEOUT,
                       "a device wait (bin-sort look-back or tensor-core pipeline) gave up; results are invalid"};
  }
}

void NufftPlan::info(b200nufft_plan_info* out) const {
  std::memset(out, 0, sizeof(*out));
  out->type = type_;
  out->dimensions = dim_;
  out->precision = precision_;
  out->kernel_width = kernel_.width;
  out->kernel_beta = kernel_.beta;
  for (int a = 0; a < dim_; ++a) out->fine_shape[a] = fine_[a];
  out->mode_count = mode_count_;
  out->batch = batch_;
  out->geometry_count = static_cast<int32_t>(std::min<size_t>(layout_.geometries.size(), 16));
  for (int g = 0; g < out->geometry_count; ++g) {
    for (int a = 0; a < dim_; ++a) {
      out->geometry_sides[g][a] = static_cast<int32_t>(layout_.geometries[static_cast<size_t>(g)].side[a]);
    }
  }
  out->point_count = point_count_;
  out->chosen_geometry = geometry_;
  out->bin_count = static_cast<int64_t>(bins_);
}

}  // namespace b200nufft
