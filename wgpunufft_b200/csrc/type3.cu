// Type-3 plans: f(k) = sum_j c(j) exp(i isign s(k).x(j)).
//
// The composition follows the reference (src/type3.rs:288-345,
// src/gpu_type3.rs:53-430): per axis the source interval (half width X,
// center C) and target interval (half width S, center D) fix an outer grid of
// nf = next even 2,3,5-smooth length >= 2 sigma s x / pi + w + 1, with
// spacing h = 2 pi / nf and rescaling gamma = nf / (2 sigma s). Sources are
// rescaled to x' = (x - C) / gamma and their strengths pre-phased by
// exp(i isign x.D); a type-1 spread (no FFT) puts them on the outer grid; the
// outer grid is the centered mode array of an inner type-2 NUFFT evaluated at
// the rescaled targets s' = h gamma (s - D); the result is multiplied by
// exp(i isign (s - D).C) / prod_a phi_hat(s'_a), phi_hat being the window's
// continuous Fourier transform by a (w + 2)-node half-interval Gauss-Legendre
// rule (es_kernel_fourier_transform, src/type3.rs:688-706). The pre- and
// post-phase run in native f64 for every precision, with CUDA's sincos, so
// phases of any magnitude are accurate (the reference bounds them because
// its shaders reduce phases by polynomials).
#include "type3.h"

#include <cmath>
#include <cstring>
#include <limits>
#include <string>

#include "util.h"

namespace b200nufft {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kCenterSnapFraction = 0.1;
constexpr uint64_t kMaxGridPoints = 1000000000000ull;

// NufftInterval::half_width_and_center with the center-snapping rule
// (src/type3.rs:64-85).
void half_width_and_center(double lower, double upper, const char* set, int axis, double& half,
                           double& center) {
  if (!std::isfinite(lower) || !std::isfinite(upper)) {
    throw NufftFailure{B200NUFFT_INVALID_TYPE3_INTERVAL,
                       std::string(set) + " interval of axis " + std::to_string(axis) +
                           ": endpoints must be finite"};
  }
  if (lower > upper) {
    throw NufftFailure{B200NUFFT_INVALID_TYPE3_INTERVAL,
                       std::string(set) + " interval of axis " + std::to_string(axis) +
                           ": lower endpoint exceeds upper endpoint"};
  }
  half = (upper - lower) * 0.5;
  center = (upper + lower) * 0.5;
  if (!std::isfinite(half) || !std::isfinite(center)) {
    throw NufftFailure{B200NUFFT_INVALID_TYPE3_INTERVAL, "interval width or center overflows f64"};
  }
  if (std::fabs(center) < kCenterSnapFraction * half) {
    half += std::fabs(center);
    center = 0.0;
  }
}

// next_even_235 (src/type3.rs:763-797): the least 2^a 3^b 5^c >= minimum, a >= 1.
int64_t next_even_235(int64_t minimum, int axis, uint64_t maximum) {
  minimum = std::max<int64_t>(minimum, 2);
  uint64_t best = 0;
  for (uint64_t p2 = 2; p2 <= maximum; p2 *= 2) {
    for (uint64_t p3 = p2; p3 <= maximum; p3 *= 3) {
      for (uint64_t c = p3; c <= maximum; c *= 5) {
        if (c >= static_cast<uint64_t>(minimum)) {
          if (best == 0 || c < best) best = c;
          break;
        }
        if (c > maximum / 5) break;
      }
      if (p3 > maximum / 3) break;
    }
    if (p2 > maximum / 2) break;
  }
  if (best == 0) {
    throw NufftFailure{B200NUFFT_TYPE3_GRID_SIZE_UNSUPPORTED,
                       "axis " + std::to_string(axis) + ": no even 2,3,5-smooth grid length fits"};
  }
  return static_cast<int64_t>(best);
}

// select_axis_metadata (src/type3.rs:708-761).
Type3Axis select_axis(int axis, double source_half, double source_center, double target_half,
                      double target_center, double sigma, int width, uint64_t maximum) {
  double x = source_half;
  double s = target_half;
  if (x == 0.0) {
    if (s == 0.0) {
      x = 1.0;
      s = 1.0;
    } else {
      x = 1.0 / s;
    }
  } else {
    s = std::max(s, 1.0 / x);
  }
  const double requested = 2.0 * sigma * s * x / kPi + static_cast<double>(width + 1);
  if (!std::isfinite(requested) || requested > static_cast<double>(maximum)) {
    throw NufftFailure{B200NUFFT_TYPE3_GRID_SIZE_UNSUPPORTED,
                       "axis " + std::to_string(axis) +
                           ": source-target space-bandwidth product is too large"};
  }
  const int64_t minimum = std::max<int64_t>(static_cast<int64_t>(requested), 2 * width);
  const int64_t outer = next_even_235(minimum, axis, maximum);
  Type3Axis a;
  a.source_half_width = source_half;
  a.source_center = source_center;
  a.target_half_width = target_half;
  a.target_center = target_center;
  a.outer = outer;
  a.grid_spacing = 2.0 * kPi / static_cast<double>(outer);
  a.source_scale = static_cast<double>(outer) / (2.0 * sigma * s);
  if (!std::isfinite(a.source_scale) || a.source_scale <= 0.0) {
    throw NufftFailure{B200NUFFT_TYPE3_RESCALING_UNSUPPORTED,
                       "axis " + std::to_string(axis) + ": non-finite or non-positive gamma"};
  }
  return a;
}

template <typename In>
__device__ __forceinline__ double load_coordinate(const In* p, int64_t i) {
  return static_cast<double>(p[i]);
}

// Rescaled sources x' = (x - C) / gamma and pre-phase factors exp(i isign x.D).
template <int D, typename In, typename Out>
__global__ void source_kernel(Type3Params p, const In* __restrict__ sources, int64_t count,
                              Out* __restrict__ rescaled, double2* __restrict__ factors) {
  const int64_t j = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= count) return;
  double phase = 0.0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const double x = load_coordinate(sources, j * D + a);
    rescaled[j * D + a] = static_cast<Out>((x - p.source_center[a]) * p.source_inv_scale[a]);
    phase += x * p.target_center[a];
  }
  double s, c;
  sincos(static_cast<double>(p.isign) * phase, &s, &c);
  factors[j] = make_double2(c, s);
}

// Rescaled targets s' = h gamma (s - D) and post-phase factors
// exp(i isign (s - D).C) / prod_a phi_hat(s'_a).
template <int D, typename In, typename Out>
__global__ void target_kernel(Type3Params p, const In* __restrict__ targets, int64_t count,
                              Out* __restrict__ rescaled, double2* __restrict__ factors) {
  const int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (k >= count) return;
  double phase = 0.0;
  double phi = 1.0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const double centered = load_coordinate(targets, k * D + a) - p.target_center[a];
    const double scaled = centered * p.target_scale[a];
    rescaled[k * D + a] = static_cast<Out>(scaled);
    phase += centered * p.source_center[a];
    double transform = 0.0;
    for (int n = 0; n < p.quadrature_count; ++n) transform += p.weights[n] * cos(scaled * p.nodes[n]);
    phi *= transform;
  }
  double s, c;
  sincos(static_cast<double>(p.isign) * phase, &s, &c);
  const double inverse = 1.0 / phi;
  factors[k] = make_double2(inverse * c, inverse * s);
}

// value * factor, per vector; computed in f64.
template <typename Complex>
__global__ void multiply_kernel(const Complex* __restrict__ values,
                                const double2* __restrict__ factors, int64_t count, int batch,
                                Complex* __restrict__ out) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count * batch) return;
  const Complex v = values[i];
  const double2 f = factors[i % count];
  const double re = static_cast<double>(v.x) * f.x - static_cast<double>(v.y) * f.y;
  const double im = static_cast<double>(v.x) * f.y + static_cast<double>(v.y) * f.x;
  Complex o;
  o.x = static_cast<decltype(o.x)>(re);
  o.y = static_cast<decltype(o.y)>(im);
  out[i] = o;
}

template <typename In, typename Out>
void launch_rescale(bool sources, const Type3Params& p, const void* in, int64_t count, void* rescaled,
                    double2* factors, cudaStream_t stream) {
  const unsigned blocks = static_cast<unsigned>((count + 255) / 256);
  const In* src = static_cast<const In*>(in);
  Out* out = static_cast<Out*>(rescaled);
  switch (p.dimensions) {
    case 1:
      if (sources) source_kernel<1, In, Out><<<blocks, 256, 0, stream>>>(p, src, count, out, factors);
      else target_kernel<1, In, Out><<<blocks, 256, 0, stream>>>(p, src, count, out, factors);
      break;
    case 2:
      if (sources) source_kernel<2, In, Out><<<blocks, 256, 0, stream>>>(p, src, count, out, factors);
      else target_kernel<2, In, Out><<<blocks, 256, 0, stream>>>(p, src, count, out, factors);
      break;
    default:
      if (sources) source_kernel<3, In, Out><<<blocks, 256, 0, stream>>>(p, src, count, out, factors);
      else target_kernel<3, In, Out><<<blocks, 256, 0, stream>>>(p, src, count, out, factors);
      break;
  }
  note_launch();
}

}  // namespace

Type3Plan::Type3Plan(const b200nufft_type3_config& c) {
  if (c.dimensions < 1 || c.dimensions > 8) {
    throw NufftFailure{B200NUFFT_INVALID_DIMENSIONS, "dimensions must lie in 1..8"};
  }
  if (c.dimensions > B200NUFFT_MAX_TYPE3_DIMENSIONS) {
    throw NufftFailure{B200NUFFT_GPU_DIMENSIONS_UNSUPPORTED, "GPU type-3 plans support 1 to 3 dimensions"};
  }
  if (c.batch <= 0) throw NufftFailure{B200NUFFT_INVALID_BATCH, "batch must be at least one"};
  dim_ = c.dimensions;
  batch_ = c.batch;
  eps_ = c.eps;
  isign_ = c.isign >= 0 ? 1 : -1;
  sigma_ = c.sigma == 0.0 ? 2.0 : c.sigma;
  precision_ = c.precision == 0 ? B200NUFFT_PRECISION_F64 : c.precision;
  if (precision_ != B200NUFFT_PRECISION_F32 && precision_ != B200NUFFT_PRECISION_F64 &&
      precision_ != B200NUFFT_PRECISION_DF64) {
    throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "precision must be F64 (1), DF64 (2) or F32 (3)"};
  }
  kernel_ = EsKernel::for_tolerance(eps_, sigma_);
  uint64_t volume = 1;
  for (int a = 0; a < dim_; ++a) {
    double sh, sc, th, tc;
    half_width_and_center(c.source_lower[a], c.source_upper[a], "source", a, sh, sc);
    half_width_and_center(c.target_lower[a], c.target_upper[a], "target", a, th, tc);
    const Type3Axis axis = select_axis(a, sh, sc, th, tc, sigma_, kernel_.width, kMaxGridPoints);
    if (static_cast<double>(volume) * static_cast<double>(axis.outer) > static_cast<double>(kMaxGridPoints)) {
      throw NufftFailure{B200NUFFT_TYPE3_GRID_SIZE_UNSUPPORTED, "outer grid volume above 10^12 cells"};
    }
    volume *= static_cast<uint64_t>(axis.outer);
    axes_.push_back(axis);
  }
  // Window transform by the (w + 2) positive nodes of a 2 (w + 2)-point rule;
  // f64 plans integrate the Horner polynomial their spreading uses, f32
  // plans the exact window (src/gpu_type3.rs:1567-1592).
  const bool horner = precision_ != B200NUFFT_PRECISION_F32;
  EsHornerTable table;
  if (horner) table = EsHornerTable::fit(kernel_);
  std::memset(&params_, 0, sizeof(params_));
  params_.dimensions = dim_;
  params_.isign = isign_;
  const int count = kernel_.width + 2;
  std::vector<double> nodes, weights;
  gauss_legendre(2 * count, nodes, weights);
  params_.quadrature_count = count;
  for (int n = 0; n < count; ++n) {
    const double distance = kernel_.half_width() * nodes[count + n];
    params_.nodes[n] = distance;
    params_.weights[n] = 2.0 * kernel_.half_width() * weights[count + n] *
                         (horner ? table.evaluate(distance) : kernel_.evaluate(distance));
  }
  for (int a = 0; a < dim_; ++a) {
    params_.source_center[a] = axes_[a].source_center;
    params_.source_inv_scale[a] = 1.0 / axes_[a].source_scale;
    params_.target_center[a] = axes_[a].target_center;
    params_.target_scale[a] = axes_[a].grid_spacing * axes_[a].source_scale;
  }
  // Outer spread: a type-1 plan whose fine grid is the outer grid; inner: a
  // type-2 plan whose centered modes are the outer grid.
  const int inner_precision =
      precision_ == B200NUFFT_PRECISION_DF64 ? B200NUFFT_PRECISION_F64 : precision_;
  b200nufft_config outer{};
  outer.type = 1;
  outer.dimensions = dim_;
  outer.batch = batch_;
  outer.eps = eps_;
  outer.isign = isign_;
  outer.mode_order = B200NUFFT_MODE_ORDER_CENTERED;
  outer.sigma = sigma_;
  outer.precision = inner_precision;
  outer.device = c.device;
  // The outer spread runs through spread_to, on the CUDA cores.
  outer.spread_method = B200NUFFT_SPREAD_CUDA_CORES;
  b200nufft_config inner = outer;
  inner.type = 2;
  for (int a = 0; a < dim_; ++a) {
    outer.n_modes[a] = axes_[a].outer / 2;
    inner.n_modes[a] = axes_[a].outer;
  }
  outer_ = std::make_unique<NufftPlan>(outer, true);
  for (int a = 0; a < dim_; ++a) {
    if (outer_->fine_shape()[a] != axes_[a].outer) {
      throw NufftFailure{B200NUFFT_LENGTH_OVERFLOW, "type-3 outer spread grid differs from the outer grid"};
    }
  }
  inner_ = std::make_unique<NufftPlan>(inner, true);
  device_ = outer_->device();
}

void Type3Plan::set_points(int64_t source_count, const void* sources, int64_t target_count,
                           const void* targets, cudaStream_t stream) {
  check_cuda(cudaSetDevice(device_), "select plan device");
  if (source_count < 0 || target_count < 0) {
    throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "negative point count"};
  }
  if ((source_count > 0 && !sources) || (target_count > 0 && !targets)) {
    throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null source or target buffer"};
  }
  const bool f32 = precision_ == B200NUFFT_PRECISION_F32;
  const size_t real = f32 ? sizeof(float) : sizeof(double);
  const void* src = sources;
  const void* tgt = targets;
  if (precision_ == B200NUFFT_PRECISION_DF64) {
    double* s64 = static_cast<double*>(sources64_.reserve(std::max<int64_t>(source_count, 1) * dim_ * 8, "f64 sources"));
    double* t64 = static_cast<double*>(targets64_.reserve(std::max<int64_t>(target_count, 1) * dim_ * 8, "f64 targets"));
    df64_to_f64(static_cast<const float*>(sources), source_count * dim_, s64, stream);
    df64_to_f64(static_cast<const float*>(targets), target_count * dim_, t64, stream);
    src = s64;
    tgt = t64;
  }
  void* xs = rescaled_sources_.reserve(std::max<int64_t>(source_count, 1) * dim_ * real, "rescaled sources");
  double2* sf = static_cast<double2*>(source_factors_.reserve(std::max<int64_t>(source_count, 1) * 16, "source factors"));
  void* ts = rescaled_targets_.reserve(std::max<int64_t>(target_count, 1) * dim_ * real, "rescaled targets");
  double2* tf = static_cast<double2*>(target_factors_.reserve(std::max<int64_t>(target_count, 1) * 16, "target factors"));
  if (source_count > 0) {
    if (f32) launch_rescale<float, float>(true, params_, src, source_count, xs, sf, stream);
    else launch_rescale<double, double>(true, params_, src, source_count, xs, sf, stream);
  }
  if (target_count > 0) {
    if (f32) launch_rescale<float, float>(false, params_, tgt, target_count, ts, tf, stream);
    else launch_rescale<double, double>(false, params_, tgt, target_count, ts, tf, stream);
  }
  outer_->set_points(source_count, xs, stream);
  inner_->set_points(target_count, ts, stream);
  source_count_ = source_count;
  target_count_ = target_count;
  check_cuda(cudaGetLastError(), "type-3 set points");
}

void Type3Plan::execute(int64_t active_batch, const void* strengths, void* output, cudaStream_t stream) {
  check_cuda(cudaSetDevice(device_), "select plan device");
  if (active_batch <= 0 || active_batch > batch_) {
    throw NufftFailure{B200NUFFT_INVALID_BATCH, "active batch outside 1..batch"};
  }
  if (source_count_ < 0) {
    throw NufftFailure{B200NUFFT_GPU_EXECUTION_UNAVAILABLE, "set the type-3 points before executing"};
  }
  const int batch = static_cast<int>(active_batch);
  if (target_count_ == 0) return;
  if (!output || (source_count_ > 0 && !strengths)) {
    throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null strengths or output"};
  }
  const bool f32 = precision_ == B200NUFFT_PRECISION_F32;
  const size_t complex_bytes = f32 ? 8 : 16;
  const void* in = strengths;
  void* out = output;
  if (precision_ == B200NUFFT_PRECISION_DF64) {
    double* s64 = static_cast<double*>(strengths64_.reserve(std::max<int64_t>(source_count_, 1) * batch * 16, "f64 strengths"));
    df64_to_f64(static_cast<const float*>(strengths), source_count_ * batch * 2, s64, stream);
    in = s64;
    out = output64_.reserve(static_cast<size_t>(target_count_) * batch * 16, "f64 output");
  }
  void* prephased = prephased_.reserve(std::max<int64_t>(source_count_, 1) * batch * complex_bytes, "prephased strengths");
  void* grid = outer_grid_.reserve(static_cast<size_t>(outer_->fine_count()) * batch * complex_bytes, "outer grid");
  void* interpolated = interpolated_.reserve(static_cast<size_t>(target_count_) * batch * complex_bytes, "interpolated values");
  const double2* sf = static_cast<const double2*>(source_factors_.get());
  const double2* tf = static_cast<const double2*>(target_factors_.get());
  if (source_count_ > 0) {
    const int64_t n = source_count_ * batch;
    const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
    if (f32) {
      multiply_kernel<float2><<<blocks, 256, 0, stream>>>(static_cast<const float2*>(in), sf, source_count_, batch,
                                                         static_cast<float2*>(prephased));
    } else {
      multiply_kernel<double2><<<blocks, 256, 0, stream>>>(static_cast<const double2*>(in), sf, source_count_,
                                                          batch, static_cast<double2*>(prephased));
    }
    note_launch();
  }
  outer_->spread_to(batch, prephased, grid, stream);
  inner_->execute(batch, grid, interpolated, stream);
  const int64_t n = target_count_ * batch;
  const unsigned blocks = static_cast<unsigned>((n + 255) / 256);
  if (f32) {
    multiply_kernel<float2><<<blocks, 256, 0, stream>>>(static_cast<const float2*>(interpolated), tf,
                                                       target_count_, batch, static_cast<float2*>(out));
  } else {
    multiply_kernel<double2><<<blocks, 256, 0, stream>>>(static_cast<const double2*>(interpolated), tf,
                                                        target_count_, batch, static_cast<double2*>(out));
  }
  note_launch();
  if (precision_ == B200NUFFT_PRECISION_DF64) {
    f64_to_df64(static_cast<const double*>(out), target_count_ * batch * 2, static_cast<float*>(output), stream);
  }
  check_cuda(cudaGetLastError(), "type-3 execute");
}

void Type3Plan::info(b200nufft_type3_info* out) const {
  std::memset(out, 0, sizeof(*out));
  out->dimensions = dim_;
  out->kernel_width = kernel_.width;
  out->kernel_beta = kernel_.beta;
  for (int a = 0; a < dim_; ++a) {
    out->outer_shape[a] = axes_[a].outer;
    out->inner_fine_shape[a] = inner_->fine_shape()[a];
    out->source_center[a] = axes_[a].source_center;
    out->target_center[a] = axes_[a].target_center;
    out->gamma[a] = axes_[a].source_scale;
    out->h[a] = axes_[a].grid_spacing;
  }
}

}  // namespace b200nufft
