// Type-1 spreading and type-2 interpolation of plans with 4 to 8 dimensions,
// the reference's rank-generic path (src/gpu_nd.rs, src/gpu_nd_spread.rs for
// d >= 4). Windows grow as w^d, so these plans have small grids and point
// sets; the kernels favour generality over locality: no bin sort, a thread
// per point walking its window cell by cell.
//
// Spreading stays bitwise repeatable without ordering the threads: every
// contribution is scaled by 2^S_b (S_b from the largest strength of vector b
// and the point count, so that no cell's sum can reach 2^62), rounded to a
// 64-bit integer and added to the fine grid with 64-bit integer atomics,
// whose sums do not depend on their order; a second pass converts the
// integer grid back to floating point. Interpolation sums each point's window
// in a fixed order.
#include <cuda_runtime.h>

#include <algorithm>

#include "nd.h"

namespace b200nufft {

namespace {

constexpr int kNdThreads = 256;
constexpr int kNdMaxWidth = 16;

template <typename Real>
struct NdTypes;
template <>
struct NdTypes<float> {
  using Complex = float2;
};
template <>
struct NdTypes<double> {
  using Complex = double2;
};

// Wrapped support starts and window weights of one point on every axis;
// false when a coordinate lies outside the fold reach (weighed zero).
template <typename Real>
__device__ bool nd_window(const NdParams& p, const Real* x, int32_t* start, double (*w)[kNdMaxWidth]) {
  const int D = p.dimensions, W = p.width;
  for (int a = 0; a < D; ++a) {
    if constexpr (sizeof(Real) == 4) {
      if (!in_fold_reach(x[a])) return false;
    } else {
      if (!in_fold_reach64(x[a])) return false;
    }
  }
  for (int a = 0; a < D; ++a) {
    if constexpr (sizeof(Real) == 4) {
      int32_t s;
      Df64 off;
      support_of(x[a], p.axis[a], p.half_width, s, off);
      start[a] = wrap_start(s, p.axis[a].length);
      const float width_f = static_cast<float>(W);
      for (int j = 0; j < W; ++j) {
        const float d = __fadd_rn(__fadd_rn(static_cast<float>(j), off.hi), off.lo);
        w[a][j] = es_weight(d, p.beta, width_f);
      }
    } else {
      int32_t s;
      double offset;
      support_of64(x[a], p.axis64[a], p.half_width64, s, offset);
      start[a] = wrap_start(s, p.axis[a].length);
      for (int j = 0; j < W; ++j) w[a][j] = horner_weight(offset, j, W, p.horner, p.horner_rows);
    }
  }
  return true;
}

// Largest |re| or |im| of every vector, as the bits of a non-negative double.
template <typename Complex>
__global__ void nd_strength_bits_kernel(const Complex* __restrict__ values, int64_t count, int batch,
                                        unsigned long long* __restrict__ max_bits) {
  const int b = blockIdx.y;
  const Complex* v = values + static_cast<int64_t>(b) * count;
  double m = 0.0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    m = fmax(m, fabs(static_cast<double>(v[i].x)));
    m = fmax(m, fabs(static_cast<double>(v[i].y)));
  }
  for (int offset = 16; offset > 0; offset >>= 1) m = fmax(m, __shfl_xor_sync(0xFFFFFFFFu, m, offset));
  if ((threadIdx.x & 31) == 0 && m > 0.0) {
    atomicMax(&max_bits[b], static_cast<unsigned long long>(__double_as_longlong(m)));
  }
}

// 2^S_b: contributions of vector b scaled below 2^(62 - headroom), so that
// count of them stay below 2^62 in any cell. Non-finite maxima leave the
// outputs unspecified but the scale bounded.
__device__ __forceinline__ int nd_exponent(unsigned long long bits, int headroom) {
  if (bits == 0ull) return 0;
  const double m = __longlong_as_double(static_cast<long long>(bits));
  const int e = isfinite(m) ? ilogb(m) + 1 : 1024;
  return 62 - headroom - e;
}

template <typename Real, typename Complex>
__global__ void __launch_bounds__(kNdThreads) nd_spread_kernel(NdParams p, const Real* __restrict__ points,
                                                               const Complex* __restrict__ strengths,
                                                               int64_t count, int batch, int headroom,
                                                               const unsigned long long* __restrict__ max_bits,
                                                               unsigned long long* __restrict__ acc) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int D = p.dimensions, W = p.width;
  Real x[kNdMaxDimensions];
  for (int a = 0; a < D; ++a) x[a] = points[i * D + a];
  int32_t start[kNdMaxDimensions];
  double w[kNdMaxDimensions][kNdMaxWidth];
  if (!nd_window<Real>(p, x, start, w)) return;
  int64_t cells = 1;
  for (int a = 0; a < D; ++a) cells *= W;
  for (int b = 0; b < batch; ++b) {
    const Complex c = strengths[static_cast<int64_t>(b) * count + i];
    const double scale = ldexp(1.0, nd_exponent(max_bits[b], headroom));
    const double sr = static_cast<double>(c.x) * scale, si = static_cast<double>(c.y) * scale;
    unsigned long long* grid = acc + 2 * static_cast<int64_t>(b) * p.fine_count;
    int idx[kNdMaxDimensions];
    for (int a = 0; a < D; ++a) idx[a] = 0;
    for (int64_t k = 0; k < cells; ++k) {
      double weight = 1.0;
      int64_t cell = 0, stride = 1;
      for (int a = 0; a < D; ++a) {
        weight *= w[a][idx[a]];
        int32_t g = start[a] + idx[a];
        g = g >= p.axis[a].length ? g - p.axis[a].length : g;
        cell += g * stride;
        stride *= p.fine[a];
      }
      atomicAdd(&grid[2 * cell], static_cast<unsigned long long>(__double2ll_rn(sr * weight)));
      atomicAdd(&grid[2 * cell + 1], static_cast<unsigned long long>(__double2ll_rn(si * weight)));
      for (int a = 0; a < D; ++a) {
        if (++idx[a] < W) break;
        idx[a] = 0;
      }
    }
  }
}

template <typename Real, typename Complex>
__global__ void nd_finish_kernel(int64_t fine_count, int batch, int headroom,
                                 const unsigned long long* __restrict__ max_bits,
                                 const unsigned long long* __restrict__ acc, Complex* __restrict__ fine) {
  const int64_t cell = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (cell >= fine_count) return;
  const int S = nd_exponent(max_bits[b], headroom);
  const int64_t at = static_cast<int64_t>(b) * fine_count + cell;
  Complex v;
  v.x = static_cast<Real>(ldexp(static_cast<double>(static_cast<long long>(acc[2 * at])), -S));
  v.y = static_cast<Real>(ldexp(static_cast<double>(static_cast<long long>(acc[2 * at + 1])), -S));
  fine[at] = v;
}

template <typename Real, typename Complex>
__global__ void __launch_bounds__(kNdThreads) nd_interpolate_kernel(NdParams p, const Real* __restrict__ points,
                                                                    const Complex* __restrict__ fine,
                                                                    int64_t count, int batch,
                                                                    Complex* __restrict__ output) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int D = p.dimensions, W = p.width;
  Real x[kNdMaxDimensions];
  for (int a = 0; a < D; ++a) x[a] = points[i * D + a];
  int32_t start[kNdMaxDimensions];
  double w[kNdMaxDimensions][kNdMaxWidth];
  const bool reach = nd_window<Real>(p, x, start, w);
  int64_t cells = 1;
  for (int a = 0; a < D; ++a) cells *= W;
  for (int b = 0; b < batch; ++b) {
    Real re = 0, im = 0;
    if (reach) {
      const Complex* grid = fine + static_cast<int64_t>(b) * p.fine_count;
      int idx[kNdMaxDimensions];
      for (int a = 0; a < D; ++a) idx[a] = 0;
      for (int64_t k = 0; k < cells; ++k) {
        double weight = 1.0;
        int64_t cell = 0, stride = 1;
        for (int a = 0; a < D; ++a) {
          weight *= w[a][idx[a]];
          int32_t g = start[a] + idx[a];
          g = g >= p.axis[a].length ? g - p.axis[a].length : g;
          cell += g * stride;
          stride *= p.fine[a];
        }
        const Complex v = grid[cell];
        const Real r = static_cast<Real>(weight);
        re += v.x * r;
        im += v.y * r;
        for (int a = 0; a < D; ++a) {
          if (++idx[a] < W) break;
          idx[a] = 0;
        }
      }
    }
    Complex o;
    o.x = re;
    o.y = im;
    output[static_cast<int64_t>(b) * count + i] = o;
  }
}

int ceil_log2(int64_t v) {
  int bits = 0;
  while ((int64_t(1) << bits) < v) ++bits;
  return bits;
}

template <typename Real>
void spread_typed(const NdParams& p, const void* points, const void* strengths, int64_t count, int batch,
                  unsigned long long* acc, unsigned long long* max_bits, void* fine, cudaStream_t stream) {
  using Complex = typename NdTypes<Real>::Complex;
  check_cuda(cudaMemsetAsync(acc, 0, 2 * sizeof(unsigned long long) * batch * p.fine_count, stream),
             "clear integer grid");
  check_cuda(cudaMemsetAsync(max_bits, 0, sizeof(unsigned long long) * batch, stream), "clear maxima");
  const int headroom = ceil_log2(count + 1);
  if (count > 0) {
    const unsigned blocks = static_cast<unsigned>(std::min<int64_t>((count + kNdThreads - 1) / kNdThreads, 148 * 8));
    nd_strength_bits_kernel<Complex><<<dim3(blocks, batch), kNdThreads, 0, stream>>>(
        static_cast<const Complex*>(strengths), count, batch, max_bits);
    nd_spread_kernel<Real, Complex><<<static_cast<unsigned>((count + kNdThreads - 1) / kNdThreads), kNdThreads, 0,
                                      stream>>>(p, static_cast<const Real*>(points),
                                                static_cast<const Complex*>(strengths), count, batch, headroom,
                                                max_bits, acc);
    note_launch(2);
  }
  const dim3 grid(static_cast<unsigned>((p.fine_count + kNdThreads - 1) / kNdThreads), static_cast<unsigned>(batch));
  nd_finish_kernel<Real, Complex><<<grid, kNdThreads, 0, stream>>>(p.fine_count, batch, headroom, max_bits, acc,
                                                                   static_cast<Complex*>(fine));
  note_launch();
}

}  // namespace

void nd_spread(const NdParams& p, const void* points, const void* strengths, int64_t count, int batch,
               unsigned long long* acc, unsigned long long* max_bits, void* fine, cudaStream_t stream) {
  if (p.f32) {
    spread_typed<float>(p, points, strengths, count, batch, acc, max_bits, fine, stream);
  } else {
    spread_typed<double>(p, points, strengths, count, batch, acc, max_bits, fine, stream);
  }
}

void nd_interpolate(const NdParams& p, const void* points, const void* fine, int64_t count, int batch,
                    void* output, cudaStream_t stream) {
  if (count == 0) return;
  const unsigned blocks = static_cast<unsigned>((count + kNdThreads - 1) / kNdThreads);
  if (p.f32) {
    nd_interpolate_kernel<float, float2><<<blocks, kNdThreads, 0, stream>>>(
        p, static_cast<const float*>(points), static_cast<const float2*>(fine), count, batch,
        static_cast<float2*>(output));
  } else {
    nd_interpolate_kernel<double, double2><<<blocks, kNdThreads, 0, stream>>>(
        p, static_cast<const double*>(points), static_cast<const double2*>(fine), count, batch,
        static_cast<double2*>(output));
  }
  note_launch();
}

}  // namespace b200nufft
