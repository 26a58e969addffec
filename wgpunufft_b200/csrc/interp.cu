// Type-2 interpolation of the transformed fine grid at the nonuniform
// points.
//
// Each thread evaluates one point, visited in bin order so that neighbouring
// threads read the same fine-grid rows from cache: it folds the coordinate,
// evaluates the window per axis into registers once, and then sums the w^d
// support cells of every vector in a fixed order, so every output is bitwise
// repeatable (the reference sums its lanes in lane order,
// src/gpu_2d.rs:1022-1113). Values are written in input order. A point
// outside the fold's reach gets zero weight, as the reference's prepared
// offsets past the support give it (src/gpu_nd_bins.rs:31-33). f32 plans use
// the exp window of the reference's f32 shaders, f64 plans its Horner table
// (src/gpu_nd_wgsl.rs:373-481).
#include <cuda_runtime.h>

#include "device.h"
#include "interp.h"

namespace b200nufft {

namespace {

struct F32Window {
  static constexpr bool kPreparedWindows = true;
  using Real = float;
  using Complex = float2;
  static __device__ __forceinline__ bool in_reach(float x) { return in_fold_reach(x); }
  template <int W>
  static __device__ __forceinline__ void window(float x, const GridParams& g, int a, int& first,
                                                float* w) {
    int32_t start;
    Df64 off;
    support_of(x, g.axis[a], g.half_width, start, off);
    first = wrap_start(start, g.axis[a].length);
    const float width_f = static_cast<float>(W);
#pragma unroll
    for (int j = 0; j < W; ++j) {
      const float d = __fadd_rn(__fadd_rn(static_cast<float>(j), off.hi), off.lo);
      w[j] = es_weight(d, g.beta, width_f);
    }
  }
  static __device__ __forceinline__ float fma_(float a, float b, float c) { return fmaf(a, b, c); }
};

struct F64Window {
  static constexpr bool kPreparedWindows = false;
  using Real = double;
  using Complex = double2;
  static __device__ __forceinline__ bool in_reach(double x) { return in_fold_reach64(x); }
  template <int W>
  static __device__ __forceinline__ void window(double x, const GridParams& g, int a, int& first,
                                                double* w) {
    int32_t start;
    double offset;
    support_of64(x, g.axis64[a], g.half_width64, start, offset);
    first = wrap_start(start, g.axis[a].length);
#pragma unroll
    for (int j = 0; j < W; ++j) w[j] = horner_weight(offset, j, W, g.horner, g.horner_rows);
  }
  static __device__ __forceinline__ double fma_(double a, double b, double c) { return fma(a, b, c); }
};

// Resident blocks per SM the register budget is tuned for: narrow 1D and 2D
// f32 windows (w <= 4) fit three 256-thread blocks without spilling, the others two.
template <int D, int W, typename T>
struct InterpBlocks {
  static constexpr int value = (D <= 2 && W <= 4 && sizeof(typename T::Real) == 4) ? 3 : 2;
};

template <int D, int W, typename T>
__global__ void __launch_bounds__(256, InterpBlocks<D, W, T>::value)
    interpolate_kernel(GridParams g, const typename T::Real* __restrict__ points,
                       const void* __restrict__ windows, int64_t count,
                       const uint32_t* __restrict__ perm,
                       const typename T::Complex* __restrict__ fine, int batch,
                       typename T::Complex* __restrict__ output) {
  using Real = typename T::Real;
  using Complex = typename T::Complex;
  const int64_t slot = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (slot >= count) return;
  const uint32_t point = perm[slot];
  int first[D];
  Real w[D][W];
  bool reach = true;
  if constexpr (T::kPreparedWindows) {
    // f32 plans: the window start and offset prepared at set_points.
    const PreparedWindow<D> win = static_cast<const PreparedWindow<D>*>(windows)[slot];
    reach = win.start[0] >= 0;
    if (reach) {
#pragma unroll
      for (int a = 0; a < D; ++a) {
        first[a] = win.start[a];
        horner32_window<W>(win.offset[a], g.horner32, w[a]);
      }
    }
  } else {
    Real p[D];
#pragma unroll
    for (int a = 0; a < D; ++a) p[a] = points[slot * D + a];
#pragma unroll
    for (int a = 0; a < D; ++a) reach = reach && T::in_reach(p[a]);
    if (reach) {
#pragma unroll
      for (int a = 0; a < D; ++a) T::template window<W>(p[a], g, a, first[a], w[a]);
    }
  }
  if (!reach) {
    Complex zero;
    zero.x = 0;
    zero.y = 0;
    for (int b = 0; b < batch; ++b) output[static_cast<int64_t>(b) * count + point] = zero;
    return;
  }
  const int32_t n0 = g.axis[0].length;
  int x[W];
#pragma unroll
  for (int i = 0; i < W; ++i) {
    const int c = first[0] + i;
    x[i] = c >= n0 ? c - n0 : c;
  }
  for (int b = 0; b < batch; ++b) {
    const Complex* grid = fine + static_cast<int64_t>(b) * g.fine_count;
    Real re = 0, im = 0;
    if (D == 1) {
#pragma unroll
      for (int i = 0; i < W; ++i) {
        const Complex v = __ldg(&grid[x[i]]);
        re = T::fma_(v.x, w[0][i], re);
        im = T::fma_(v.y, w[0][i], im);
      }
    } else if (D == 2) {
      const int32_t n1 = g.axis[1].length;
#pragma unroll
      for (int j = 0; j < W; ++j) {
        int y = first[1] + j;
        y = y >= n1 ? y - n1 : y;
        const Complex* row = grid + static_cast<int64_t>(y) * n0;
        Real rr = 0, ri = 0;
#pragma unroll
        for (int i = 0; i < W; ++i) {
          const Complex v = __ldg(&row[x[i]]);
          rr = T::fma_(v.x, w[0][i], rr);
          ri = T::fma_(v.y, w[0][i], ri);
        }
        re = T::fma_(rr, w[1][j], re);
        im = T::fma_(ri, w[1][j], im);
      }
    } else {
      const int32_t n1 = g.axis[1].length;
      const int32_t n2 = g.axis[2].length;
#pragma unroll 1
      for (int k = 0; k < W; ++k) {
        int z = first[2] + k;
        z = z >= n2 ? z - n2 : z;
        Real pr = 0, pi = 0;
#pragma unroll
        for (int j = 0; j < W; ++j) {
          int y = first[1] + j;
          y = y >= n1 ? y - n1 : y;
          const Complex* row = grid + (static_cast<int64_t>(z) * n1 + y) * n0;
          Real rr = 0, ri = 0;
#pragma unroll
          for (int i = 0; i < W; ++i) {
            const Complex v = __ldg(&row[x[i]]);
            rr = T::fma_(v.x, w[0][i], rr);
            ri = T::fma_(v.y, w[0][i], ri);
          }
          pr = T::fma_(rr, w[1][j], pr);
          pi = T::fma_(ri, w[1][j], pi);
        }
        re = T::fma_(pr, w[2][k], re);
        im = T::fma_(pi, w[2][k], im);
      }
    }
    Complex o;
    o.x = re;
    o.y = im;
    output[static_cast<int64_t>(b) * count + point] = o;
  }
}

template <typename T>
struct Launch {
  const typename T::Real* points;
  const void* windows;
  int64_t point_count;
  const uint32_t* perm;
  const typename T::Complex* fine;
  int batch;
  typename T::Complex* output;
};

template <int D, int W, typename T>
void launch_width(const GridParams& g, const Launch<T>& l, cudaStream_t stream) {
  const unsigned blocks = static_cast<unsigned>((l.point_count + 255) / 256);
  interpolate_kernel<D, W, T><<<blocks, 256, 0, stream>>>(g, l.points, l.windows, l.point_count, l.perm,
                                                           l.fine, l.batch, l.output);
  note_launch();
}

template <int D, typename T>
void launch_dim(const GridParams& g, const Launch<T>& l, cudaStream_t stream) {
  switch (g.width) {
    case 2: launch_width<D, 2, T>(g, l, stream); break;
    case 3: launch_width<D, 3, T>(g, l, stream); break;
    case 4: launch_width<D, 4, T>(g, l, stream); break;
    case 5: launch_width<D, 5, T>(g, l, stream); break;
    case 6: launch_width<D, 6, T>(g, l, stream); break;
    case 7: launch_width<D, 7, T>(g, l, stream); break;
    case 8: launch_width<D, 8, T>(g, l, stream); break;
    case 9: launch_width<D, 9, T>(g, l, stream); break;
    case 10: launch_width<D, 10, T>(g, l, stream); break;
    case 11: launch_width<D, 11, T>(g, l, stream); break;
    case 12: launch_width<D, 12, T>(g, l, stream); break;
    case 13: launch_width<D, 13, T>(g, l, stream); break;
    case 14: launch_width<D, 14, T>(g, l, stream); break;
    case 15: launch_width<D, 15, T>(g, l, stream); break;
    default: launch_width<D, 16, T>(g, l, stream); break;
  }
}

template <typename T>
void execute_impl(const GridParams& g, const Launch<T>& l, cudaStream_t stream) {
  if (l.point_count == 0) return;
  switch (g.dimensions) {
    case 1: launch_dim<1, T>(g, l, stream); break;
    case 2: launch_dim<2, T>(g, l, stream); break;
    default: launch_dim<3, T>(g, l, stream); break;
  }
}

}  // namespace

void interpolate_execute(const GridParams& g, const InterpLaunch& l, cudaStream_t stream) {
  execute_impl<F32Window>(g, Launch<F32Window>{l.points, l.windows, l.point_count, l.perm, l.fine, l.batch, l.output},
                          stream);
}

void interpolate_execute64(const GridParams& g, const InterpLaunch64& l, cudaStream_t stream) {
  execute_impl<F64Window>(g, Launch<F64Window>{l.points, nullptr, l.point_count, l.perm, l.fine, l.batch, l.output},
                          stream);
}

}  // namespace b200nufft
