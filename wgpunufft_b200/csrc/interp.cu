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
// offsets past the support give it (src/gpu_nd_bins.rs:31-33).
#include <cuda_runtime.h>

#include "device.h"
#include "interp.h"

namespace b200nufft {

namespace {

__device__ __forceinline__ float es_weight(float distance, float beta, float width_f) {
  const float scaled = (2.0f * fabsf(distance)) / width_f;
  const float squared = scaled * scaled;
  if (squared >= 1.0f) return 0.0f;
  return expf(beta * (sqrtf(fmaxf(0.0f, 1.0f - squared)) - 1.0f));
}

// Resident blocks per SM the register budget is tuned for: narrow 1D and 2D
// windows fit three 256-thread blocks without spilling, wider ones two.
template <int D, int W>
struct InterpBlocks {
  static constexpr int value = (D <= 2 && W <= 6) ? 3 : 2;
};

template <int D, int W>
__global__ void __launch_bounds__(256, InterpBlocks<D, W>::value) interpolate_kernel(GridParams g,
                                                          const float* __restrict__ points,
                                                          int64_t count,
                                                          const uint32_t* __restrict__ perm,
                                                          const float2* __restrict__ fine,
                                                          int batch, float2* __restrict__ output) {
  const int64_t slot = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (slot >= count) return;
  const uint32_t point = perm[slot];
  float p[D];
#pragma unroll
  for (int a = 0; a < D; ++a) p[a] = points[slot * D + a];
  bool reach = true;
#pragma unroll
  for (int a = 0; a < D; ++a) reach = reach && in_fold_reach(p[a]);
  if (!reach) {
    for (int b = 0; b < batch; ++b) output[static_cast<int64_t>(b) * count + point] = make_float2(0.f, 0.f);
    return;
  }
  const float width_f = static_cast<float>(W);
  int first[D];
  float w[D][W];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    int32_t start;
    Df64 off;
    support_of(p[a], g.axis[a], g.half_width, start, off);
    first[a] = wrap_start(start, g.axis[a].length);
#pragma unroll
    for (int j = 0; j < W; ++j) {
      const float d = __fadd_rn(__fadd_rn(static_cast<float>(j), off.hi), off.lo);
      w[a][j] = es_weight(d, g.beta, width_f);
    }
  }
  const int32_t n0 = g.axis[0].length;
  int x[W];
#pragma unroll
  for (int i = 0; i < W; ++i) {
    const int c = first[0] + i;
    x[i] = c >= n0 ? c - n0 : c;
  }
  for (int b = 0; b < batch; ++b) {
    const float2* grid = fine + static_cast<int64_t>(b) * g.fine_count;
    float re = 0.0f, im = 0.0f;
    if (D == 1) {
#pragma unroll
      for (int i = 0; i < W; ++i) {
        const float2 v = __ldg(&grid[x[i]]);
        re = fmaf(v.x, w[0][i], re);
        im = fmaf(v.y, w[0][i], im);
      }
    } else if (D == 2) {
      const int32_t n1 = g.axis[1].length;
#pragma unroll
      for (int j = 0; j < W; ++j) {
        int y = first[1] + j;
        y = y >= n1 ? y - n1 : y;
        const float2* row = grid + static_cast<int64_t>(y) * n0;
        float rr = 0.0f, ri = 0.0f;
#pragma unroll
        for (int i = 0; i < W; ++i) {
          const float2 v = __ldg(&row[x[i]]);
          rr = fmaf(v.x, w[0][i], rr);
          ri = fmaf(v.y, w[0][i], ri);
        }
        re = fmaf(rr, w[1][j], re);
        im = fmaf(ri, w[1][j], im);
      }
    } else {
      const int32_t n1 = g.axis[1].length;
      const int32_t n2 = g.axis[2].length;
#pragma unroll 1
      for (int k = 0; k < W; ++k) {
        int z = first[2] + k;
        z = z >= n2 ? z - n2 : z;
        float pr = 0.0f, pi = 0.0f;
#pragma unroll
        for (int j = 0; j < W; ++j) {
          int y = first[1] + j;
          y = y >= n1 ? y - n1 : y;
          const float2* row = grid + (static_cast<int64_t>(z) * n1 + y) * n0;
          float rr = 0.0f, ri = 0.0f;
#pragma unroll
          for (int i = 0; i < W; ++i) {
            const float2 v = __ldg(&row[x[i]]);
            rr = fmaf(v.x, w[0][i], rr);
            ri = fmaf(v.y, w[0][i], ri);
          }
          pr = fmaf(rr, w[1][j], pr);
          pi = fmaf(ri, w[1][j], pi);
        }
        re = fmaf(pr, w[2][k], re);
        im = fmaf(pi, w[2][k], im);
      }
    }
    output[static_cast<int64_t>(b) * count + point] = make_float2(re, im);
  }
}

template <int D, int W>
void launch_width(const GridParams& g, const InterpLaunch& l, cudaStream_t stream) {
  const unsigned blocks = static_cast<unsigned>((l.point_count + 255) / 256);
  interpolate_kernel<D, W><<<blocks, 256, 0, stream>>>(g, l.points, l.point_count, l.perm, l.fine,
                                                        l.batch, l.output);
  note_launch();
}

template <int D>
void launch_dim(const GridParams& g, const InterpLaunch& l, cudaStream_t stream) {
  switch (g.width) {
    case 2: launch_width<D, 2>(g, l, stream); break;
    case 3: launch_width<D, 3>(g, l, stream); break;
    case 4: launch_width<D, 4>(g, l, stream); break;
    case 5: launch_width<D, 5>(g, l, stream); break;
    case 6: launch_width<D, 6>(g, l, stream); break;
    case 7: launch_width<D, 7>(g, l, stream); break;
    case 8: launch_width<D, 8>(g, l, stream); break;
    case 9: launch_width<D, 9>(g, l, stream); break;
    case 10: launch_width<D, 10>(g, l, stream); break;
    case 11: launch_width<D, 11>(g, l, stream); break;
    case 12: launch_width<D, 12>(g, l, stream); break;
    case 13: launch_width<D, 13>(g, l, stream); break;
    case 14: launch_width<D, 14>(g, l, stream); break;
    case 15: launch_width<D, 15>(g, l, stream); break;
    default: launch_width<D, 16>(g, l, stream); break;
  }
}

}  // namespace

void interpolate_execute(const GridParams& g, const InterpLaunch& l, cudaStream_t stream) {
  if (l.point_count == 0) return;
  switch (g.dimensions) {
    case 1: launch_dim<1>(g, l, stream); break;
    case 2: launch_dim<2>(g, l, stream); break;
    default: launch_dim<3>(g, l, stream); break;
  }
}

}  // namespace b200nufft
