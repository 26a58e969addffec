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

#include <algorithm>

#include "device.h"
#include "interp.h"
#include "spread.h"

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

// v mod n in [0, n): one conditional add or subtract for the offsets the
// region kernels meet (within one period), the remainder otherwise.
__device__ __forceinline__ int wrap_index(int v, int n) {
  if (v < 0) v += n;
  if (v >= n) v -= n;
  if (v < 0 || v >= n) {
    v %= n;
    if (v < 0) v += n;
  }
  return v;
}

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
    // (re, im) sums: each part the fixed-order fused multiply-adds of the
    // scalar form, two at a time (cfma).
    Complex e;
    e.x = e.y = Real(0);
    if (D == 1) {
#pragma unroll
      for (int i = 0; i < W; ++i) e = cfma(__ldg(&grid[x[i]]), w[0][i], e);
    } else if (D == 2) {
      const int32_t n1 = g.axis[1].length;
#pragma unroll
      for (int j = 0; j < W; ++j) {
        int y = first[1] + j;
        y = y >= n1 ? y - n1 : y;
        const Complex* row = grid + static_cast<int64_t>(y) * n0;
        Complex r;
        r.x = r.y = Real(0);
#pragma unroll
        for (int i = 0; i < W; ++i) r = cfma(__ldg(&row[x[i]]), w[0][i], r);
        e = cfma(r, w[1][j], e);
      }
    } else {
      const int32_t n1 = g.axis[1].length;
      const int32_t n2 = g.axis[2].length;
#pragma unroll 1
      for (int k = 0; k < W; ++k) {
        int z = first[2] + k;
        z = z >= n2 ? z - n2 : z;
        Complex pl;
        pl.x = pl.y = Real(0);
#pragma unroll
        for (int j = 0; j < W; ++j) {
          int y = first[1] + j;
          y = y >= n1 ? y - n1 : y;
          const Complex* row = grid + (static_cast<int64_t>(z) * n1 + y) * n0;
          Complex r;
          r.x = r.y = Real(0);
#pragma unroll
          for (int i = 0; i < W; ++i) r = cfma(__ldg(&row[x[i]]), w[0][i], r);
          pl = cfma(r, w[1][j], pl);
        }
        e = cfma(pl, w[2][k], e);
      }
    }
    output[static_cast<int64_t>(b) * count + point] = e;
  }
}

// Batched 2D f32 interpolation: one CTA per (8 x 8-cell bin, 32 vectors).
// The fine-grid region that the bin's windows can reach (8 + w + 3 cells per
// axis; the bins come from f32 approximate cells, so the exact starts may lie
// one cell beyond the bin) is staged in shared memory with the 32 vectors of a
// cell contiguous, and a warp serves one point at a time with one vector per
// lane, summing in the order of interpolate_kernel (bitwise the same values).
constexpr int kBinVectors = 32;
constexpr int kBinPitch = kBinVectors + 1;  // float2 per staged cell, padded against bank conflicts

template <int W>
__host__ __device__ constexpr int bin_region_side() { return 8 + W + 3; }

// The bin and the slots [first, last) of part blockIdx.x; false for a CTA
// beyond the last part. Each point's sum is the same whichever part (and
// CTA) serves it.
__device__ __forceinline__ bool bin_part(const InterpParts& parts, const uint32_t* __restrict__ offsets,
                                         uint64_t bins, int64_t& bin, uint32_t& first, uint32_t& last) {
  const uint32_t part = blockIdx.x;
  if (part >= parts.part_start[bins]) return false;
  const uint32_t b = parts.part_bin[part];
  const uint32_t begin = offsets[b], end = offsets[b + 1];
  first = begin + (part - parts.part_start[b]) * kInterpPartSlots;
  last = min(first + kInterpPartSlots, end);
  bin = b;
  return first < last;
}

__global__ void interp_part_count_kernel(const uint32_t* __restrict__ offsets, uint64_t bins,
                                         uint32_t* __restrict__ parts) {
  const uint64_t b = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= bins) return;
  parts[b] = (offsets[b + 1] - offsets[b] + kInterpPartSlots - 1) / kInterpPartSlots;
}

__global__ void interp_part_fill_kernel(const uint32_t* __restrict__ part_start, uint64_t bins,
                                        uint32_t* __restrict__ part_bin) {
  const uint64_t b = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= bins) return;
  for (uint32_t p = part_start[b]; p < part_start[b + 1]; ++p) part_bin[p] = static_cast<uint32_t>(b);
}

template <int W>
__global__ void __launch_bounds__(256) interpolate_bins_kernel(GridParams g, const void* __restrict__ windows,
                                                               int64_t count, const uint32_t* __restrict__ perm,
                                                               const uint32_t* __restrict__ offsets,
                                                               const float2* __restrict__ fine, int batch,
                                                               float2* __restrict__ staged, int64_t staged_stride,
                                                               InterpParts parts) {
  constexpr int S = bin_region_side<W>();
  extern __shared__ float2 region[];  // S * S cells x kBinPitch
  int64_t bin;
  uint32_t first, last;
  if (!bin_part(parts, offsets, g.axis[0].bins * static_cast<uint64_t>(g.axis[1].bins), bin, first, last)) return;
  const int vb = blockIdx.y * kBinVectors;
  const int nv = min(kBinVectors, batch - vb);
  const int bins0 = static_cast<int>(g.axis[0].bins);
  const int n0 = g.axis[0].length, n1 = g.axis[1].length;
  const int ox = static_cast<int>(bin % bins0) * 8 - W / 2 - 2;
  const int oy = static_cast<int>(bin / bins0) * 8 - W / 2 - 2;
  // Eight independent loads in flight per thread before their stores.
  constexpr int kLoads = 8;
  constexpr int kTotal = S * S * kBinVectors;
  for (int base = threadIdx.x; base < kTotal; base += kLoads * 256) {
    float2 value[kLoads];
#pragma unroll
    for (int q = 0; q < kLoads; ++q) {
      const int e = base + q * 256;
      value[q] = make_float2(0.0f, 0.0f);
      const int v = e / (S * S), cell = e - v * (S * S);
      if (e < kTotal && v < nv) {
        const int r = cell / S, c = cell - r * S;
        const int y = wrap_index(oy + r, n1);
        const int x = wrap_index(ox + c, n0);
        value[q] = __ldg(&fine[static_cast<int64_t>(vb + v) * g.fine_count + static_cast<int64_t>(y) * n0 + x]);
      }
    }
#pragma unroll
    for (int q = 0; q < kLoads; ++q) {
      const int e = base + q * 256;
      if (e < kTotal) {
        const int v = e / (S * S), cell = e - v * (S * S);
        region[cell * kBinPitch + v] = value[q];
      }
    }
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const float2* grid = fine + static_cast<int64_t>(vb + min(lane, nv - 1)) * g.fine_count;
  // The bin's windows and point indices, 256 at a time, staged by one load per thread.
  __shared__ PreparedWindow<2> s_win[256];
  __shared__ uint32_t s_point[256];
  for (uint32_t batch_first = first; batch_first < last; batch_first += 256) {
  const uint32_t batch_last = min(last, batch_first + 256);
  __syncthreads();
  if (batch_first + threadIdx.x < batch_last) {
    s_win[threadIdx.x] = static_cast<const PreparedWindow<2>*>(windows)[batch_first + threadIdx.x];
    s_point[threadIdx.x] = perm[batch_first + threadIdx.x];
  }
  __syncthreads();
  for (uint32_t slot = batch_first + warp; slot < batch_last; slot += blockDim.x >> 5) {
    const PreparedWindow<2> win = s_win[slot - batch_first];
    const uint32_t point = s_point[slot - batch_first];
    float2 e = make_float2(0.0f, 0.0f);  // (re, im), paired fused multiply-adds
    if (win.start[0] >= 0) {
      float wx[W], wy[W];
      horner32_window<W>(win.offset[0], g.horner32, wx);
      horner32_window<W>(win.offset[1], g.horner32, wy);
      const int dx = wrap_index(win.start[0] - ox, n0);
      const int dy = wrap_index(win.start[1] - oy, n1);
      if (dx + W <= S && dy + W <= S) {
#pragma unroll
        for (int j = 0; j < W; ++j) {
          const float2* row = region + ((dy + j) * S + dx) * kBinPitch + lane;
          float2 r = make_float2(0.0f, 0.0f);
#pragma unroll
          for (int i = 0; i < W; ++i) {
            const float2 v = row[i * kBinPitch];
            r = cfma(v, wx[i], r);
          }
          e = cfma(r, wy[j], e);
        }
      } else {
        // A window beyond the staged region: read the grid directly.
#pragma unroll 1
        for (int j = 0; j < W; ++j) {
          int y = win.start[1] + j;
          y = y >= n1 ? y - n1 : y;
          float2 r = make_float2(0.0f, 0.0f);
          for (int i = 0; i < W; ++i) {
            int x = win.start[0] + i;
            x = x >= n0 ? x - n0 : x;
            const float2 v = __ldg(&grid[static_cast<int64_t>(y) * n0 + x]);
            r = cfma(v, wx[i], r);
          }
          e = cfma(r, wy[j], e);
        }
      }
    }
    if (lane < nv) staged[static_cast<int64_t>(slot) * staged_stride + vb + lane] = e;
    (void)point;
  }
  }
}

// 2D f32 interpolation of fewer than kBinVectors/4 vectors: one CTA of
// kRegionThreads per 8 x 8-cell bin. The region the bin's windows reach is
// staged in shared memory one vector at a time (coalesced row loads, mostly
// L2 hits shared with the neighbouring bins), and a thread serves one point
// from it, summing in the order of interpolate_kernel (bitwise the same
// values); windows beyond the region read the grid directly. For several
// vectors the part's points are served in the order of their support
// starts, so that a warp's lanes share neighbouring region cells.
constexpr int kRegionThreads = 128;

// One vector: the points in bin order (sorting them pays only when the
// staged region serves several vectors).
template <int W>
__global__ void __launch_bounds__(kRegionThreads) interpolate_region_single_kernel(
    GridParams g, const void* __restrict__ windows, int64_t count, const uint32_t* __restrict__ perm,
    const uint32_t* __restrict__ offsets, const float2* __restrict__ fine, int batch,
    float2* __restrict__ output, InterpParts parts) {
  constexpr int S = bin_region_side<W>();
  __shared__ float2 region[S * S];
  int64_t bin;
  uint32_t first, last;
  if (!bin_part(parts, offsets, g.axis[0].bins * static_cast<uint64_t>(g.axis[1].bins), bin, first, last)) return;
  const int bins0 = static_cast<int>(g.axis[0].bins);
  const int n0 = g.axis[0].length, n1 = g.axis[1].length;
  const int ox = static_cast<int>(bin % bins0) * 8 - W / 2 - 2;
  const int oy = static_cast<int>(bin / bins0) * 8 - W / 2 - 2;
  // The first point's window and index are loaded before the region, so
  // their latency overlaps the staging.
  PreparedWindow<2> next_win{};
  uint32_t next_point = 0;
  if (first + threadIdx.x < last) {
    next_win = static_cast<const PreparedWindow<2>*>(windows)[first + threadIdx.x];
    next_point = perm[first + threadIdx.x];
  }
  for (int b = 0; b < batch; ++b) {
    const float2* grid = fine + static_cast<int64_t>(b) * g.fine_count;
    __syncthreads();  // the previous vector's reads are done
    for (int e = threadIdx.x; e < S * S; e += kRegionThreads) {
      const int r = e / S, c = e - r * S;
      const int y = wrap_index(oy + r, n1);
      const int x = wrap_index(ox + c, n0);
      region[e] = __ldg(&grid[static_cast<int64_t>(y) * n0 + x]);
    }
    __syncthreads();
    for (uint32_t slot = first + threadIdx.x; slot < last; slot += kRegionThreads) {
      const PreparedWindow<2> win = slot == first + threadIdx.x
                                        ? next_win
                                        : static_cast<const PreparedWindow<2>*>(windows)[slot];
      const uint32_t point = slot == first + threadIdx.x ? next_point : perm[slot];
      float2 e = make_float2(0.0f, 0.0f);  // (re, im), paired fused multiply-adds
      if (win.start[0] >= 0) {
        float wx[W], wy[W];
        horner32_window<W>(win.offset[0], g.horner32, wx);
        horner32_window<W>(win.offset[1], g.horner32, wy);
        const int dx = wrap_index(win.start[0] - ox, n0);
        const int dy = wrap_index(win.start[1] - oy, n1);
        if (dx + W <= S && dy + W <= S) {
#pragma unroll
          for (int j = 0; j < W; ++j) {
            const float2* row = region + (dy + j) * S + dx;
            float2 r = make_float2(0.0f, 0.0f);
#pragma unroll
            for (int i = 0; i < W; ++i) {
              const float2 v = row[i];
              r = cfma(v, wx[i], r);
            }
            e = cfma(r, wy[j], e);
          }
        } else {
#pragma unroll 1
          for (int j = 0; j < W; ++j) {
            int y = win.start[1] + j;
            y = y >= n1 ? y - n1 : y;
            float2 r = make_float2(0.0f, 0.0f);
            for (int i = 0; i < W; ++i) {
              int x = win.start[0] + i;
              x = x >= n0 ? x - n0 : x;
              const float2 v = __ldg(&grid[static_cast<int64_t>(y) * n0 + x]);
              r = cfma(v, wx[i], r);
            }
            e = cfma(r, wy[j], e);
          }
        }
      }
      output[static_cast<int64_t>(b) * count + point] = e;
    }
  }
}

// Several vectors: the part's points ordered by support start first.
template <int W>
__global__ void __launch_bounds__(kRegionThreads) interpolate_region_kernel(
    GridParams g, const void* __restrict__ windows, int64_t count, const uint32_t* __restrict__ perm,
    const uint32_t* __restrict__ offsets, const float2* __restrict__ fine, int batch,
    float2* __restrict__ output, InterpParts parts) {
  constexpr int S = bin_region_side<W>();
  constexpr int kKeys = S * S + 1;  // start cells of the region, then the windows that leave it
  __shared__ float2 region[S * S];
  __shared__ PreparedWindow<2> part_win[kInterpPartSlots];
  __shared__ uint32_t part_point[kInterpPartSlots];
  __shared__ uint16_t order[kInterpPartSlots];
  __shared__ uint32_t key_start[kKeys];
  __shared__ uint32_t warp_total[kRegionThreads / 32];
  int64_t bin;
  uint32_t first, last;
  if (!bin_part(parts, offsets, g.axis[0].bins * static_cast<uint64_t>(g.axis[1].bins), bin, first, last)) return;
  const int bins0 = static_cast<int>(g.axis[0].bins);
  const int n0 = g.axis[0].length, n1 = g.axis[1].length;
  const int ox = static_cast<int>(bin % bins0) * 8 - W / 2 - 2;
  const int oy = static_cast<int>(bin / bins0) * 8 - W / 2 - 2;
  const int n = static_cast<int>(last - first);
  // The part's points ordered by support start (a counting sort in shared
  // memory; the order within a start is arbitrary, and each point's sum does
  // not depend on it), so that a warp's lanes read neighbouring region cells
  // and share them instead of colliding in the banks.
  for (int k = threadIdx.x; k < kKeys; k += kRegionThreads) key_start[k] = 0;
  __syncthreads();
  constexpr int kPerThread = kInterpPartSlots / kRegionThreads;
  int key[kPerThread];
  uint32_t rank[kPerThread];
#pragma unroll
  for (int q = 0; q < kPerThread; ++q) {
    const int i = threadIdx.x + q * kRegionThreads;
    key[q] = -1;
    rank[q] = 0;
    if (i < n) {
      const PreparedWindow<2> win = static_cast<const PreparedWindow<2>*>(windows)[first + i];
      part_win[i] = win;
      part_point[i] = perm[first + i];
      int k = S * S;
      if (win.start[0] >= 0) {
        const int dx = wrap_index(win.start[0] - ox, n0);
        const int dy = wrap_index(win.start[1] - oy, n1);
        if (dx + W <= S && dy + W <= S) k = dy * S + dx;
      }
      key[q] = k;
      rank[q] = atomicAdd(&key_start[k], 1u);
    }
  }
  __syncthreads();
  {
    // Exclusive scan of the key counts: a thread sums a few consecutive
    // keys, the warps and then the block add up.
    constexpr int kKeysPerThread = (kKeys + kRegionThreads - 1) / kRegionThreads;
    uint32_t local[kKeysPerThread];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kKeysPerThread; ++k) {
      const int e = threadIdx.x * kKeysPerThread + k;
      local[k] = e < kKeys ? key_start[e] : 0u;
      sum += local[k];
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = sum;
#pragma unroll
    for (int offset = 1; offset < 32; offset <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, offset);
      if (lane >= offset) x += y;
    }
    if (lane == 31) warp_total[warp] = x;
    __syncthreads();
    uint32_t running = x - sum;
    for (int w = 0; w < warp; ++w) running += warp_total[w];
#pragma unroll
    for (int k = 0; k < kKeysPerThread; ++k) {
      const int e = threadIdx.x * kKeysPerThread + k;
      if (e < kKeys) key_start[e] = running;
      running += local[k];
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < kPerThread; ++q) {
    if (key[q] >= 0) order[key_start[key[q]] + rank[q]] = static_cast<uint16_t>(threadIdx.x + q * kRegionThreads);
  }
  for (int b = 0; b < batch; ++b) {
    const float2* grid = fine + static_cast<int64_t>(b) * g.fine_count;
    __syncthreads();  // the order is written; the previous vector's reads are done
    for (int e = threadIdx.x; e < S * S; e += kRegionThreads) {
      const int r = e / S, c = e - r * S;
      const int y = wrap_index(oy + r, n1);
      const int x = wrap_index(ox + c, n0);
      region[e] = __ldg(&grid[static_cast<int64_t>(y) * n0 + x]);
    }
    __syncthreads();
    for (int pos = threadIdx.x; pos < n; pos += kRegionThreads) {
      const int i = order[pos];
      const PreparedWindow<2> win = part_win[i];
      const uint32_t point = part_point[i];
      float2 e = make_float2(0.0f, 0.0f);  // (re, im), paired fused multiply-adds
      if (win.start[0] >= 0) {
        float wx[W], wy[W];
        horner32_window<W>(win.offset[0], g.horner32, wx);
        horner32_window<W>(win.offset[1], g.horner32, wy);
        const int dx = wrap_index(win.start[0] - ox, n0);
        const int dy = wrap_index(win.start[1] - oy, n1);
        if (dx + W <= S && dy + W <= S) {
#pragma unroll
          for (int j = 0; j < W; ++j) {
            const float2* row = region + (dy + j) * S + dx;
            float2 r = make_float2(0.0f, 0.0f);
#pragma unroll
            for (int k = 0; k < W; ++k) {
              const float2 v = row[k];
              r = cfma(v, wx[k], r);
            }
            e = cfma(r, wy[j], e);
          }
        } else {
#pragma unroll 1
          for (int j = 0; j < W; ++j) {
            int y = win.start[1] + j;
            y = y >= n1 ? y - n1 : y;
            float2 r = make_float2(0.0f, 0.0f);
            for (int k = 0; k < W; ++k) {
              int x = win.start[0] + k;
              x = x >= n0 ? x - n0 : x;
              const float2 v = __ldg(&grid[static_cast<int64_t>(y) * n0 + x]);
              r = cfma(v, wx[k], r);
            }
            e = cfma(r, wy[j], e);
          }
        }
      }
      output[static_cast<int64_t>(b) * count + point] = e;
    }
  }
}

// 2D f64 interpolation over the type-2 bins of 4 x 4 cells, which f64 plans
// key by the exact support start: one CTA of kRegionThreads per bin stages
// the (4 + w - 1)^2 cells the bin's windows cover in shared memory, one
// vector at a time, and a thread serves one point from it, summing in the
// order of interpolate_kernel (bitwise the same values). A window that the
// region does not hold (not expected with start keys) reads the grid.
template <int W>
__global__ void __launch_bounds__(kRegionThreads) interpolate_region64_kernel(
    GridParams g, const double* __restrict__ points, int64_t count, const uint32_t* __restrict__ perm,
    const uint32_t* __restrict__ offsets, const double2* __restrict__ fine, int batch,
    double2* __restrict__ output, InterpParts parts) {
  constexpr int S = 4 + W - 1;
  __shared__ double2 region[S * S];
  int64_t bin;
  uint32_t first, last;
  if (!bin_part(parts, offsets, g.axis[0].bins * static_cast<uint64_t>(g.axis[1].bins), bin, first, last)) return;
  const int bins0 = static_cast<int>(g.axis[0].bins);
  const int n0 = g.axis[0].length, n1 = g.axis[1].length;
  const int ox = static_cast<int>(bin % bins0) * 4;
  const int oy = static_cast<int>(bin / bins0) * 4;
  for (int b = 0; b < batch; ++b) {
    const double2* grid = fine + static_cast<int64_t>(b) * g.fine_count;
    __syncthreads();  // the previous vector's reads are done
    for (int e = threadIdx.x; e < S * S; e += kRegionThreads) {
      const int r = e / S, c = e - r * S;
      const int y = wrap_index(oy + r, n1), x = wrap_index(ox + c, n0);
      region[e] = __ldg(&grid[static_cast<int64_t>(y) * n0 + x]);
    }
    __syncthreads();
    for (uint32_t slot = first + threadIdx.x; slot < last; slot += kRegionThreads) {
      const uint32_t point = perm[slot];
      const double px = points[static_cast<int64_t>(slot) * 2], py = points[static_cast<int64_t>(slot) * 2 + 1];
      double re = 0.0, im = 0.0;
      if (F64Window::in_reach(px) && F64Window::in_reach(py)) {
        int first_x, first_y;
        double wx[W], wy[W];
        F64Window::window<W>(px, g, 0, first_x, wx);
        F64Window::window<W>(py, g, 1, first_y, wy);
        const int dx = wrap_index(first_x - ox, n0);
        const int dy = wrap_index(first_y - oy, n1);
        if (dx + W <= S && dy + W <= S) {
#pragma unroll
          for (int j = 0; j < W; ++j) {
            const double2* row = region + (dy + j) * S + dx;
            double rr = 0.0, ri = 0.0;
#pragma unroll
            for (int i = 0; i < W; ++i) {
              const double2 v = row[i];
              rr = fma(v.x, wx[i], rr);
              ri = fma(v.y, wx[i], ri);
            }
            re = fma(rr, wy[j], re);
            im = fma(ri, wy[j], im);
          }
        } else {
#pragma unroll 1
          for (int j = 0; j < W; ++j) {
            int y = first_y + j;
            y = y >= n1 ? y - n1 : y;
            double rr = 0.0, ri = 0.0;
            for (int i = 0; i < W; ++i) {
              int x = first_x + i;
              x = x >= n0 ? x - n0 : x;
              const double2 v = __ldg(&grid[static_cast<int64_t>(y) * n0 + x]);
              rr = fma(v.x, wx[i], rr);
              ri = fma(v.y, wx[i], ri);
            }
            re = fma(rr, wy[j], re);
            im = fma(ri, wy[j], im);
          }
        }
      }
      output[static_cast<int64_t>(b) * count + point] = make_double2(re, im);
    }
  }
}

// output[b][i] = staged[slot of i][b]: 32 points x 64 vectors per CTA through
// shared memory, so both the staged rows and the output rows move in whole
// sectors.
__global__ void __launch_bounds__(256) unpermute_kernel(const float2* __restrict__ staged, int64_t staged_stride,
                                                        const uint32_t* __restrict__ inverse, int64_t count,
                                                        int batch, float2* __restrict__ output) {
  __shared__ float2 tile[32][65];
  __shared__ uint32_t rows[32];
  const int64_t i0 = static_cast<int64_t>(blockIdx.x) * 32;
  const int b0 = blockIdx.y * 64;
  if (threadIdx.x < 32) rows[threadIdx.x] = i0 + threadIdx.x < count ? inverse[i0 + threadIdx.x] : 0u;
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int e = threadIdx.x + q * 256;
    const int k = e >> 6, v = e & 63;
    if (i0 + k < count && b0 + v < batch) tile[k][v] = staged[static_cast<int64_t>(rows[k]) * staged_stride + b0 + v];
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int e = threadIdx.x + q * 256;
    const int v = e >> 5, k = e & 31;
    if (i0 + k < count && b0 + v < batch) output[static_cast<int64_t>(b0 + v) * count + i0 + k] = tile[k][v];
  }
}

template <int W>
void launch_bins_width(const GridParams& g, const InterpBinsLaunch& l, cudaStream_t stream) {
  constexpr int S = bin_region_side<W>();
  const size_t smem = static_cast<size_t>(S) * S * kBinPitch * sizeof(float2);
  auto kernel = interpolate_bins_kernel<W>;
  check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
             "interpolation region shared memory");
  const dim3 grid(static_cast<unsigned>(l.parts.upper_bound),
                  static_cast<unsigned>((l.batch + kBinVectors - 1) / kBinVectors));
  const int64_t stride = (l.batch + kBinVectors - 1) / kBinVectors * kBinVectors;
  kernel<<<grid, 256, smem, stream>>>(g, l.windows, l.point_count, l.perm, l.offsets, l.fine, l.batch, l.staged,
                                      stride, l.parts);
  const dim3 grid2(static_cast<unsigned>((l.point_count + 31) / 32), static_cast<unsigned>((l.batch + 63) / 64));
  unpermute_kernel<<<grid2, 256, 0, stream>>>(l.staged, stride, l.inverse, l.point_count, l.batch, l.output);
  note_launch(2);
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

void interpolate_region_execute(const GridParams& g, const InterpBinsLaunch& l, cudaStream_t stream) {
  if (l.point_count == 0) return;
  const dim3 grid(static_cast<unsigned>(l.parts.upper_bound));
  switch (g.width) {
#define B200NUFFT_REGION_CASE(WIDTH)                                                                   \
  case WIDTH:                                                                                          \
    if (l.batch > 1) {                                                                                 \
      interpolate_region_kernel<WIDTH><<<grid, kRegionThreads, 0, stream>>>(                            \
          g, l.windows, l.point_count, l.perm, l.offsets, l.fine, l.batch, l.output, l.parts);          \
    } else {                                                                                           \
      interpolate_region_single_kernel<WIDTH><<<grid, kRegionThreads, 0, stream>>>(                     \
          g, l.windows, l.point_count, l.perm, l.offsets, l.fine, l.batch, l.output, l.parts);          \
    }                                                                                                  \
    break;
    B200NUFFT_REGION_CASE(2)
    B200NUFFT_REGION_CASE(3)
    B200NUFFT_REGION_CASE(4)
    B200NUFFT_REGION_CASE(5)
    B200NUFFT_REGION_CASE(6)
    B200NUFFT_REGION_CASE(7)
    default:
    B200NUFFT_REGION_CASE(8)
#undef B200NUFFT_REGION_CASE
  }
  note_launch();
}

bool interpolate_bins_supported(const GridParams& g) {
  return g.dimensions == 2 && g.width <= 8 && g.axis[0].shift == 3 && g.axis[1].shift == 3;
}

void unpermute_values(const float2* staged, int64_t stride, const uint32_t* inverse, int64_t count, int batch,
                      float2* output, cudaStream_t stream) {
  if (count <= 0) return;
  const dim3 grid(static_cast<unsigned>((count + 31) / 32), static_cast<unsigned>((batch + 63) / 64));
  unpermute_kernel<<<grid, 256, 0, stream>>>(staged, stride, inverse, count, batch, output);
  note_launch();
}

void interpolate_bins_execute(const GridParams& g, const InterpBinsLaunch& l, cudaStream_t stream) {
  if (l.point_count == 0) return;
  switch (g.width) {
    case 2: launch_bins_width<2>(g, l, stream); break;
    case 3: launch_bins_width<3>(g, l, stream); break;
    case 4: launch_bins_width<4>(g, l, stream); break;
    case 5: launch_bins_width<5>(g, l, stream); break;
    case 6: launch_bins_width<6>(g, l, stream); break;
    case 7: launch_bins_width<7>(g, l, stream); break;
    default: launch_bins_width<8>(g, l, stream); break;
  }
}

bool interpolate_region64_supported(const GridParams& g) {
  return g.dimensions == 2 && g.width >= 2 && g.width <= 16 && g.axis[0].shift == 2 && g.axis[1].shift == 2;
}

void interpolate_region64_execute(const GridParams& g, const InterpLaunch64& l, const uint32_t* offsets,
                                  uint64_t bins, const InterpParts& parts, cudaStream_t stream) {
  if (l.point_count == 0) return;
  (void)bins;
  const dim3 grid(static_cast<unsigned>(parts.upper_bound));
  switch (g.width) {
#define B200NUFFT_REGION64_CASE(WIDTH)                                                                  \
  case WIDTH:                                                                                          \
    interpolate_region64_kernel<WIDTH><<<grid, kRegionThreads, 0, stream>>>(                            \
        g, l.points, l.point_count, l.perm, offsets, l.fine, l.batch, l.output, parts);                 \
    break;
    B200NUFFT_REGION64_CASE(2)
    B200NUFFT_REGION64_CASE(3)
    B200NUFFT_REGION64_CASE(4)
    B200NUFFT_REGION64_CASE(5)
    B200NUFFT_REGION64_CASE(6)
    B200NUFFT_REGION64_CASE(7)
    B200NUFFT_REGION64_CASE(8)
    B200NUFFT_REGION64_CASE(9)
    B200NUFFT_REGION64_CASE(10)
    B200NUFFT_REGION64_CASE(11)
    B200NUFFT_REGION64_CASE(12)
    B200NUFFT_REGION64_CASE(13)
    B200NUFFT_REGION64_CASE(14)
    B200NUFFT_REGION64_CASE(15)
    default:
    B200NUFFT_REGION64_CASE(16)
#undef B200NUFFT_REGION64_CASE
  }
  note_launch();
}

void interp_bin_parts(const uint32_t* offsets, uint64_t bins, uint32_t* parts, uint32_t* part_start,
                      uint32_t* part_bin, cudaStream_t stream) {
  const unsigned blocks = static_cast<unsigned>((bins + 255) / 256);
  interp_part_count_kernel<<<blocks, 256, 0, stream>>>(offsets, bins, parts);
  exclusive_scan_u32(parts, static_cast<int64_t>(bins), part_start, stream);
  interp_part_fill_kernel<<<blocks, 256, 0, stream>>>(part_start, bins, part_bin);
  note_launch(2);
}

void interpolate_execute64(const GridParams& g, const InterpLaunch64& l, cudaStream_t stream) {
  execute_impl<F64Window>(g, Launch<F64Window>{l.points, nullptr, l.point_count, l.perm, l.fine, l.batch, l.output},
                          stream);
}

}  // namespace b200nufft
