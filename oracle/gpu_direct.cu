// FP64 direct NUFFT sums on the GPU (oracle; test infrastructure only).
//
// The CPU direct sums of oracle.cpp restate the reference's FP64 oracle
// (src/direct.rs:9-118, src/type3.rs:609-673) but cost seconds per 10^9
// terms; the subsets that check the full-size workloads (>= 1,000 modes of a
// 10^7-point type-1 transform, >= 10,000 points of a 1024^2-mode type-2
// transform) need 10^10 to 10^11 terms. This file evaluates the same sums
// on the GPU, every term in FP64 with its own sincos:
//
//   out[b, t] = sum_j values[b, j] * exp(i * isign * <target_t, term_j>)
//
// Type 1: targets are the integer mode vectors, terms the points. Type 2:
// targets are points, terms the mode grid (generated from the flat index in
// the reference's storage order, src/direct.rs:120-131). Type 3: targets are
// the target frequencies, terms the sources. Each thread owns one target
// and sums a contiguous range of terms in FP64; the ranges of a target are
// summed by the caller in a fixed order. Only tests/ and bench.py's accuracy
// checks call it, and it is validated against oracle.cpp's CPU sums.
#include <cuda_runtime.h>

#include <cstdint>

namespace {

constexpr int kThreads = 256;
constexpr int kTile = 256;

struct ModeGrid {
  int64_t n[3];
  int centered;
};

__device__ __forceinline__ double mode_of(int64_t index, int64_t length, int centered) {
  // src/direct.rs:120-131: centered order k = index - N/2; FFT order
  // k = index for index < (N + 1) / 2, else index - N.
  if (centered) return static_cast<double>(index - length / 2);
  return static_cast<double>(index < (length + 1) / 2 ? index : index - length);
}

template <int D, int B>
__global__ void __launch_bounds__(kThreads) direct_kernel(const double* __restrict__ targets, int64_t target_count,
                                                          const double* __restrict__ terms, ModeGrid grid,
                                                          int64_t term_count, int64_t term_chunk,
                                                          const double2* __restrict__ values, double sign,
                                                          double2* __restrict__ partial) {
  __shared__ double s_u[kTile][D];
  __shared__ double2 s_v[B][kTile];
  const int64_t t = static_cast<int64_t>(blockIdx.x) * kThreads + threadIdx.x;
  double x[D];
#pragma unroll
  for (int a = 0; a < D; ++a) x[a] = t < target_count ? sign * targets[t * D + a] : 0.0;
  double2 acc[B];
#pragma unroll
  for (int b = 0; b < B; ++b) acc[b] = make_double2(0.0, 0.0);
  const int64_t j_begin = static_cast<int64_t>(blockIdx.y) * term_chunk;
  const int64_t j_end = min(term_count, j_begin + term_chunk);
  for (int64_t base = j_begin; base < j_end; base += kTile) {
    const int n = static_cast<int>(min(static_cast<int64_t>(kTile), j_end - base));
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += kThreads) {
      const int64_t j = base + i;
      if (terms != nullptr) {
#pragma unroll
        for (int a = 0; a < D; ++a) s_u[i][a] = terms[j * D + a];
      } else {
        int64_t rest = j;
#pragma unroll
        for (int a = 0; a < D; ++a) {
          const int64_t index = rest % grid.n[a];
          rest /= grid.n[a];
          s_u[i][a] = mode_of(index, grid.n[a], grid.centered);
        }
      }
#pragma unroll
      for (int b = 0; b < B; ++b) s_v[b][i] = values[static_cast<int64_t>(b) * term_count + j];
    }
    __syncthreads();
    for (int i = 0; i < n; ++i) {
      double phase = 0.0;
#pragma unroll
      for (int a = 0; a < D; ++a) phase = fma(x[a], s_u[i][a], phase);
      double s, c;
      sincos(phase, &s, &c);
#pragma unroll
      for (int b = 0; b < B; ++b) {
        const double2 v = s_v[b][i];
        acc[b].x = fma(v.x, c, fma(-v.y, s, acc[b].x));
        acc[b].y = fma(v.x, s, fma(v.y, c, acc[b].y));
      }
    }
  }
  if (t < target_count) {
#pragma unroll
    for (int b = 0; b < B; ++b) {
      partial[(static_cast<int64_t>(blockIdx.y) * B + b) * target_count + t] = acc[b];
    }
  }
}

template <int D, int B>
int launch(const double* targets, int64_t target_count, const double* terms, const ModeGrid& grid,
           int64_t term_count, int splits, const double2* values, double sign, double2* partial,
           cudaStream_t stream) {
  const int64_t chunk = (term_count + splits - 1) / splits;
  const dim3 blocks(static_cast<unsigned>((target_count + kThreads - 1) / kThreads), static_cast<unsigned>(splits));
  direct_kernel<D, B><<<blocks, kThreads, 0, stream>>>(targets, target_count, terms, grid, term_count,
                                                       chunk > 0 ? chunk : 1, values, sign, partial);
  return cudaGetLastError() == cudaSuccess ? 0 : 3;
}

template <int D>
int launch_batch(int batch, const double* targets, int64_t target_count, const double* terms, const ModeGrid& grid,
                 int64_t term_count, int splits, const double2* values, double sign, double2* partial,
                 cudaStream_t stream) {
  switch (batch) {
    case 1: return launch<D, 1>(targets, target_count, terms, grid, term_count, splits, values, sign, partial, stream);
    case 2: return launch<D, 2>(targets, target_count, terms, grid, term_count, splits, values, sign, partial, stream);
    case 4: return launch<D, 4>(targets, target_count, terms, grid, term_count, splits, values, sign, partial, stream);
    default: return 2;
  }
}

}  // namespace

// Partial FP64 direct sums: partial[s][b][t] over the s-th of `splits`
// contiguous term ranges. `terms` null selects the mode grid of `modes`
// (storage order `order`: 0 centered, 1 FFT) as the terms. All arrays are
// device arrays; values and partial hold interleaved complex doubles.
// Returns 0, 2 for an unsupported dimension or batch, 3 for a launch error.
extern "C" int oracle_gpu_direct(int dimensions, int batch, int isign, int64_t target_count,
                                 const double* targets, int64_t term_count, const double* terms,
                                 const int64_t* modes, int order, const double* values, int splits,
                                 double* partial, void* stream) {
  if (target_count <= 0 || term_count <= 0 || splits <= 0) return 2;
  ModeGrid grid{{1, 1, 1}, order == 0 ? 1 : 0};
  if (terms == nullptr) {
    for (int a = 0; a < dimensions && a < 3; ++a) grid.n[a] = modes[a];
  }
  const double sign = isign >= 0 ? 1.0 : -1.0;
  const auto* v = reinterpret_cast<const double2*>(values);
  auto* p = reinterpret_cast<double2*>(partial);
  auto s = static_cast<cudaStream_t>(stream);
  switch (dimensions) {
    case 1: return launch_batch<1>(batch, targets, target_count, terms, grid, term_count, splits, v, sign, p, s);
    case 2: return launch_batch<2>(batch, targets, target_count, terms, grid, term_count, splits, v, sign, p, s);
    case 3: return launch_batch<3>(batch, targets, target_count, terms, grid, term_count, splits, v, sign, p, s);
    default: return 2;
  }
}
