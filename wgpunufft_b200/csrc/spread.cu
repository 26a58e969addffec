// Type-1 spreading: bin subproblems accumulated in shared memory.
//
// The reference spreads with an output-stationary block spreader that sums
// every cell's points in a fixed order, with no floating-point atomics, so
// that outputs are bitwise repeatable (src/gpu_nd_spread.rs:1-35). Here each
// CTA takes one subproblem: the points whose support starts in one tile of the
// fine grid (or one part of a crowded tile), read from the bins of the stable
// sort. Every point evaluates its window per axis into registers and adds
// its w^d contributions to a padded copy of the tile in shared memory. The
// contributions are accumulated as fixed-point integers (each rounded to a
// 32-bit integer after scaling by a power of two derived from the largest
// strength, and summed exactly in two 32-bit halves), so the sum of a cell is
// the exact integer sum of its rounded contributions whatever order the
// threads add them in: the accumulation is deterministic without ordering the
// threads, and it carries more bits than an f32 sum. Each padded tile is then
// converted to f32 and written out, and a fold pass adds, for every fine-grid
// cell, the padded tiles and parts that cover it in a fixed order (halos
// wrap periodically). Nothing is accumulated with floating-point atomics.
#include <cuda_runtime.h>

#include <algorithm>

#include "device.h"
#include "spread.h"

namespace b200nufft {

namespace {

constexpr int kSpreadThreads = 256;

__device__ __forceinline__ float es_weight(float distance, float beta, float width_f) {
  // The F32 window of the reference's spreading shader (src/gpu_nd_wgsl.rs:383-395).
  const float scaled = (2.0f * fabsf(distance)) / width_f;
  const float squared = scaled * scaled;
  if (squared >= 1.0f) return 0.0f;
  return expf(beta * (sqrtf(fmaxf(0.0f, 1.0f - squared)) - 1.0f));
}

// Largest |re| or |im| of every strength vector, as float bits.
__global__ void strength_magnitude_kernel(const float2* __restrict__ values, int64_t count,
                                          int batch, uint32_t* __restrict__ max_bits) {
  const int b = blockIdx.y;
  const float2* v = values + static_cast<int64_t>(b) * count;
  uint32_t m = 0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
       i += stride) {
    const float2 s = v[i];
    m = max(m, __float_as_uint(s.x) & 0x7fffffffu);
    m = max(m, __float_as_uint(s.y) & 0x7fffffffu);
  }
#pragma unroll
  for (int offset = 16; offset > 0; offset >>= 1) m = max(m, __shfl_xor_sync(0xFFFFFFFFu, m, offset));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(&max_bits[b], m);
}

// Power-of-two exponent S that scales every contribution, at most the largest
// strength magnitude, below 2^30 in magnitude: each then rounds to a 32-bit
// integer with a resolution of 2^-30 of the largest strength.
__device__ __forceinline__ int fixed_point_exponent(uint32_t max_bits) {
  if (max_bits == 0u) return 0;
  // Non-finite strengths (bits at or above infinity) leave the outputs
  // unspecified but the exponent bounded.
  const int e = max_bits >= 0x7f800000u ? 128 : ilogbf(__uint_as_float(max_bits)) + 1;  // max < 2^e
  return 30 - e;
}

// Adds a fixed-point contribution v (|v| < 2^31) to cell c as two exact
// 32-bit sums: its low 16 bits, unsigned, and its arithmetic high part. Both
// stay exact for up to 2^16 contributions per cell, and the cell's value is
// hi * 2^16 + lo. Integer addition is associative, so the sums do not depend
// on the order in which threads add.
__device__ __forceinline__ void add_fixed(uint32_t* lo, int32_t* hi, int c, float value) {
  const int32_t v = __float2int_rn(value);
  atomicAdd(&lo[c], static_cast<uint32_t>(v) & 0xFFFFu);
  atomicAdd(&hi[c], v >> 16);
}

__device__ __forceinline__ float fixed_to_float(uint32_t lo, int32_t hi, int S) {
  const long long total = static_cast<long long>(hi) * 65536ll + static_cast<long long>(lo);
  return ldexpf(__ll2float_rn(total), -S);
}

// Records in the reach of every tile's bins, and the parts of every tile.
template <int D>
__global__ void tile_records_kernel(SpreadParams sp, const uint32_t* __restrict__ offsets,
                                    uint32_t* __restrict__ parts) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= sp.tile_count) return;
  int64_t rest = t;
  int lo[3], hi[3];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const int64_t ta = rest % sp.ntiles[a];
    rest /= sp.ntiles[a];
    const int64_t origin = ta * sp.tile[a];
    const int64_t last = min(origin + sp.tile[a], sp.grid.fine[a]) - 1;
    lo[a] = static_cast<int>(origin >> sp.grid.axis[a].shift);
    hi[a] = static_cast<int>(last >> sp.grid.axis[a].shift);
  }
  uint64_t count = 0;
  const uint32_t b0 = sp.grid.axis[0].bins;
  const uint32_t b1 = D > 1 ? sp.grid.axis[1].bins : 1u;
  const int lo1 = D > 1 ? lo[1] : 0, hi1 = D > 1 ? hi[1] : 0;
  const int lo2 = D > 2 ? lo[2] : 0, hi2 = D > 2 ? hi[2] : 0;
  for (int z = lo2; z <= hi2; ++z) {
    for (int y = lo1; y <= hi1; ++y) {
      const uint64_t row = static_cast<uint64_t>(b0) * (y + static_cast<uint64_t>(b1) * z);
      count += offsets[row + hi[0] + 1] - offsets[row + lo[0]];
    }
  }
  parts[t] = static_cast<uint32_t>((count + sp.part_cap - 1) / sp.part_cap);
}

// Exclusive scan of the parts per tile in one block; part_start[tile_count]
// receives the total.
__global__ void __launch_bounds__(1024) part_scan_kernel(const uint32_t* __restrict__ parts,
                                                         int64_t tile_count,
                                                         uint32_t* __restrict__ part_start) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t carry_shared;
  if (threadIdx.x == 0) carry_shared = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int64_t base = 0; base < tile_count; base += 1024) {
    const int64_t i = base + threadIdx.x;
    const uint32_t v = i < tile_count ? parts[i] : 0u;
    uint32_t x = v;
#pragma unroll
    for (int offset = 1; offset < 32; offset <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, offset);
      if (lane >= offset) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t s = warp_sums[lane];
#pragma unroll
      for (int offset = 1; offset < 32; offset <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, offset);
        if (lane >= offset) s += y;
      }
      warp_sums[lane] = s;
    }
    __syncthreads();
    const uint32_t carry = carry_shared;
    const uint32_t inclusive = x + (warp > 0 ? warp_sums[warp - 1] : 0u);
    if (i < tile_count) part_start[i] = carry + inclusive - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry_shared = carry + inclusive;
    __syncthreads();
  }
  if (threadIdx.x == 0) part_start[tile_count] = carry_shared;
}

// One CTA per (part, vector): spreads the part's records into a padded tile
// of 64-bit fixed-point sums and writes the tile out as f32.
template <int D, int W>
__global__ void __launch_bounds__(kSpreadThreads) spread_tiles_kernel(
    SpreadParams sp, const float* __restrict__ points, const float2* __restrict__ strengths,
    int64_t point_count, int batch, const uint32_t* __restrict__ perm,
    const uint32_t* __restrict__ offsets, const uint32_t* __restrict__ part_start,
    const uint32_t* __restrict__ max_bits, float2* __restrict__ scratch) {
  extern __shared__ uint32_t acc[];
  __shared__ uint32_t row_begin[kMaxTileRows];
  __shared__ uint32_t row_prefix[kMaxTileRows + 1];
  __shared__ int64_t s_tile;
  __shared__ uint32_t warp_totals[kSpreadThreads / 32];

  const uint32_t part = blockIdx.x;
  const int b = blockIdx.y;
  const uint32_t total_parts = part_start[sp.tile_count];
  if (part >= total_parts) return;
  const int tid = threadIdx.x;
  if (tid == 0) {
    // Last tile whose first part is at or below `part`.
    int64_t low = 0, high = sp.tile_count - 1;
    while (low < high) {
      const int64_t mid = (low + high + 1) >> 1;
      if (part_start[mid] <= part) low = mid; else high = mid - 1;
    }
    s_tile = low;
  }
  const int padded = sp.padded_cells;
  for (int c = tid; c < 4 * padded; c += kSpreadThreads) acc[c] = 0u;
  __syncthreads();
  const int64_t tile = s_tile;
  const uint32_t part_in_tile = part - part_start[tile];

  // Tile origin and bin rows.
  int origin[3], bin_lo[3], bin_hi[3], rows_along[3];
  {
    int64_t rest = tile;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      const int64_t ta = rest % sp.ntiles[a];
      rest /= sp.ntiles[a];
      origin[a] = static_cast<int>(ta * sp.tile[a]);
      const int64_t last = min(static_cast<int64_t>(origin[a]) + sp.tile[a], sp.grid.fine[a]) - 1;
      bin_lo[a] = origin[a] >> sp.grid.axis[a].shift;
      bin_hi[a] = static_cast<int>(last >> sp.grid.axis[a].shift);
      rows_along[a] = bin_hi[a] - bin_lo[a] + 1;
    }
  }
  const int rows = D == 1 ? 1 : (D == 2 ? rows_along[1] : rows_along[1] * rows_along[2]);
  // Row slot ranges and their exclusive prefix (rows <= kMaxTileRows).
  constexpr int kRowsPerThread = kMaxTileRows / kSpreadThreads;
  uint32_t local[kRowsPerThread];
  uint32_t local_sum = 0;
  const uint32_t bins0 = sp.grid.axis[0].bins;
  const uint32_t bins1 = D > 1 ? sp.grid.axis[1].bins : 1u;
#pragma unroll
  for (int k = 0; k < kRowsPerThread; ++k) {
    const int r = tid * kRowsPerThread + k;
    uint32_t n = 0;
    if (r < rows) {
      int y = 0, z = 0;
      if (D == 2) y = bin_lo[1] + r;
      if (D == 3) {
        y = bin_lo[1] + r % rows_along[1];
        z = bin_lo[2] + r / rows_along[1];
      }
      const uint64_t row = static_cast<uint64_t>(bins0) * (y + static_cast<uint64_t>(bins1) * z);
      const uint32_t begin = offsets[row + bin_lo[0]];
      n = offsets[row + bin_hi[0] + 1] - begin;
      row_begin[r] = begin;
    }
    local[k] = n;
    local_sum += n;
  }
  {
    const int lane = tid & 31, warp = tid >> 5;
    uint32_t x = local_sum;
#pragma unroll
    for (int offset = 1; offset < 32; offset <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, offset);
      if (lane >= offset) x += y;
    }
    if (lane == 31) warp_totals[warp] = x;
    __syncthreads();
    uint32_t warp_offset = 0;
    for (int w = 0; w < warp; ++w) warp_offset += warp_totals[w];
    uint32_t running = warp_offset + x - local_sum;
#pragma unroll
    for (int k = 0; k < kRowsPerThread; ++k) {
      const int r = tid * kRowsPerThread + k;
      if (r <= rows) row_prefix[r] = running;
      running += local[k];
    }
    if (tid == kSpreadThreads - 1) row_prefix[min(rows, kMaxTileRows)] = running;
  }
  __syncthreads();
  const uint32_t tile_total = row_prefix[rows];
  const uint32_t record_begin = part_in_tile * static_cast<uint32_t>(sp.part_cap);
  const uint32_t record_end = min(tile_total, record_begin + static_cast<uint32_t>(sp.part_cap));
  const int S = fixed_point_exponent(max_bits[b]);
  const float width_f = static_cast<float>(W);
  const float2* sv = strengths + static_cast<int64_t>(b) * point_count;
  uint32_t* re_lo = acc;
  int32_t* re_hi = reinterpret_cast<int32_t*>(acc + padded);
  uint32_t* im_lo = acc + 2 * padded;
  int32_t* im_hi = reinterpret_cast<int32_t*>(acc + 3 * padded);

  int row = 0;
  for (uint32_t r = record_begin + tid; r < record_end; r += kSpreadThreads) {
    // Advance to the row holding record r (rows are visited in order).
    if (r >= row_prefix[row + 1] || r < row_prefix[row]) {
      int low = 0, high = rows - 1;
      while (low < high) {
        const int mid = (low + high + 1) >> 1;
        if (row_prefix[mid] <= r) low = mid; else high = mid - 1;
      }
      row = low;
    }
    const uint32_t slot = row_begin[row] + (r - row_prefix[row]);
    float p[D];
#pragma unroll
    for (int a = 0; a < D; ++a) p[a] = points[static_cast<int64_t>(slot) * D + a];
    bool reach = true;
#pragma unroll
    for (int a = 0; a < D; ++a) reach = reach && in_fold_reach(p[a]);
    if (!reach) continue;  // weighed zero by the reference
    int local_start[D];
    float w[D][W];
    bool inside = true;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      int32_t start;
      Df64 off;
      support_of(p[a], sp.grid.axis[a], sp.grid.half_width, start, off);
      const int32_t wrapped = wrap_start(start, sp.grid.axis[a].length);
      local_start[a] = wrapped - origin[a];
      inside = inside && local_start[a] >= 0 && local_start[a] < sp.tile[a];
#pragma unroll
      for (int j = 0; j < W; ++j) {
        const float d = __fadd_rn(__fadd_rn(static_cast<float>(j), off.hi), off.lo);
        w[a][j] = es_weight(d, sp.grid.beta, width_f);
      }
    }
    if (!inside) continue;  // a bin wider than the tile: another tile owns it
    const float2 s = sv[perm[slot]];
    const float sr = ldexpf(s.x, S);
    const float si = ldexpf(s.y, S);
    if (D == 1) {
#pragma unroll
      for (int i = 0; i < W; ++i) {
        const int c = local_start[0] + i;
        add_fixed(re_lo, re_hi, c, sr * w[0][i]);
        add_fixed(im_lo, im_hi, c, si * w[0][i]);
      }
    } else if (D == 2) {
#pragma unroll
      for (int j = 0; j < W; ++j) {
        const float wr = sr * w[1][j];
        const float wi = si * w[1][j];
        const int base = (local_start[1] + j) * sp.pad[0] + local_start[0];
#pragma unroll
        for (int i = 0; i < W; ++i) {
          add_fixed(re_lo, re_hi, base + i, wr * w[0][i]);
          add_fixed(im_lo, im_hi, base + i, wi * w[0][i]);
        }
      }
    } else {
#pragma unroll 1
      for (int k = 0; k < W; ++k) {
#pragma unroll
        for (int j = 0; j < W; ++j) {
          const float wyz = w[1][j] * w[2][k];
          const float wr = sr * wyz;
          const float wi = si * wyz;
          const int base =
              ((local_start[2] + k) * sp.pad[1] + local_start[1] + j) * sp.pad[0] + local_start[0];
#pragma unroll
          for (int i = 0; i < W; ++i) {
            add_fixed(re_lo, re_hi, base + i, wr * w[0][i]);
            add_fixed(im_lo, im_hi, base + i, wi * w[0][i]);
          }
        }
      }
    }
  }
  __syncthreads();
  float2* out = scratch + (static_cast<int64_t>(part) * batch + b) * padded;
  for (int c = tid; c < padded; c += kSpreadThreads) {
    out[c] = make_float2(fixed_to_float(re_lo[c], re_hi[c], S), fixed_to_float(im_lo[c], im_hi[c], S));
  }
}

// Every fine-grid cell as the sum, in a fixed order, of the padded tiles and
// parts that cover it.
template <int D>
__global__ void fold_tiles_kernel(SpreadParams sp, int batch, const float2* __restrict__ scratch,
                                  const uint32_t* __restrict__ part_start, int64_t part_limit,
                                  const int2* __restrict__ candidates,
                                  float2* __restrict__ fine) {
  const int64_t cell = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (cell >= sp.grid.fine_count) return;
  const int b = blockIdx.y;
  int coord[3] = {0, 0, 0};
  {
    int64_t rest = cell;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      coord[a] = static_cast<int>(rest % sp.grid.fine[a]);
      rest /= sp.grid.fine[a];
    }
  }
  const int2* c0 = candidates + sp.candidate_base[0] + coord[0] * sp.candidate_count[0];
  const int2* c1 = D > 1 ? candidates + sp.candidate_base[1] + coord[1] * sp.candidate_count[1] : nullptr;
  const int2* c2 = D > 2 ? candidates + sp.candidate_base[2] + coord[2] * sp.candidate_count[2] : nullptr;
  const int k2n = D > 2 ? sp.candidate_count[2] : 1;
  const int k1n = D > 1 ? sp.candidate_count[1] : 1;
  float re = 0.0f, im = 0.0f;
  for (int k2 = 0; k2 < k2n; ++k2) {
    int t2 = 0, l2 = 0;
    if (D > 2) {
      const int2 e = c2[k2];
      if (e.x < 0) break;
      t2 = e.x;
      l2 = e.y;
    }
    for (int k1 = 0; k1 < k1n; ++k1) {
      int t1 = 0, l1 = 0;
      if (D > 1) {
        const int2 e = c1[k1];
        if (e.x < 0) break;
        t1 = e.x;
        l1 = e.y;
      }
      for (int k0 = 0; k0 < sp.candidate_count[0]; ++k0) {
        const int2 e = c0[k0];
        if (e.x < 0) break;
        const int64_t tile =
            e.x + static_cast<int64_t>(sp.ntiles[0]) * (t1 + static_cast<int64_t>(sp.ntiles[1]) * t2);
        const int local = e.y + sp.pad[0] * (l1 + sp.pad[1] * l2);
        const uint32_t first = part_start[tile];
        const uint32_t last = min(part_start[tile + 1], static_cast<uint32_t>(part_limit));
        for (uint32_t part = first; part < last; ++part) {
          const float2 v = scratch[(static_cast<int64_t>(part) * batch + b) * sp.padded_cells + local];
          re += v.x;
          im += v.y;
        }
      }
    }
  }
  fine[static_cast<int64_t>(b) * sp.grid.fine_count + cell] = make_float2(re, im);
}

template <int D, int W>
void launch_spread_width(const SpreadParams& sp, const SpreadLaunch& l, cudaStream_t stream) {
  const size_t smem = static_cast<size_t>(4) * sp.padded_cells * sizeof(uint32_t);
  auto kernel = spread_tiles_kernel<D, W>;
  check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)),
             "spread shared memory");
  const dim3 grid(static_cast<unsigned>(l.part_upper_bound), static_cast<unsigned>(l.batch));
  kernel<<<grid, kSpreadThreads, smem, stream>>>(sp, l.points, l.strengths, l.point_count, l.batch,
                                                 l.perm, l.offsets, l.part_start, l.max_bits,
                                                 l.scratch);
  note_launch();
}

template <int D>
void launch_spread_dim(const SpreadParams& sp, const SpreadLaunch& l, cudaStream_t stream) {
  switch (sp.grid.width) {
    case 2: launch_spread_width<D, 2>(sp, l, stream); break;
    case 3: launch_spread_width<D, 3>(sp, l, stream); break;
    case 4: launch_spread_width<D, 4>(sp, l, stream); break;
    case 5: launch_spread_width<D, 5>(sp, l, stream); break;
    case 6: launch_spread_width<D, 6>(sp, l, stream); break;
    case 7: launch_spread_width<D, 7>(sp, l, stream); break;
    case 8: launch_spread_width<D, 8>(sp, l, stream); break;
    case 9: launch_spread_width<D, 9>(sp, l, stream); break;
    case 10: launch_spread_width<D, 10>(sp, l, stream); break;
    case 11: launch_spread_width<D, 11>(sp, l, stream); break;
    case 12: launch_spread_width<D, 12>(sp, l, stream); break;
    case 13: launch_spread_width<D, 13>(sp, l, stream); break;
    case 14: launch_spread_width<D, 14>(sp, l, stream); break;
    case 15: launch_spread_width<D, 15>(sp, l, stream); break;
    default: launch_spread_width<D, 16>(sp, l, stream); break;
  }
}

}  // namespace

void spread_count_parts(const SpreadParams& sp, const uint32_t* offsets, uint32_t* parts,
                        uint32_t* part_start, cudaStream_t stream, StageTimer* timer) {
  StageScope scope(timer, kStageTileParts, stream);
  const unsigned blocks = static_cast<unsigned>((sp.tile_count + 255) / 256);
  switch (sp.grid.dimensions) {
    case 1: tile_records_kernel<1><<<blocks, 256, 0, stream>>>(sp, offsets, parts); break;
    case 2: tile_records_kernel<2><<<blocks, 256, 0, stream>>>(sp, offsets, parts); break;
    default: tile_records_kernel<3><<<blocks, 256, 0, stream>>>(sp, offsets, parts); break;
  }
  part_scan_kernel<<<1, 1024, 0, stream>>>(parts, sp.tile_count, part_start);
  note_launch(2);
}

void spread_execute(const SpreadParams& sp, const SpreadLaunch& l, cudaStream_t stream,
                    StageTimer* timer) {
  if (l.point_count > 0) {
    {
      StageScope scope(timer, kStageStrengthScale, stream);
      check_cuda(cudaMemsetAsync(l.max_bits, 0, sizeof(uint32_t) * l.batch, stream), "clear maxima");
      const unsigned blocks =
          static_cast<unsigned>(std::min<int64_t>((l.point_count + 255) / 256, 148 * 8));
      strength_magnitude_kernel<<<dim3(blocks, l.batch), 256, 0, stream>>>(
          l.strengths, l.point_count, l.batch, l.max_bits);
      note_launch();
    }
    StageScope scope(timer, kStageSpread, stream);
    switch (sp.grid.dimensions) {
      case 1: launch_spread_dim<1>(sp, l, stream); break;
      case 2: launch_spread_dim<2>(sp, l, stream); break;
      default: launch_spread_dim<3>(sp, l, stream); break;
    }
  }
  StageScope scope(timer, kStageFold, stream);
  const dim3 grid(static_cast<unsigned>((sp.grid.fine_count + 255) / 256),
                  static_cast<unsigned>(l.batch));
  switch (sp.grid.dimensions) {
    case 1:
      fold_tiles_kernel<1><<<grid, 256, 0, stream>>>(sp, l.batch, l.scratch, l.part_start,
                                                     l.part_upper_bound, l.candidates, l.fine);
      break;
    case 2:
      fold_tiles_kernel<2><<<grid, 256, 0, stream>>>(sp, l.batch, l.scratch, l.part_start,
                                                     l.part_upper_bound, l.candidates, l.fine);
      break;
    default:
      fold_tiles_kernel<3><<<grid, 256, 0, stream>>>(sp, l.batch, l.scratch, l.part_start,
                                                     l.part_upper_bound, l.candidates, l.fine);
      break;
  }
  note_launch();
}

}  // namespace b200nufft
