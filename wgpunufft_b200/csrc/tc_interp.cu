// Batched 2D type-2 interpolation on the tcgen05 tensor cores.
//
// The reference interpolates every vector separately: a workgroup of lanes
// per point sums its w x w cells in lane order (src/gpu_2d.rs:1022-1113,
// workgroups over the batch at :566-575). With many vectors on one point set
// the same sums are a dense contraction, which this file runs on the tensor
// cores.
//
// A tcgen05 MMA of M = 128 costs about the same issue time for any N up to
// 128 (measured with b200nufft_tf32_peak), so the contraction is cut into
// wide chunks: per point set (set_points) the points are ordered a second
// time, by the exact support start in bins of 8 x 4 cells (a column group of
// 8 cells over a band of 4 rows), and every point gets its window record (y
// weights, and x weights placed at their column within the 16 columns the
// group's windows reach). A tile is one column group over kTi2TileRows rows;
// its chunks are the runs of at most 128 points of one band, in row order.
//
// Precision: f16 has the 11-bit significand of tf32 and K = 16 per MMA, so a
// 16-cell row is one MMA step. Values are scaled by powers of two before the
// split (grid values of vector v by 2^(14 - e_v), with 2^e_v above the
// vector's largest |re|, |im| found by a max pass after the FFT; weights by
// 2^14), which keeps the high parts and all but the tiniest low parts normal;
// the high part is the value cut to f16's 10 significand bits (as the tf32
// split of the spreader cuts to tf32's), the low part the rounded remainder;
// A_hi B_hi + A_hi B_lo + A_lo B_hi accumulate in f32 and the read-out
// multiplies the power of two back (exact).
//
// Per execution, one CTA per (tile part, 64 vectors) walks its chunks in row
// order with warp-specialised roles joined by mbarriers. A producer warp
// brings the fine-grid rows the chunks reach (16 columns x 64 vectors, one
// tensor copy per row) into shared memory, ten rows ahead; four converter
// warps scale every row and split it into f16 high and low parts, each lane
// one of the 128 A rows (real or imaginary part of a vector), into a ring of
// 16 rows in tensor memory; four builder warps, a lane per point, write B
// steps (per window-union row u of the chunk: wy[u - dy] wx over the 16
// columns, high and low parts) into a ring of 12 steps, with the next
// chunk's window records copied while they build; one elected lane issues,
// per chunk at band row y, w + 3 steps of 3 MMAs (M = 128, N = 16 .. 128,
// K = 16, A = ring row y + u) into one of two tensor-memory accumulators and
// retires ring rows the next chunk no longer reads; four read-out warps move
// each accumulator to the values in tensor-core slot order, and a final pass
// writes them in the caller's point order. Every output comes from the MMAs
// of one chunk issued in a fixed order, so results are bitwise repeatable.
//
// Every wait is bounded: a wait that gives up stops the CTA's work, lets the
// copies and MMAs in flight finish (again with a bound), frees the tensor
// memory and increments the plan's error flag.
#include "tc_interp.h"

#include <cuda.h>
#include <cuda_fp16.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "interp.h"
#include "spread.h"
#include "tc_common.cuh"

namespace b200nufft {

namespace {

using namespace tc;

// Warp roles. Converter and read-out warps access the tensor-memory lane
// quadrant warp % 4.
constexpr int kProducerWarp = 0;
constexpr int kMmaWarp = 1;
constexpr int kConvertWarp0 = 2;   // four warps: each lane converts one A row of a fetched row
constexpr int kBuildWarp0 = 6;     // four warps: a lane per point of the chunk
constexpr int kReadWarp0 = 10;     // four warps: one per tensor-memory lane quadrant
constexpr int kThreads = 14 * 32;
constexpr int kConvertThreads = 128;
constexpr int kBuildThreads = 128;
constexpr int kReadThreads = 128;
static_assert(kBuildThreads == kTi2ChunkPoints, "a builder lane per chunk point");
static_assert((kBuildWarp0 - kConvertWarp0) * 32 == kConvertThreads, "a converter lane per A row");

constexpr int kBuffers = 2;                  // accumulators of kTi2ChunkPoints columns
constexpr int kRingSlotColumns = 16;         // one converted row: 8 columns of f16 pairs, high then low
constexpr int kRing = 16;                    // converted rows in tensor memory
constexpr int kRingColumn0 = kBuffers * kTi2ChunkPoints;
constexpr int kTmemColumns = 512;
static_assert(kRingColumn0 + kRing * kRingSlotColumns <= kTmemColumns, "tensor-memory ring exceeds the allocation");
static_assert(kRing > kTi2MaxWidth + kTi2BandRows - 1, "the ring holds a chunk's window rows and one more");
constexpr int kRawSlots = 10;                // fetched rows in flight
constexpr int kRawPitch = 144;               // bytes per vector of a fetched row: 16 complex cells and 2 more
                                             // (the tensor copy's box), a pitch without bank conflicts
constexpr int kRawBytes = kTi2Vectors * kRawPitch;
constexpr int kSteps = 12;                   // B steps in flight
constexpr int kStepHalf = kTi2ChunkPoints * kTi2Pitch * 2;  // one f16 part of a step: 128 points x 16 cells
constexpr int kStepBytes = 2 * kStepHalf;
constexpr int kWeightStages = 2;
constexpr int kWeightStage = kTi2ChunkPoints * static_cast<int>(sizeof(TcWeights));
constexpr float kWeightScale = 16384.0f;     // 2^14: weights (at most 1) stay below the f16 maximum
constexpr int kWeightScaleLog2 = 14;
constexpr int kValueScaleLog2 = 14;          // grid values scaled below 2^14

constexpr int kStepBase = 0;
constexpr int kRawBase = kStepBase + kSteps * kStepBytes;
constexpr int kWeightsBase = kRawBase + kRawSlots * kRawBytes;
constexpr int kSmemBytes = kWeightsBase + kWeightStages * kWeightStage;

// Window records in tensor-core slot order and the slot of every point:
// the support start and offsets of the prepared windows (the fold of
// src/gpu_nd_wgsl.rs:263-298) and the f32 Horner panels of the window.
template <int W>
__global__ void ti2_weights_kernel(GridParams g, const float* __restrict__ points, int64_t count,
                                   const uint32_t* __restrict__ perm, TcWeights* __restrict__ out,
                                   uint32_t* __restrict__ inverse) {
  const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= count) return;
  const uint32_t p = perm[s];
  TcWeights r;
  r.sx = r.sy = 0;
  r.unused[0] = r.unused[1] = 0;
#pragma unroll
  for (int j = 0; j < kTcMaxWidth; ++j) r.wy[j] = 0.0f;
#pragma unroll
  for (int c = 0; c < 2 * kTcTileX; ++c) r.wxs[c] = 0.0f;
  const float x = points[2 * static_cast<int64_t>(p)], y = points[2 * static_cast<int64_t>(p) + 1];
  if (in_fold_reach(x) && in_fold_reach(y)) {
    int32_t start;
    Df64 off;
    float wx[W], wy[W];
    support_of(x, g.axis[0], g.half_width, start, off);
    r.sx = wrap_start(start, g.axis[0].length);
    horner32_window<W>(__fadd_rn(off.hi, off.lo), g.horner32, wx);
    support_of(y, g.axis[1], g.half_width, start, off);
    r.sy = wrap_start(start, g.axis[1].length);
    horner32_window<W>(__fadd_rn(off.hi, off.lo), g.horner32, wy);
    const int dx = r.sx & (kTi2GroupX - 1);
#pragma unroll
    for (int j = 0; j < W; ++j) {
      r.wy[j] = wy[j];
#pragma unroll
      for (int d = 0; d < kTi2GroupX; ++d) {
        if (d == dx) r.wxs[d + j] = wx[j];
      }
    }
  }
  out[s] = r;
  inverse[p] = static_cast<uint32_t>(s);
}

__device__ __forceinline__ void tile_origin(const GridParams& g, int64_t t, int& tx, int& ty) {
  const int64_t groups = g.axis[0].bins;
  tx = static_cast<int>(t % groups);
  ty = static_cast<int>(t / groups);
}

// Chunks and parts of every tile: runs of at most kTi2ChunkPoints points of
// one band, bands in row order.
__global__ void ti2_tile_chunks_kernel(GridParams g, int64_t tiles, const uint32_t* __restrict__ offsets,
                                       uint32_t* __restrict__ tile_chunks, uint32_t* __restrict__ parts) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= tiles) return;
  int tx, ty;
  tile_origin(g, t, tx, ty);
  const int bands = static_cast<int>(g.axis[1].bins);
  const int b0 = ty * (kTi2TileRows / kTi2BandRows);
  const int b_end = min(b0 + kTi2TileRows / kTi2BandRows, bands);
  const uint64_t groups = g.axis[0].bins;
  uint32_t chunks = 0;
  for (int band = b0; band < b_end; ++band) {
    const uint64_t b = tx + groups * static_cast<uint64_t>(band);
    const uint32_t n = offsets[b + 1] - offsets[b];
    chunks += (n + kTi2ChunkPoints - 1) / kTi2ChunkPoints;
  }
  tile_chunks[t] = chunks;
  parts[t] = (chunks + kTi2ChunksPerPart - 1) / kTi2ChunksPerPart;
}

__global__ void ti2_chunk_fill_kernel(GridParams g, int64_t tiles, const uint32_t* __restrict__ offsets,
                                      const uint32_t* __restrict__ tile_chunk_start, Ti2Chunk* __restrict__ chunks) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= tiles) return;
  int tx, ty;
  tile_origin(g, t, tx, ty);
  const int bands = static_cast<int>(g.axis[1].bins);
  const int b0 = ty * (kTi2TileRows / kTi2BandRows);
  const int b_end = min(b0 + kTi2TileRows / kTi2BandRows, bands);
  const uint64_t groups = g.axis[0].bins;
  uint32_t next = tile_chunk_start[t];
  for (int band = b0; band < b_end; ++band) {
    const uint64_t b = tx + groups * static_cast<uint64_t>(band);
    const uint32_t begin = offsets[b], end = offsets[b + 1];
    for (uint32_t s = begin; s < end; s += kTi2ChunkPoints) {
      Ti2Chunk c;
      c.slot = s;
      c.count = static_cast<uint16_t>(min(static_cast<uint32_t>(kTi2ChunkPoints), end - s));
      c.row = static_cast<uint16_t>((band - b0) * kTi2BandRows);
      chunks[next++] = c;
    }
  }
}

// Largest |re|, |im| of every vector's fine grid, as float bits (atomicMax on
// the bits of non-negative floats does not depend on the order).
__global__ void ti2_vector_max_kernel(const float4* __restrict__ fine, int64_t pairs_per_vector,
                                      uint32_t* __restrict__ vector_max) {
  const int v = blockIdx.y;
  const float4* grid = fine + static_cast<int64_t>(v) * pairs_per_vector;
  float m = 0.0f;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < pairs_per_vector;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const float4 q = grid[i];
    m = fmaxf(m, fmaxf(fmaxf(fabsf(q.x), fabsf(q.y)), fmaxf(fabsf(q.z), fabsf(q.w))));
  }
  const uint32_t bits = __reduce_max_sync(0xFFFFFFFFu, __float_as_uint(m));
  if ((threadIdx.x & 31) == 0) atomicMax(&vector_max[v], bits);
}

// The power-of-two scale of a vector's grid values from their largest
// magnitude (bits): 2^(14 - e) with 2^e above it; 1 for a zero or non-finite
// maximum.
__device__ __forceinline__ int value_scale_exponent(uint32_t max_bits) {
  const float m = __uint_as_float(max_bits);
  if (!(m > 0.0f) || !isfinite(m)) return 0;
  int e;
  frexpf(m, &e);  // m = f 2^e, f in [0.5, 1)
  return max(-100, min(100, kValueScaleLog2 - e));
}

// f16 high and low parts of two scaled values: the high part keeps the sign,
// exponent and 10 explicit significand bits (exact in f16 for the normal
// range the scales keep values in), the low part is the exact remainder
// rounded to f16; two conversions per pair.
__device__ __forceinline__ void split_f16x2(float x0, float x1, uint32_t& hi, uint32_t& lo) {
  const float h0 = __uint_as_float(__float_as_uint(x0) & 0xFFFFE000u);
  const float h1 = __uint_as_float(__float_as_uint(x1) & 0xFFFFE000u);
  const __half2 h = __floats2half2_rn(h0, h1);
  const __half2 l = __floats2half2_rn(x0 - h0, x1 - h1);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

// Converts A row m = 2 v + part of fetched row `raw` (vector v's 16 complex
// cells at kRawPitch), scaled by `scale`, into 8 columns of f16 high-part
// pairs followed by 8 columns of low-part pairs (lower cell in the low half;
// zero for vectors at or beyond nv).
__device__ __forceinline__ void ti2_convert_lane(const unsigned char* raw, int m, int nv, float scale, uint32_t* out) {
  const int v = m >> 1, part = m & 1;
  const float4* row = reinterpret_cast<const float4*>(raw + v * kRawPitch);
  float4 cells[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) cells[i] = row[i];
  const float s = v < nv ? scale : 0.0f;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const float x0 = (part ? cells[i].y : cells[i].x) * s;
    const float x1 = (part ? cells[i].w : cells[i].z) * s;
    split_f16x2(x0, x1, out[i], out[8 + i]);
  }
}

template <int W>
__global__ void __launch_bounds__(kThreads, 1) tc_interp_kernel(
    GridParams g, const float2* __restrict__ fine, int batch, const TcWeights* __restrict__ weights,
    const Ti2Chunk* __restrict__ chunks, const uint32_t* __restrict__ tile_chunk_start,
    const uint32_t* __restrict__ part_start, int64_t tiles, float2* __restrict__ staged, int64_t staged_stride,
    const uint32_t* __restrict__ vector_max, uint32_t* __restrict__ error_flag,
    const __grid_constant__ CUtensorMap fine_map, int use_map) {
  constexpr int kRows = W + kTi2BandRows - 1;  // window-union rows of a chunk: MMA steps
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t raw_full[kRawSlots], raw_empty[kRawSlots];
  __shared__ __align__(8) uint64_t a_full[kRing], a_empty[kRing];
  __shared__ __align__(8) uint64_t b_full[kSteps], b_empty[kSteps];
  __shared__ __align__(8) uint64_t w_full[kWeightStages], w_empty[kWeightStages];
  __shared__ __align__(8) uint64_t d_full[kBuffers], d_empty[kBuffers];
  __shared__ uint32_t tmem_base;
  __shared__ int64_t s_tile;
  __shared__ int s_abort;
  __shared__ float s_scale[kTi2Vectors], s_unscale[kTi2Vectors];
  __shared__ Ti2Chunk s_chunks[kTi2ChunksPerPart];

  const uint32_t part = blockIdx.x;
  if (part >= part_start[tiles]) return;
  const int group = blockIdx.y;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int vb = group * kTi2Vectors;
  const int nv = min(kTi2Vectors, batch - vb);
  if (tid == 0) {
    int64_t low = 0, high = tiles - 1;
    while (low < high) {
      const int64_t mid = (low + high + 1) >> 1;
      if (part_start[mid] <= part) low = mid; else high = mid - 1;
    }
    s_tile = low;
    s_abort = 0;
    for (int s = 0; s < kRawSlots; ++s) {
      mbar_init(&raw_full[s], 1);
      mbar_init(&raw_empty[s], kConvertThreads);
    }
    for (int s = 0; s < kRing; ++s) {
      mbar_init(&a_full[s], kConvertThreads);
      mbar_init(&a_empty[s], 1);
    }
    for (int s = 0; s < kSteps; ++s) {
      mbar_init(&b_full[s], kBuildThreads);
      mbar_init(&b_empty[s], 1);
    }
    for (int s = 0; s < kWeightStages; ++s) {
      mbar_init(&w_full[s], 1);
      mbar_init(&w_empty[s], kBuildThreads);
    }
    for (int b = 0; b < kBuffers; ++b) {
      mbar_init(&d_full[b], 1);
      mbar_init(&d_empty[b], kReadThreads);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (tid < kTi2Vectors) {
    const int e = tid < nv ? value_scale_exponent(vector_max[vb + tid]) : 0;
    s_scale[tid] = ldexpf(1.0f, e);
    s_unscale[tid] = ldexpf(1.0f, -e - kWeightScaleLog2);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(kTmemColumns));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tm = tmem_base;
  const int64_t tile = s_tile;
  const uint32_t first = tile_chunk_start[tile] + (part - part_start[tile]) * kTi2ChunksPerPart;
  const uint32_t stop = min(first + static_cast<uint32_t>(kTi2ChunksPerPart), tile_chunk_start[tile + 1]);
  const int n = stop > first ? static_cast<int>(stop - first) : 0;
  for (int c = tid; c < n; c += kThreads) s_chunks[c] = chunks[first + c];
  __syncthreads();

  int tx, ty;
  tile_origin(g, tile, tx, ty);
  const int n0 = g.axis[0].length, n1 = g.axis[1].length;
  const int x0 = tx * kTi2GroupX, y0 = ty * kTi2TileRows;
  // Rows [r_begin, r_begin + rows) relative to y0 are fetched and converted in order.
  const int r_begin = n > 0 ? s_chunks[0].row : 0;
  const int rows = n > 0 ? s_chunks[n - 1].row + kRows - r_begin : 0;
  unsigned char* raw = smem + kRawBase;
  volatile int* abort_flag = &s_abort;

  if (warp == kProducerWarp) {
    // Row k into raw slot k % kRawSlots once the converters are done with row k - kRawSlots.
    int issued = 0;
    for (int k = 0; k < rows; ++k) {
      const int slot = k % kRawSlots;
      bool ok = true;
      if (lane == 0 && k >= kRawSlots) {
        ok = mbar_wait(smem_u32(&raw_empty[slot]), static_cast<uint32_t>(k / kRawSlots - 1) & 1u, abort_flag);
      }
      ok = __shfl_sync(0xFFFFFFFFu, ok ? 1 : 0, 0) != 0;
      if (!ok) break;
      const uint32_t bar = smem_u32(&raw_full[slot]);
      const int y = (y0 + r_begin + k) % n1;
      unsigned char* dst = raw + slot * kRawBytes;
      if (use_map && x0 + 2 * kTi2GroupX <= n0) {
        // One tensor copy: 18 cells (36 floats; the last two unused, zeros
        // beyond the row) of row y for vectors vb .. vb + 63 (vectors beyond
        // the batch arrive as zeros).
        if (lane == 0) {
          mbar_expect(bar, static_cast<uint32_t>(kRawBytes));
          tensor_load_3d(smem_u32(dst), &fine_map, 2 * x0, y, vb, bar);
        }
        __syncwarp();
      } else {
        if (lane == 0) mbar_expect(bar, static_cast<uint32_t>(nv) * 128u);  // 16 cells of each vector
        __syncwarp();
        const int64_t row = static_cast<int64_t>(y) * n0;
        for (int v = lane; v < nv; v += 32) {
          const float2* grid = fine + static_cast<int64_t>(vb + v) * g.fine_count + row;
          const uint32_t d = smem_u32(dst + v * kRawPitch);
          if (x0 + 2 * kTi2GroupX <= n0) {
            bulk_load(d, grid + x0, 128, bar);
          } else {
            bulk_load(d, grid + x0, 64, bar);
            bulk_load(d + 64, grid, 64, bar);
          }
        }
      }
      issued = k + 1;
    }
    // Copies in flight land before the CTA leaves (bounded, without abort).
    if (lane == 0) {
      for (int k = max(0, issued - kRawSlots); k < issued; ++k) {
        if (!mbar_wait(smem_u32(&raw_full[k % kRawSlots]), static_cast<uint32_t>(k / kRawSlots) & 1u, nullptr)) {
          *abort_flag = 1;
        }
      }
    }
  } else if (warp == kMmaWarp) {
    // The whole warp walks the chunks (operands warp-uniform); one elected
    // lane issues each MMA and commit.
    int ready = 0;    // rows [0, ready) relative to r_begin are converted
    int retired = 0;  // rows [0, retired) are released to the converters
    int issued = 0;
    uint32_t step = 0;
    bool ok = true;
    for (int c = 0; c < n && ok; ++c) {
      const Ti2Chunk ch = s_chunks[c];
      const int r = ch.row - r_begin;
      while (ok && ready < r + kRows) {
        ok = mbar_wait(smem_u32(&a_full[ready % kRing]), static_cast<uint32_t>(ready / kRing) & 1u, abort_flag);
        ok = __all_sync(0xFFFFFFFFu, ok);
        ready += ok ? 1 : 0;
        // Rows below this chunk's first row are read by no later chunk:
        // release them at once, so rows skipped between chunks free their
        // ring slots while this chunk waits for its own rows.
        for (; retired < min(r, ready); ++retired) {
          if (elect_one()) mma_commit(smem_u32(&a_empty[retired % kRing]));
          __syncwarp();
        }
      }
      if (ok && c >= kBuffers) {
        ok = mbar_wait(smem_u32(&d_empty[c % kBuffers]), static_cast<uint32_t>(c / kBuffers - 1) & 1u, abort_flag);
      }
      ok = __all_sync(0xFFFFFFFFu, ok);
      if (!ok) break;
      tc_fence_after();
      const uint32_t cols = static_cast<uint32_t>((ch.count + 15) & ~15);
      const uint32_t idesc = idesc_f16(128, cols);
      const uint32_t d = tm + static_cast<uint32_t>((c % kBuffers) * kTi2ChunkPoints);
      // Steps in pairs: both B steps are waited for, then one elected block
      // issues their 6 MMAs and 2 commits.
#pragma unroll 1
      for (int u = 0; u < kRows && ok; u += 2) {
        const int pair = min(2, kRows - u);
        const int stage0 = static_cast<int>(step % kSteps), stage1 = static_cast<int>((step + 1) % kSteps);
        ok = mbar_wait(smem_u32(&b_full[stage0]), (step / kSteps) & 1u, abort_flag);
        if (ok && pair == 2) ok = mbar_wait(smem_u32(&b_full[stage1]), ((step + 1) / kSteps) & 1u, abort_flag);
        ok = __all_sync(0xFFFFFFFFu, ok);
        if (!ok) break;
        tc_fence_after();
        // Ring slot of window-union row u: high pairs in columns 0 .. 7, low pairs in 8 .. 15.
        const uint32_t a0 = tm + static_cast<uint32_t>(kRingColumn0 + ((r + u) % kRing) * kRingSlotColumns);
        const uint32_t a1 = tm + static_cast<uint32_t>(kRingColumn0 + ((r + u + 1) % kRing) * kRingSlotColumns);
        const uint32_t b0 = smem_u32(smem + kStepBase + stage0 * kStepBytes);
        const uint32_t b1 = smem_u32(smem + kStepBase + stage1 * kStepBytes);
        const uint64_t b0hi = kmajor_desc(b0), b0lo = kmajor_desc(b0 + kStepHalf);
        const uint64_t b1hi = kmajor_desc(b1), b1lo = kmajor_desc(b1 + kStepHalf);
        if (elect_one()) {
          mma_f16_tmem_a(d, a0, b0hi, idesc, u > 0);
          mma_f16_tmem_a(d, a0, b0lo, idesc, true);
          mma_f16_tmem_a(d, a0 + 8, b0hi, idesc, true);
          mma_commit(smem_u32(&b_empty[stage0]));
          if (pair == 2) {
            mma_f16_tmem_a(d, a1, b1hi, idesc, true);
            mma_f16_tmem_a(d, a1, b1lo, idesc, true);
            mma_f16_tmem_a(d, a1 + 8, b1hi, idesc, true);
            mma_commit(smem_u32(&b_empty[stage1]));
          }
        }
        __syncwarp();
        step += static_cast<uint32_t>(pair);
      }
      if (!ok) break;
      if (elect_one()) mma_commit(smem_u32(&d_full[c % kBuffers]));
      __syncwarp();
      issued = c + 1;
      // Rows below the next chunk's first row are read by no later chunk.
      const int next = c + 1 < n ? s_chunks[c + 1].row - r_begin : rows;
      for (; retired < min(next, ready); ++retired) {
        if (elect_one()) mma_commit(smem_u32(&a_empty[retired % kRing]));
        __syncwarp();
      }
    }
    if (lane == 0) {
      // Every MMA issued (of the last full chunk and of a chunk left
      // part-way) completes before the tensor memory is freed: the commits
      // of its steps cover it.
      if (step > 0 &&
          !mbar_wait(smem_u32(&b_empty[(step - 1) % kSteps]), ((step - 1) / kSteps) & 1u, nullptr)) {
        *abort_flag = 1;
      }
      if (issued > 0 &&
          !mbar_wait(smem_u32(&d_full[(issued - 1) % kBuffers]), static_cast<uint32_t>((issued - 1) / kBuffers) & 1u,
                     nullptr)) {
        *abort_flag = 1;
      }
      if (!ok) *abort_flag = 1;
    }
  } else if (warp < kBuildWarp0) {
    // Converters: lane (warp % 4, lane) owns A row m = 32 (warp % 4) + lane
    // and writes its 16 columns of every ring slot.
    const int quadrant = warp & 3;
    const int m = quadrant * 32 + lane;
    const float scale = s_scale[m >> 1];
    const uint32_t lane_base = tm + (static_cast<uint32_t>(quadrant * 32) << 16);
    for (int k = 0; k < rows; ++k) {
      if (!mbar_wait(smem_u32(&raw_full[k % kRawSlots]), static_cast<uint32_t>(k / kRawSlots) & 1u, abort_flag)) break;
      uint32_t cols[16];
      ti2_convert_lane(raw + (k % kRawSlots) * kRawBytes, m, nv, scale, cols);
      mbar_arrive(smem_u32(&raw_empty[k % kRawSlots]));
      if (k >= kRing &&
          !mbar_wait(smem_u32(&a_empty[k % kRing]), static_cast<uint32_t>(k / kRing - 1) & 1u, abort_flag)) {
        break;
      }
      tc_fence_after();
      tmem_st16(lane_base + static_cast<uint32_t>(kRingColumn0 + (k % kRing) * kRingSlotColumns), cols);
      tmem_wait_st();
      tc_fence_before();
      mbar_arrive(smem_u32(&a_full[k % kRing]));
    }
  } else if (warp < kReadWarp0) {
    // Builders: lane t (of 128) holds point t of the chunk: its window record
    // in registers, from which it writes its B column of every step. The
    // records of chunk c + 2 are copied into the stage of chunk c once every
    // lane holds its record.
    const int t = tid - kBuildWarp0 * 32;
    static_assert(kWeightStages == 2, "record copies per stage are counted in two registers");
    int loads0 = 0, loads1 = 0;  // record copies issued into stage 0 and stage 1
    if (t == 0) {
      for (int c = 0; c < min(n, kWeightStages); ++c) {
        const Ti2Chunk ch = s_chunks[c];
        const uint32_t bytes = static_cast<uint32_t>(ch.count) * static_cast<uint32_t>(sizeof(TcWeights));
        mbar_expect(smem_u32(&w_full[c]), bytes);
        bulk_load(smem_u32(smem + kWeightsBase + c * kWeightStage), weights + ch.slot, bytes, smem_u32(&w_full[c]));
      }
      loads0 = n > 0 ? 1 : 0;
      loads1 = n > 1 ? 1 : 0;
    }
    uint32_t step = 0;
    for (int c = 0; c < n; ++c) {
      const Ti2Chunk ch = s_chunks[c];
      const int ws = c % kWeightStages;
      if (!mbar_wait(smem_u32(&w_full[ws]), static_cast<uint32_t>(c / kWeightStages) & 1u, abort_flag)) break;
      const TcWeights* s_w = reinterpret_cast<const TcWeights*>(smem + kWeightsBase + ws * kWeightStage);
      float wy[W];
      float4 wx[4];
      int dy = 0;
      if (t < ch.count) {
        dy = s_w[t].sy - (y0 + ch.row);
#pragma unroll
        for (int j = 0; j < W; ++j) wy[j] = s_w[t].wy[j] * kWeightScale;
#pragma unroll
        for (int q = 0; q < 4; ++q) wx[q] = *reinterpret_cast<const float4*>(&s_w[t].wxs[4 * q]);
      } else {
#pragma unroll
        for (int j = 0; j < W; ++j) wy[j] = 0.0f;
#pragma unroll
        for (int q = 0; q < 4; ++q) wx[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      }
      mbar_arrive(smem_u32(&w_empty[ws]));
      if (t == 0 && c + kWeightStages < n) {
        // Every lane holds its record: the stage takes chunk c + 2's.
        if (!mbar_wait(smem_u32(&w_empty[ws]), static_cast<uint32_t>(c / kWeightStages) & 1u, abort_flag)) break;
        const Ti2Chunk nx = s_chunks[c + kWeightStages];
        const uint32_t bytes = static_cast<uint32_t>(nx.count) * static_cast<uint32_t>(sizeof(TcWeights));
        mbar_expect(smem_u32(&w_full[ws]), bytes);
        bulk_load(smem_u32(smem + kWeightsBase + ws * kWeightStage), weights + nx.slot, bytes, smem_u32(&w_full[ws]));
        if (ws == 0) ++loads0; else ++loads1;
      }
      // B column of point t for step u: wy[u - dy] wx[0 .. 15] (zero outside
      // the window), K-major f16: cells 0-7 and 8-15 of the high part 128
      // bytes apart, 8-point groups 256 bytes apart, the low part kStepHalf on.
      const int column = (t >> 3) * 256 + (t & 7) * 16;
      bool ok = true;
#pragma unroll
      for (int u = 0; u < kRows; ++u, ++step) {
        const int stage = static_cast<int>(step % kSteps);
        if (step >= static_cast<uint32_t>(kSteps) &&
            !mbar_wait(smem_u32(&b_empty[stage]), ((step / kSteps) - 1) & 1u, abort_flag)) {
          ok = false;
          break;
        }
        float w = 0.0f;
#pragma unroll
        for (int j = 0; j < W; ++j) {
          if (u - j == dy) w = wy[j];
        }
        const float v[16] = {w * wx[0].x, w * wx[0].y, w * wx[0].z, w * wx[0].w, w * wx[1].x, w * wx[1].y,
                             w * wx[1].z, w * wx[1].w, w * wx[2].x, w * wx[2].y, w * wx[2].z, w * wx[2].w,
                             w * wx[3].x, w * wx[3].y, w * wx[3].z, w * wx[3].w};
        uint32_t hi[8], lo[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) split_f16x2(v[2 * i], v[2 * i + 1], hi[i], lo[i]);
        unsigned char* st = smem + kStepBase + stage * kStepBytes + column;
        *reinterpret_cast<uint4*>(st) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
        *reinterpret_cast<uint4*>(st + 128) = make_uint4(hi[4], hi[5], hi[6], hi[7]);
        *reinterpret_cast<uint4*>(st + kStepHalf) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
        *reinterpret_cast<uint4*>(st + kStepHalf + 128) = make_uint4(lo[4], lo[5], lo[6], lo[7]);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive(smem_u32(&b_full[stage]));
      }
      if (!ok) break;
    }
    // Record copies in flight land before the CTA leaves.
    if (t == 0) {
      if (loads0 > 0 && !mbar_wait(smem_u32(&w_full[0]), static_cast<uint32_t>(loads0 - 1) & 1u, nullptr)) {
        *abort_flag = 1;
      }
      if (loads1 > 0 && !mbar_wait(smem_u32(&w_full[1]), static_cast<uint32_t>(loads1 - 1) & 1u, nullptr)) {
        *abort_flag = 1;
      }
    }
  } else {
    // Read-out: warp (warp % 4 = q) holds rows 32 q + lane (vector m / 2,
    // real part when m is even) of each accumulator; values go out in
    // tensor-core slot order, scaled back.
    const int q = warp & 3;
    const int m = q * 32 + lane;
    const int vec = m >> 1;
    const float unscale = s_unscale[vec];
    for (int c = 0; c < n; ++c) {
      if (!mbar_wait(smem_u32(&d_full[c % kBuffers]), static_cast<uint32_t>(c / kBuffers) & 1u, abort_flag)) break;
      tc_fence_after();
      const Ti2Chunk ch = s_chunks[c];
      const uint32_t addr =
          tm + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>((c % kBuffers) * kTi2ChunkPoints);
      const int pieces = (ch.count + 31) >> 5;
      for (int piece = 0; piece < pieces; ++piece) {
        uint32_t v[32];
        tmem_ld32(addr + static_cast<uint32_t>(piece * 32), v);
        tmem_wait_ld();
        if (piece == pieces - 1) {
          tc_fence_before();
          mbar_arrive(smem_u32(&d_empty[c % kBuffers]));
        }
#pragma unroll
        for (int i = 0; i < 32; ++i) {
          const float x = __uint_as_float(v[i]) * unscale;
          const float y = __shfl_xor_sync(0xFFFFFFFFu, x, 1);
          const int point = piece * 32 + i;
          if ((m & 1) == 0 && point < ch.count && vec < nv) {
            staged[(static_cast<int64_t>(ch.slot) + point) * staged_stride + vb + vec] = make_float2(x, y);
          }
        }
      }
    }
  }

  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(kTmemColumns));
  }
  if (tid == 0 && *abort_flag) atomicAdd(error_flag, 1u);
}

template <int W>
void launch_weights(const GridParams& g, const Ti2Prepare& p, cudaStream_t stream) {
  const unsigned blocks = static_cast<unsigned>((p.count + 255) / 256);
  ti2_weights_kernel<W><<<blocks, 256, 0, stream>>>(g, p.points, p.count, p.perm, p.weights, p.inverse);
  note_launch();
}

// The fine grid of `batch` vectors as a 3D tensor (32-bit elements: 2 n0
// floats per row, n1 rows, batch vectors) with boxes of 36 floats x 1 row x
// 64 vectors (a 144-byte pitch in shared memory); false when the driver
// offers no tensor-map encoder.
bool encode_fine_map(const float2* fine, int n0, int n1, int64_t fine_count, int batch, CUtensorMap* map) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult status;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &status) != cudaSuccess ||
        status != cudaDriverEntryPointSuccess) {
      fn = nullptr;
    }
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }();
  if (encode == nullptr) return false;
  const cuuint64_t dims[3] = {static_cast<cuuint64_t>(2 * n0), static_cast<cuuint64_t>(n1),
                              static_cast<cuuint64_t>(batch)};
  const cuuint64_t strides[2] = {static_cast<cuuint64_t>(n0) * 8, static_cast<cuuint64_t>(fine_count) * 8};
  const cuuint32_t box[3] = {static_cast<cuuint32_t>(kRawPitch / 4), 1, static_cast<cuuint32_t>(kTi2Vectors)};
  const cuuint32_t element_strides[3] = {1, 1, 1};
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float2*>(fine), dims, strides, box,
                element_strides, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int W>
void launch_interp(const GridParams& g, const Ti2Launch& l, int64_t tiles, int64_t stride, const CUtensorMap& map,
                   bool use_map, cudaStream_t stream) {
  static_assert(kSmemBytes + 4096 <= 227 * 1024, "tensor-core interpolation stages exceed shared memory");
  auto kernel = tc_interp_kernel<W>;
  check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemBytes),
             "tensor-core interpolation shared memory");
  const int groups = (l.batch + kTi2Vectors - 1) / kTi2Vectors;
  const dim3 grid(static_cast<unsigned>(l.part_upper_bound), static_cast<unsigned>(groups));
  kernel<<<grid, kThreads, kSmemBytes, stream>>>(g, l.fine, l.batch, l.weights, l.chunks, l.tile_chunk_start,
                                                 l.part_start, tiles, l.staged, stride, l.vector_max, l.error_flag,
                                                 map, use_map ? 1 : 0);
  note_launch();
}

}  // namespace

bool tc_interp_supported(const GridParams& g) {
  return g.dimensions == 2 && g.width >= 2 && g.width <= kTi2MaxWidth && g.fine[0] % kTi2GroupX == 0 &&
         g.fine[0] >= 2 * kTi2GroupX && g.fine[1] % kTi2BandRows == 0 && g.fine[1] >= g.width;
}

GridParams tc_interp_bins(const GridParams& g, uint64_t* bins) {
  GridParams b = g;
  const uint32_t groups = static_cast<uint32_t>(g.fine[0] / kTi2GroupX);
  const uint32_t bands = static_cast<uint32_t>(g.fine[1] / kTi2BandRows);
  b.axis[0].shift = 3;
  b.axis[0].bins = groups;
  b.axis[0].stride = 1;
  b.axis[1].shift = kTi2BandRows == 4 ? 2 : (kTi2BandRows == 2 ? 1 : 0);
  b.axis[1].bins = bands;
  b.axis[1].stride = groups;
  *bins = static_cast<uint64_t>(groups) * static_cast<uint64_t>(bands);
  return b;
}

int64_t tc_interp_tiles(const GridParams& g) {
  return (g.fine[0] / kTi2GroupX) * ((g.fine[1] + kTi2TileRows - 1) / kTi2TileRows);
}

int64_t tc_interp_chunk_bound(const GridParams& g, int64_t count) {
  return count / kTi2ChunkPoints + 1 + (g.fine[0] / kTi2GroupX) * (g.fine[1] / kTi2BandRows);
}

void tc_interp_prepare(const GridParams& g, const Ti2Prepare& p, cudaStream_t stream) {
  if (p.count > 0) {
    switch (g.width) {
      case 2: launch_weights<2>(g, p, stream); break;
      case 3: launch_weights<3>(g, p, stream); break;
      case 4: launch_weights<4>(g, p, stream); break;
      case 5: launch_weights<5>(g, p, stream); break;
      case 6: launch_weights<6>(g, p, stream); break;
      default: launch_weights<7>(g, p, stream); break;
    }
  }
  const unsigned blocks = static_cast<unsigned>((p.tile_count + 255) / 256);
  ti2_tile_chunks_kernel<<<blocks, 256, 0, stream>>>(g, p.tile_count, p.offsets, p.tile_chunks, p.parts);
  note_launch();
  exclusive_scan_u32(p.tile_chunks, p.tile_count, p.tile_chunk_start, stream);
  exclusive_scan_u32(p.parts, p.tile_count, p.part_start, stream);
  ti2_chunk_fill_kernel<<<blocks, 256, 0, stream>>>(g, p.tile_count, p.offsets, p.tile_chunk_start, p.chunks);
  note_launch();
}

void tc_interp_execute(const GridParams& g, const Ti2Launch& l, cudaStream_t stream) {
  const int64_t tiles = tc_interp_tiles(g);
  const int64_t stride = static_cast<int64_t>((l.batch + kTi2Vectors - 1) / kTi2Vectors) * kTi2Vectors;
  if (l.count > 0) {
    // Largest magnitude of every vector's grid: the power-of-two scales of the f16 split.
    check_cuda(cudaMemsetAsync(l.vector_max, 0, static_cast<size_t>(l.batch) * sizeof(uint32_t), stream),
               "clear vector maxima");
    const int64_t pairs = g.fine_count / 2;
    const unsigned blocks = static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>((pairs + 255) / 256, 64)));
    for (int v0 = 0; v0 < l.batch; v0 += 65535) {
      const int vectors = std::min(65535, l.batch - v0);
      ti2_vector_max_kernel<<<dim3(blocks, static_cast<unsigned>(vectors)), 256, 0, stream>>>(
          reinterpret_cast<const float4*>(l.fine) + static_cast<int64_t>(v0) * pairs, pairs, l.vector_max + v0);
      note_launch();
    }
    CUtensorMap map{};
    const bool use_map = encode_fine_map(l.fine, g.axis[0].length, g.axis[1].length, g.fine_count, l.batch, &map);
    switch (g.width) {
      case 2: launch_interp<2>(g, l, tiles, stride, map, use_map, stream); break;
      case 3: launch_interp<3>(g, l, tiles, stride, map, use_map, stream); break;
      case 4: launch_interp<4>(g, l, tiles, stride, map, use_map, stream); break;
      case 5: launch_interp<5>(g, l, tiles, stride, map, use_map, stream); break;
      case 6: launch_interp<6>(g, l, tiles, stride, map, use_map, stream); break;
      default: launch_interp<7>(g, l, tiles, stride, map, use_map, stream); break;
    }
  }
  unpermute_values(l.staged, stride, l.inverse, l.count, l.batch, l.output, stream);
}

}  // namespace b200nufft
