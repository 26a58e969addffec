// Batched 2D type-2 interpolation on the tcgen05 tensor cores.
//
// The reference interpolates every vector separately: a workgroup of lanes
// per point sums its w x w cells in lane order (src/gpu_2d.rs:1022-1113,
// workgroups over the batch at :566-575). With many vectors on one point set
// the same sums are a dense contraction, which this file runs on the tensor
// cores.
//
// Per point set (set_points): the points are ordered a second time, by the
// exact support start in bins of 8 x 1 cells (a column group of 8 cells in
// one grid row), and every point gets its window record (y weights, and x
// weights placed at their column within the 16 columns the group's windows
// reach). A tile is one column group over kTi2TileRows rows; its chunks are
// the runs of at most 32 points of one (row, group) bin, in row order.
//
// Per execution, one CTA per (tile part, 64 vectors) walks its chunks in row
// order with warp-specialised roles joined by mbarriers. A producer warp
// brings the fine-grid rows the chunks reach (16 columns x 64 vectors) into
// shared memory by bulk copies, three rows ahead; two converter warps split
// every row into tf32 high and low parts in the UMMA K-major layout (128
// rows: real and imaginary part of every vector) into a ring of w + 1 rows;
// two builder teams take alternate chunks, bulk-copy their points' window
// records and write B = wy[j] wx over the chunk's cells (zero outside each
// window); one thread issues, per chunk at row y, 2 w MMA steps (window row
// j, column half h) of M = 128, N = 16 or 32 points, K = 8 cells, A = ring
// row y + j, each split into three tf32 MMAs (A_hi B_hi + A_hi B_lo + A_lo
// B_hi), into one of four tensor-memory accumulators, and retires ring rows
// the next chunk no longer reads; four read-out warps move each accumulator
// to the values in tensor-core slot order, and a final pass writes them in
// the caller's point order. Every output comes from the MMAs of one chunk
// issued in a fixed order, so results are bitwise repeatable.
//
// Every wait is bounded: a wait that gives up stops the CTA's work, lets the
// copies and MMAs in flight finish (again with a bound), frees the tensor
// memory and increments the plan's error flag.
#include "tc_interp.h"

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
constexpr int kConvertWarp0 = 2;   // four warps: every lane converts one A row (vector part) of a fetched row
constexpr int kBuildWarp0 = 6;     // four warps: one builder team each, chunks c = team (mod 4)
constexpr int kReadWarp0 = 10;     // four warps: one per tensor-memory lane quadrant
constexpr int kThreads = 14 * 32;
constexpr int kConvertThreads = 128;
constexpr int kTeamThreads = 32;
constexpr int kReadThreads = 128;

constexpr int kBuffers = 4;            // accumulators of 32 columns (tensor-memory columns 0 .. 127)
constexpr int kRing = 12;              // converted rows in tensor memory (32 columns each, from column 128)
constexpr int kRingColumn0 = kBuffers * 32;
constexpr int kTmemColumns = 512;
static_assert(kRingColumn0 + kRing * 32 <= kTmemColumns, "tensor-memory ring exceeds the allocation");
static_assert(kRing > kTi2MaxWidth, "the ring holds a chunk's window rows and one more");
constexpr int kRawSlots = 10;          // fetched rows in flight
constexpr int kBStages = 4;            // one per builder team
constexpr int kRawPitch = 144;         // bytes per vector of a fetched row (128 + 16 against bank conflicts)
constexpr int kRawBytes = kTi2Vectors * kRawPitch;
constexpr int kWeightStage = kTi2ChunkPoints * static_cast<int>(sizeof(TcWeights));

template <int W>
struct Ti2Layout {
  static constexpr int kBHalf = kTi2ChunkPoints * kTi2Pitch * W * 4;  // one tf32 part of B: 32 x 16 W
  static constexpr int kBBase = 0;
  static constexpr int kRawBase = kBBase + kBStages * 2 * kBHalf;
  static constexpr int kWeightsBase = kRawBase + kRawSlots * kRawBytes;
  static constexpr int kBytes = kWeightsBase + kBStages * kWeightStage;
  static constexpr uint32_t kBStride = 512u * W;  // bytes between 8-point groups of B
};

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

// Chunks and parts of every tile.
__global__ void ti2_tile_chunks_kernel(GridParams g, int64_t tiles, const uint32_t* __restrict__ offsets,
                                       uint32_t* __restrict__ tile_chunks, uint32_t* __restrict__ parts) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= tiles) return;
  int tx, ty;
  tile_origin(g, t, tx, ty);
  const int n1 = g.axis[1].length;
  const int y_end = min((ty + 1) * kTi2TileRows, n1);
  const uint64_t groups = g.axis[0].bins;
  uint32_t chunks = 0;
  for (int y = ty * kTi2TileRows; y < y_end; ++y) {
    const uint64_t b = tx + groups * static_cast<uint64_t>(y);
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
  const int n1 = g.axis[1].length;
  const int y0 = ty * kTi2TileRows;
  const int y_end = min(y0 + kTi2TileRows, n1);
  const uint64_t groups = g.axis[0].bins;
  uint32_t next = tile_chunk_start[t];
  for (int y = y0; y < y_end; ++y) {
    const uint64_t b = tx + groups * static_cast<uint64_t>(y);
    const uint32_t begin = offsets[b], end = offsets[b + 1];
    for (uint32_t s = begin; s < end; s += kTi2ChunkPoints) {
      Ti2Chunk c;
      c.slot = s;
      c.count = static_cast<uint16_t>(min(static_cast<uint32_t>(kTi2ChunkPoints), end - s));
      c.row = static_cast<uint16_t>(y - y0);
      chunks[next++] = c;
    }
  }
}

// Converts A row m = 2 v + part of fetched row `raw` (vector v's 16 complex
// cells at kRawPitch) into 16 tf32 high parts followed by 16 low parts, the
// 32 columns of a ring slot (zero for vectors at or beyond nv).
__device__ __forceinline__ void ti2_convert_lane(const unsigned char* raw, int m, int nv, uint32_t* out) {
  const int v = m >> 1, part = m & 1;
  const float4* row = reinterpret_cast<const float4*>(raw + v * kRawPitch);
  float4 cells[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) cells[i] = row[i];
  const bool live = v < nv;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const float x0 = live ? (part ? cells[i].y : cells[i].x) : 0.0f;
    const float x1 = live ? (part ? cells[i].w : cells[i].z) : 0.0f;
    float hi, lo;
    split_tf32(x0, hi, lo);
    out[2 * i] = __float_as_uint(hi);
    out[16 + 2 * i] = __float_as_uint(lo);
    split_tf32(x1, hi, lo);
    out[2 * i + 1] = __float_as_uint(hi);
    out[16 + 2 * i + 1] = __float_as_uint(lo);
  }
}

template <int W>
__global__ void __launch_bounds__(kThreads, 1) tc_interp_kernel(
    GridParams g, const float2* __restrict__ fine, int batch, const TcWeights* __restrict__ weights,
    const Ti2Chunk* __restrict__ chunks, const uint32_t* __restrict__ tile_chunk_start,
    const uint32_t* __restrict__ part_start, int64_t tiles, float2* __restrict__ staged, int64_t staged_stride,
    uint32_t* __restrict__ error_flag) {
  using L = Ti2Layout<W>;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t raw_full[kRawSlots], raw_empty[kRawSlots];
  __shared__ __align__(8) uint64_t a_full[kRing], a_empty[kRing];
  __shared__ __align__(8) uint64_t b_full[kBStages], b_empty[kBStages], w_full[kBStages], w_empty[kBStages];
  __shared__ __align__(8) uint64_t d_full[kBuffers], d_empty[kBuffers];
  __shared__ uint32_t tmem_base;
  __shared__ int64_t s_tile;
  __shared__ int s_abort;
  __shared__ Ti2Chunk s_chunks[kTi2ChunksPerPart];

  const uint32_t part = blockIdx.x;
  if (part >= part_start[tiles]) return;
  const int group = blockIdx.y;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
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
    for (int s = 0; s < kBStages; ++s) {
      mbar_init(&b_full[s], kTeamThreads);
      mbar_init(&b_empty[s], 1);
      mbar_init(&w_full[s], 1);
      mbar_init(&w_empty[s], kTeamThreads);
    }
    for (int b = 0; b < kBuffers; ++b) {
      mbar_init(&d_full[b], 1);
      mbar_init(&d_empty[b], kReadThreads);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
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
  const int vb = group * kTi2Vectors;
  const int nv = min(kTi2Vectors, batch - vb);
  // Rows [r_begin, r_begin + rows) relative to y0 are fetched and converted in order.
  const int r_begin = n > 0 ? s_chunks[0].row : 0;
  const int rows = n > 0 ? s_chunks[n - 1].row + W - r_begin : 0;
  unsigned char* raw = smem + L::kRawBase;
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
      if (lane == 0) mbar_expect(bar, static_cast<uint32_t>(nv) * 128u);
      __syncwarp();
      const int y = (y0 + r_begin + k) % n1;
      const int64_t row = static_cast<int64_t>(y) * n0;
      unsigned char* dst = raw + slot * kRawBytes;
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
    bool ok = true;
    for (int c = 0; c < n && ok; ++c) {
      const Ti2Chunk ch = s_chunks[c];
      const int r = ch.row - r_begin;
      while (ok && ready < r + W) {
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
      ok = ok && mbar_wait(smem_u32(&b_full[c % kBStages]), static_cast<uint32_t>(c / kBStages) & 1u, abort_flag);
      if (ok && c >= kBuffers) {
        ok = mbar_wait(smem_u32(&d_empty[c % kBuffers]), static_cast<uint32_t>(c / kBuffers - 1) & 1u, abort_flag);
      }
      ok = __all_sync(0xFFFFFFFFu, ok);
      if (!ok) break;
      tc_fence_after();
      const int cols = ch.count <= 16 ? 16 : 32;
      const uint32_t idesc = idesc_tf32(128, static_cast<uint32_t>(cols));
      const uint32_t d = tm + static_cast<uint32_t>((c % kBuffers) * 32);
      const uint32_t bh = smem_u32(smem + L::kBBase + (c % kBStages) * 2 * L::kBHalf);
      const uint32_t bl = bh + L::kBHalf;
#pragma unroll
      for (int j = 0; j < W; ++j) {
        // Ring slot of window row j: high parts in columns 0 .. 15, low parts in 16 .. 31.
        const uint32_t a = tm + static_cast<uint32_t>(kRingColumn0 + ((r + j) % kRing) * 32);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const uint64_t bhi = kmajor_desc(bh + (4 * j + 2 * h) * 128, 128, L::kBStride);
          const uint64_t blo = kmajor_desc(bl + (4 * j + 2 * h) * 128, 128, L::kBStride);
          if (elect_one()) {
            mma_tf32_tmem_a(d, a + 8 * h, bhi, idesc, j > 0 || h > 0);
            mma_tf32_tmem_a(d, a + 8 * h, blo, idesc, true);
            mma_tf32_tmem_a(d, a + 16 + 8 * h, bhi, idesc, true);
          }
          __syncwarp();
        }
      }
      if (elect_one()) {
        mma_commit(smem_u32(&b_empty[c % kBStages]));
        mma_commit(smem_u32(&d_full[c % kBuffers]));
      }
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
      if (issued > 0 &&
          !mbar_wait(smem_u32(&d_full[(issued - 1) % kBuffers]), static_cast<uint32_t>((issued - 1) / kBuffers) & 1u,
                     nullptr)) {
        *abort_flag = 1;
      }
      if (!ok) *abort_flag = 1;
    }
  } else if (warp < kBuildWarp0) {
    // Converters: lane (warp % 4, lane) owns A row m = 32 (warp % 4) + lane
    // and writes its 32 columns of every ring slot.
    const int quadrant = warp & 3;
    const int m = quadrant * 32 + lane;
    const uint32_t lane_base = tm + (static_cast<uint32_t>(quadrant * 32) << 16);
    for (int k = 0; k < rows; ++k) {
      if (!mbar_wait(smem_u32(&raw_full[k % kRawSlots]), static_cast<uint32_t>(k / kRawSlots) & 1u, abort_flag)) break;
      uint32_t cols[32];
      ti2_convert_lane(raw + (k % kRawSlots) * kRawBytes, m, nv, cols);
      mbar_arrive(smem_u32(&raw_empty[k % kRawSlots]));
      if (k >= kRing &&
          !mbar_wait(smem_u32(&a_empty[k % kRing]), static_cast<uint32_t>(k / kRing - 1) & 1u, abort_flag)) {
        break;
      }
      tc_fence_after();
      tmem_st32(lane_base + static_cast<uint32_t>(kRingColumn0 + (k % kRing) * 32), cols);
      tmem_wait_st();
      tc_fence_before();
      mbar_arrive(smem_u32(&a_full[k % kRing]));
    }
  } else if (warp < kReadWarp0) {
    // Builder teams: team e takes chunks c = e (mod 4) into B stage e. A
    // lane holds one point's window record in registers and writes its share
    // of the window rows of that point's B column; the team's next record
    // copy is issued as soon as every lane holds its record, so it lands
    // while the team builds.
    const int team = warp - kBuildWarp0;
    unsigned char* wst = smem + L::kWeightsBase + team * kWeightStage;
    const TcWeights* s_w = reinterpret_cast<const TcWeights*>(wst);
    unsigned char* b_hi = smem + L::kBBase + team * 2 * L::kBHalf;
    unsigned char* b_lo = b_hi + L::kBHalf;
    const uint32_t wbar = smem_u32(&w_full[team]);
    int loads = 0;
    if (lane == 0 && team < n) {
      const Ti2Chunk ch = s_chunks[team];
      const uint32_t bytes = static_cast<uint32_t>(ch.count) * static_cast<uint32_t>(sizeof(TcWeights));
      mbar_expect(wbar, bytes);
      bulk_load(smem_u32(wst), weights + ch.slot, bytes, wbar);
      loads = 1;
    }
    for (int c = team; c < n; c += kBStages) {
      const Ti2Chunk ch = s_chunks[c];
      const int use = c / kBStages;
      if (!mbar_wait(wbar, static_cast<uint32_t>(use) & 1u, abort_flag)) break;
      const int shift = ch.count <= 16 ? 4 : 5;  // log2 of the B columns
      const int pn = lane & ((1 << shift) - 1);  // the lane's point (B column)
      const int share = lane >> shift, shares = 32 >> shift;
      float wy[W];
      float4 wx[4];
      if (pn < ch.count) {
#pragma unroll
        for (int j = 0; j < W; ++j) wy[j] = s_w[pn].wy[j];
#pragma unroll
        for (int q = 0; q < 4; ++q) wx[q] = *reinterpret_cast<const float4*>(&s_w[pn].wxs[4 * q]);
      } else {
#pragma unroll
        for (int j = 0; j < W; ++j) wy[j] = 0.0f;
#pragma unroll
        for (int q = 0; q < 4; ++q) wx[q] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      }
      mbar_arrive(smem_u32(&w_empty[team]));
      if (lane == 0 && c + kBStages < n) {
        // Every lane holds its record: the stage takes the next chunk's.
        if (!mbar_wait(smem_u32(&w_empty[team]), static_cast<uint32_t>(use) & 1u, abort_flag)) break;
        const Ti2Chunk nx = s_chunks[c + kBStages];
        const uint32_t bytes = static_cast<uint32_t>(nx.count) * static_cast<uint32_t>(sizeof(TcWeights));
        mbar_expect(wbar, bytes);
        bulk_load(smem_u32(wst), weights + nx.slot, bytes, wbar);
        loads = use + 2;
      }
      if (use >= 1 && !mbar_wait(smem_u32(&b_empty[team]), static_cast<uint32_t>(use - 1) & 1u, abort_flag)) break;
      const int column = (pn >> 3) * static_cast<int>(L::kBStride) + (pn & 7) * 16;
#pragma unroll
      for (int j = 0; j < W; ++j) {
        if (j % shares != share) continue;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float4 hi, lo;
          split_tf32(wy[j] * wx[q].x, hi.x, lo.x);
          split_tf32(wy[j] * wx[q].y, hi.y, lo.y);
          split_tf32(wy[j] * wx[q].z, hi.z, lo.z);
          split_tf32(wy[j] * wx[q].w, hi.w, lo.w);
          const int off = (4 * j + q) * 128 + column;
          *reinterpret_cast<float4*>(b_hi + off) = hi;
          *reinterpret_cast<float4*>(b_lo + off) = lo;
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(smem_u32(&b_full[team]));
    }
    // A weight copy in flight lands before the CTA leaves.
    if (lane == 0 && loads > 0 &&
        !mbar_wait(smem_u32(&w_full[team]), static_cast<uint32_t>(loads - 1) & 1u, nullptr)) {
      *abort_flag = 1;
    }
  } else {
    // Read-out: warp (warp % 4 = q) holds rows 32 q + lane (vector m / 2,
    // real part when m is even) of each accumulator; values go out in
    // tensor-core slot order.
    const int q = warp & 3;
    const int m = q * 32 + lane;
    const int vec = m >> 1;
    for (int c = 0; c < n; ++c) {
      if (!mbar_wait(smem_u32(&d_full[c % kBuffers]), static_cast<uint32_t>(c / kBuffers) & 1u, abort_flag)) break;
      tc_fence_after();
      const Ti2Chunk ch = s_chunks[c];
      const uint32_t addr = tm + (static_cast<uint32_t>(q * 32) << 16) + static_cast<uint32_t>((c % kBuffers) * 32);
      uint32_t v0[16], v1[16];
      tmem_ld16(addr, v0);
      if (ch.count > 16) tmem_ld16(addr + 16, v1);
      tmem_wait_ld();
      tc_fence_before();
      mbar_arrive(smem_u32(&d_empty[c % kBuffers]));
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const float x = __uint_as_float(v0[i]);
        const float y = __shfl_xor_sync(0xFFFFFFFFu, x, 1);
        if ((m & 1) == 0 && i < ch.count && vec < nv) {
          staged[(static_cast<int64_t>(ch.slot) + i) * staged_stride + vb + vec] = make_float2(x, y);
        }
      }
      if (ch.count > 16) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const float x = __uint_as_float(v1[i]);
          const float y = __shfl_xor_sync(0xFFFFFFFFu, x, 1);
          if ((m & 1) == 0 && 16 + i < ch.count && vec < nv) {
            staged[(static_cast<int64_t>(ch.slot) + 16 + i) * staged_stride + vb + vec] = make_float2(x, y);
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

template <int W>
void launch_interp(const GridParams& g, const Ti2Launch& l, int64_t tiles, int64_t stride, cudaStream_t stream) {
  using L = Ti2Layout<W>;
  static_assert(L::kBytes + 4096 <= 227 * 1024, "tensor-core interpolation stages exceed shared memory");
  auto kernel = tc_interp_kernel<W>;
  check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, L::kBytes),
             "tensor-core interpolation shared memory");
  const int groups = (l.batch + kTi2Vectors - 1) / kTi2Vectors;
  const dim3 grid(static_cast<unsigned>(l.part_upper_bound), static_cast<unsigned>(groups));
  kernel<<<grid, kThreads, L::kBytes, stream>>>(g, l.fine, l.batch, l.weights, l.chunks, l.tile_chunk_start,
                                                l.part_start, tiles, l.staged, stride, l.error_flag);
  note_launch();
}

}  // namespace

bool tc_interp_supported(const GridParams& g) {
  return g.dimensions == 2 && g.width >= 2 && g.width <= kTi2MaxWidth && g.fine[0] % kTi2GroupX == 0 &&
         g.fine[0] >= 2 * kTi2GroupX && g.fine[1] >= g.width;
}

GridParams tc_interp_bins(const GridParams& g, uint64_t* bins) {
  GridParams b = g;
  const uint32_t groups = static_cast<uint32_t>(g.fine[0] / kTi2GroupX);
  b.axis[0].shift = 3;
  b.axis[0].bins = groups;
  b.axis[0].stride = 1;
  b.axis[1].shift = 0;
  b.axis[1].bins = static_cast<uint32_t>(g.fine[1]);
  b.axis[1].stride = groups;
  *bins = static_cast<uint64_t>(groups) * static_cast<uint64_t>(g.fine[1]);
  return b;
}

int64_t tc_interp_tiles(const GridParams& g) {
  return (g.fine[0] / kTi2GroupX) * ((g.fine[1] + kTi2TileRows - 1) / kTi2TileRows);
}

int64_t tc_interp_chunk_bound(const GridParams& g, int64_t count) {
  return count / kTi2ChunkPoints + 1 + (g.fine[0] / kTi2GroupX) * g.fine[1];
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
    switch (g.width) {
      case 2: launch_interp<2>(g, l, tiles, stride, stream); break;
      case 3: launch_interp<3>(g, l, tiles, stride, stream); break;
      case 4: launch_interp<4>(g, l, tiles, stride, stream); break;
      case 5: launch_interp<5>(g, l, tiles, stride, stream); break;
      case 6: launch_interp<6>(g, l, tiles, stride, stream); break;
      default: launch_interp<7>(g, l, tiles, stride, stream); break;
    }
  }
  unpermute_values(l.staged, stride, l.inverse, l.count, l.batch, l.output, stream);
}

}  // namespace b200nufft
