// Batched 2D type-1 spreading on the tcgen05 tensor cores.
//
// Per point set (set_points): the window of every point in slot order
// (support start and w weights per axis), the slot of every original index,
// and a table of chunks: up to eight consecutive slots of one bin row of a
// tile. Tiles are 8 cells wide and 17 - w rows high, so that a padded tile
// ((8 + w - 1) x 16 cells at a row pitch of 16 columns) fits 256
// tensor-memory columns: two CTAs share an SM, so one CTA's setup and
// read-out overlap the other's MMAs.
//
// Per execution: the strengths of 64 vectors are packed point-major in slot
// order (128 floats per point: real and imaginary parts interleaved), so a
// chunk's strengths are one contiguous 4 KB block. One CTA per (tile part,
// group of 64 vectors) streams its chunks through a 4-stage pipeline: a bulk
// copy brings the chunk's packed strengths and windows into shared memory,
// 256 threads split them into tf32 high and low parts in the UMMA K-major
// layout (A: 128 rows x 8 points; B: 16 w accumulator columns x 8 points,
// the w window rows of the chunk one after another), and one thread issues
// three MMAs of M = 128, N = 16 w, K = 8 (A_hi B_hi + A_hi B_lo + A_lo B_hi)
// into the accumulator columns of the chunk's bin row. The accumulator starts at zero and is
// written to the padded-tile scratch at the end; the fold pass then sums the
// padded tiles per fine-grid cell in a fixed order. MMAs complete in issue
// order, so results are bitwise repeatable.
//
// Every wait on an mbarrier is bounded; a wait that gives up raises the
// plan's error flag, lets the copies and MMAs in flight finish (again with a
// bound), frees the tensor memory and leaves the CTA.
#include "tc_spread.h"

#include <algorithm>

#include "tc_common.cuh"

namespace b200nufft {

namespace {

using namespace tc;

// Instruction descriptor of the spread MMAs: M = 128, N = 16 w.
template <int W>
__host__ __device__ constexpr uint32_t tc_idesc() {
  return idesc_tf32(128, 16 * W);
}

constexpr int kTcTeams = 4;          // converter teams, each converting every fourth chunk
constexpr int kTcTeamThreads = 64;
constexpr int kTcThreads = 64 + kTcTeams * kTcTeamThreads;  // producer warp, MMA warp, converters
constexpr int kTcCopyStages = 8;     // chunks whose copies are in flight or unread
constexpr int kTcOperandStages = 4;  // chunks whose MMAs may still read their operands
constexpr size_t kTcSharedBytes = 108 * 1024;  // two CTAs per SM, 256 tensor-memory columns each

// Window records in slot order and the slot of every original index.
template <int W>
__global__ void tc_weights_kernel(GridParams g, const float* __restrict__ sorted, int64_t count,
                                  const uint32_t* __restrict__ perm, TcWeights* __restrict__ out,
                                  uint32_t* __restrict__ inverse) {
  const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= count) return;
  TcWeights r;
  r.sx = r.sy = 0;
  r.unused[0] = r.unused[1] = 0;
#pragma unroll
  for (int j = 0; j < kTcMaxWidth; ++j) r.wy[j] = 0.0f;
#pragma unroll
  for (int c = 0; c < 2 * kTcTileX; ++c) r.wxs[c] = 0.0f;
  const float x = sorted[2 * s], y = sorted[2 * s + 1];
  if (in_fold_reach(x) && in_fold_reach(y)) {
    float wx[W], wy[W];
    f32_window<W>(x, g.axis[0], g.half_width, g.beta, r.sx, wx);
    f32_window<W>(y, g.axis[1], g.half_width, g.beta, r.sy, wy);
    // Tiles start at multiples of 8 cells: the column of the first weight.
    const int dx = r.sx & (kTcTileX - 1);
#pragma unroll
    for (int j = 0; j < W; ++j) {
      r.wy[j] = wy[j];
#pragma unroll
      for (int d = 0; d < kTcTileX; ++d) {
        if (d == dx) r.wxs[d + j] = wx[j];
      }
    }
  }
  out[s] = r;
  inverse[perm[s]] = static_cast<uint32_t>(s);
}

// Chunks of every tile (one-cell bin rows, column groups of 8 cells).
__global__ void tc_tile_chunks_kernel(SpreadParams sp, const uint32_t* __restrict__ offsets,
                                      uint32_t* __restrict__ tile_chunks, uint32_t* __restrict__ parts) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= sp.tile_count) return;
  const int ox = static_cast<int>(t % sp.ntiles[0]) * sp.tile[0];
  const int oy = static_cast<int>(t / sp.ntiles[0]) * sp.tile[1];
  const int fine0 = static_cast<int>(sp.grid.fine[0]);
  const int y_end = min(oy + sp.tile[1], static_cast<int>(sp.grid.fine[1]));
  const int shift = sp.grid.axis[0].shift;
  const uint64_t bins0 = sp.grid.axis[0].bins;
  uint32_t chunks = 0;
  for (int y = oy; y < y_end; ++y) {
    const uint64_t row = bins0 * static_cast<uint64_t>(y);
    for (int gx = 0; gx < kTcTileX; gx += 8) {
      const int x_lo = ox + gx;
      if (x_lo >= fine0) break;
      const int x_hi = min(x_lo + 8, fine0) - 1;
      const uint32_t n = offsets[row + (x_hi >> shift) + 1] - offsets[row + (x_lo >> shift)];
      chunks += (n + kTcChunkPoints - 1) / kTcChunkPoints;
    }
  }
  tile_chunks[t] = chunks;
  parts[t] = (chunks + kTcChunksPerPart - 1) / kTcChunksPerPart;
}

__global__ void tc_chunk_fill_kernel(SpreadParams sp, const uint32_t* __restrict__ offsets,
                                     const uint32_t* __restrict__ tile_chunk_start,
                                     TcChunk* __restrict__ chunks) {
  const int64_t t = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (t >= sp.tile_count) return;
  const int ox = static_cast<int>(t % sp.ntiles[0]) * sp.tile[0];
  const int oy = static_cast<int>(t / sp.ntiles[0]) * sp.tile[1];
  const int fine0 = static_cast<int>(sp.grid.fine[0]);
  const int y_end = min(oy + sp.tile[1], static_cast<int>(sp.grid.fine[1]));
  const int shift = sp.grid.axis[0].shift;
  const uint64_t bins0 = sp.grid.axis[0].bins;
  uint32_t next = tile_chunk_start[t];
  for (int y = oy; y < y_end; ++y) {
    const uint64_t row = bins0 * static_cast<uint64_t>(y);
    for (int gx = 0; gx < kTcTileX; gx += 8) {
      const int x_lo = ox + gx;
      if (x_lo >= fine0) break;
      const int x_hi = min(x_lo + 8, fine0) - 1;
      const uint32_t begin = offsets[row + (x_lo >> shift)];
      const uint32_t end = offsets[row + (x_hi >> shift) + 1];
      for (uint32_t s = begin; s < end; s += kTcChunkPoints) {
        TcChunk c;
        c.slot = s;
        c.count = static_cast<uint16_t>(min(static_cast<uint32_t>(kTcChunkPoints), end - s));
        c.row0 = static_cast<uint8_t>(y - oy);
        c.x0 = static_cast<uint8_t>(gx);
        chunks[next++] = c;
      }
    }
  }
}

// Strengths of 64 vectors per group, point-major in slot order: 128 floats
// (re, im of each vector) per point; vectors beyond the batch are zero.
__global__ void __launch_bounds__(256) tc_pack_kernel(const float2* __restrict__ strengths, int64_t count,
                                                      int batch, const uint32_t* __restrict__ inverse,
                                                      float* __restrict__ packed) {
  __shared__ __align__(16) float tile[64][kTcRows + 4];
  const int64_t i0 = static_cast<int64_t>(blockIdx.x) * 64;
  const int group = blockIdx.y;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    const int bl = warp * 8 + v;
    const int b = group * kTcVectors + bl;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int p = h * 32 + lane;
      const int64_t i = i0 + p;
      float2 s = make_float2(0.0f, 0.0f);
      if (b < batch && i < count) s = strengths[static_cast<int64_t>(b) * count + i];
      tile[p][2 * bl] = s.x;
      tile[p][2 * bl + 1] = s.y;
    }
  }
  __syncthreads();
  for (int p = warp; p < 64; p += 8) {
    const int64_t i = i0 + p;
    if (i >= count) break;
    const uint32_t slot = inverse[i];
    const float4 v = *reinterpret_cast<const float4*>(&tile[p][4 * lane]);
    *reinterpret_cast<float4*>(packed + (static_cast<int64_t>(group) * count + slot) * kTcRows + 4 * lane) = v;
  }
}

template <int W>
struct TcLayout {
  // Copy ring (kTcCopyStages): a chunk's packed strengths and windows.
  static constexpr int kRawC = 0;      // 8 points x 128 floats
  static constexpr int kRawW = 4096;   // 8 window records
  static constexpr int kCopyStage = 5120;
  // Operand ring (kTcOperandStages): tf32 splits in the UMMA K-major layout.
  static constexpr int kAHi = 0;       // 128 x 8
  static constexpr int kALo = 4096;
  static constexpr int kBHi = 8192;    // 16 W x 8
  static constexpr int kBLo = kBHi + W * 512;
  static constexpr int kOperandStage = (kBLo + W * 512 + 1023) / 1024 * 1024;
  static constexpr int kOperandBase = kTcCopyStages * kCopyStage;
  static constexpr int kBytes = kOperandBase + kTcOperandStages * kOperandStage;
  static constexpr int kPadX = kTcTileX + W - 1;
};

// Converts chunk `ch` from its copy stage into its operand stage with the
// kTcTeamThreads threads of one team (t = thread index in the team).
template <int W>
__device__ __forceinline__ void tc_convert(const TcChunk& ch, const unsigned char* raw, unsigned char* op, int t) {
  using L = TcLayout<W>;
  const int cnt = ch.count;
  const float* raw_c = reinterpret_cast<const float*>(raw + L::kRawC);
  const TcWeights* raw_w = reinterpret_cast<const TcWeights*>(raw + L::kRawW);
  // A: row m, points 4h .. 4h + 3 (256 units).
#pragma unroll
  for (int i = 0; i < 256 / kTcTeamThreads; ++i) {
    const int u = t + i * kTcTeamThreads;
    const int m = u & (kTcRows - 1), h = u >> 7;
    float v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int k = 4 * h + q;
      v[q] = k < cnt ? raw_c[k * kTcRows + m] : 0.0f;
    }
    float4 hi, lo;
    split_tf32(v[0], hi.x, lo.x);
    split_tf32(v[1], hi.y, lo.y);
    split_tf32(v[2], hi.z, lo.z);
    split_tf32(v[3], hi.w, lo.w);
    const int off = kmajor_unit(m, h);
    *reinterpret_cast<float4*>(op + L::kAHi + off) = hi;
    *reinterpret_cast<float4*>(op + L::kALo + off) = lo;
  }
  // B: accumulator column 16 j + nn (window row j, padded column nn), points
  // 4h .. 4h + 3 (32 W units).
#pragma unroll
  for (int i = 0; i < (32 * W + kTcTeamThreads - 1) / kTcTeamThreads; ++i) {
    const int u = t + i * kTcTeamThreads;
    if (u < 32 * W) {
      const int j = u >> 5, nn = (u >> 1) & 15, h = u & 1;
      float v[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int k = 4 * h + q;
        v[q] = k < cnt ? raw_w[k].wy[j] * raw_w[k].wxs[nn] : 0.0f;
      }
      float4 hi, lo;
      split_tf32(v[0], hi.x, lo.x);
      split_tf32(v[1], hi.y, lo.y);
      split_tf32(v[2], hi.z, lo.z);
      split_tf32(v[3], hi.w, lo.w);
      const int off = j * 512 + kmajor_unit(nn, h);
      *reinterpret_cast<float4*>(op + L::kBHi + off) = hi;
      *reinterpret_cast<float4*>(op + L::kBLo + off) = lo;
    }
  }
}

// Warp roles: warp 0 issues the bulk copies, warp 1 issues the MMAs, and
// warps 2 .. 9 convert: four teams of two warps, team t taking chunks
// c = t (mod 4). Barriers: full (copy landed), copy_free (copy read),
// op_full (operands written), op_empty (MMAs done with the operands).
template <int W>
__global__ void __launch_bounds__(kTcThreads, 2) tc_spread_kernel(
    SpreadParams sp, const float* __restrict__ packed, int64_t count, const TcWeights* __restrict__ weights,
    const TcChunk* __restrict__ chunks, const uint32_t* __restrict__ tile_chunk_start,
    const uint32_t* __restrict__ part_start, int groups, float* __restrict__ scratch,
    uint32_t* __restrict__ error_flag) {
  using L = TcLayout<W>;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t full_bar[kTcCopyStages];
  __shared__ __align__(8) uint64_t copy_free_bar[kTcCopyStages];
  __shared__ __align__(8) uint64_t op_full_bar[kTcOperandStages];
  __shared__ __align__(8) uint64_t op_empty_bar[kTcOperandStages];
  __shared__ uint32_t tmem_base;
  __shared__ int64_t s_tile;
  __shared__ int s_abort;
  __shared__ TcChunk s_chunks[kTcChunksPerPart];

  const uint32_t part = blockIdx.x;
  const int group = blockIdx.y;
  if (part >= part_start[sp.tile_count]) return;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) {
    int64_t low = 0, high = sp.tile_count - 1;
    while (low < high) {
      const int64_t mid = (low + high + 1) >> 1;
      if (part_start[mid] <= part) low = mid; else high = mid - 1;
    }
    s_tile = low;
    s_abort = 0;
#pragma unroll
    for (int s = 0; s < kTcCopyStages; ++s) {
      mbar_init(&full_bar[s], 1);
      mbar_init(&copy_free_bar[s], kTcTeamThreads);
    }
#pragma unroll
    for (int s = 0; s < kTcOperandStages; ++s) {
      mbar_init(&op_full_bar[s], kTcTeamThreads);
      mbar_init(&op_empty_bar[s], 1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(kTcColumns));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tm = tmem_base;
  const int64_t tile = s_tile;
  const uint32_t first = tile_chunk_start[tile] + (part - part_start[tile]) * kTcChunksPerPart;
  const uint32_t stop = min(first + static_cast<uint32_t>(kTcChunksPerPart), tile_chunk_start[tile + 1]);
  const int n = stop > first ? static_cast<int>(stop - first) : 0;
  for (int c = tid; c < n; c += kTcThreads) s_chunks[c] = chunks[first + c];

  // Zero the accumulator: the eight converter warps, two per lane quadrant,
  // clear half of the columns each.
  if (warp >= 2) {
    const int cw = warp - 2;
    constexpr int kHalf = kTcColumns / 2;
    const uint32_t base = tm + (static_cast<uint32_t>((warp & 3) * 32) << 16) + static_cast<uint32_t>((cw >> 2) * kHalf);
    for (int c = 0; c < kHalf; c += 8) tmem_zero8(base + c);
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();

  volatile int* abort_flag = &s_abort;
  int issued_copies = 0;
  int issued_mmas = 0;
  if (warp == 0) {
    if (lane == 0) {
      // Producer: chunk c reuses the copy stage of chunk c - kTcCopyStages once it has been read.
      const float* packed_group = packed + static_cast<int64_t>(group) * count * kTcRows;
      for (int c = 0; c < n; ++c) {
        const int cs = c % kTcCopyStages;
        if (c >= kTcCopyStages &&
            !mbar_wait(smem_u32(&copy_free_bar[cs]), static_cast<uint32_t>(c / kTcCopyStages - 1) & 1u, abort_flag)) {
          break;
        }
        const TcChunk ch = s_chunks[c];
        unsigned char* st = smem + cs * L::kCopyStage;
        const uint32_t bar = smem_u32(&full_bar[cs]);
        const uint32_t cbytes = static_cast<uint32_t>(ch.count) * kTcRows * 4u;
        const uint32_t wbytes = static_cast<uint32_t>(ch.count) * static_cast<uint32_t>(sizeof(TcWeights));
        mbar_expect(bar, cbytes + wbytes);
        bulk_load(smem_u32(st + L::kRawC), packed_group + static_cast<int64_t>(ch.slot) * kTcRows, cbytes, bar);
        bulk_load(smem_u32(st + L::kRawW), weights + ch.slot, wbytes, bar);
        issued_copies = c + 1;
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer: chunks in order, so the accumulation order is fixed.
      constexpr uint32_t idesc = tc_idesc<W>();
      for (int c = 0; c < n; ++c) {
        const int os = c % kTcOperandStages;
        if (!mbar_wait(smem_u32(&op_full_bar[os]), static_cast<uint32_t>(c / kTcOperandStages) & 1u, abort_flag)) {
          break;
        }
        tc_fence_after();
        const unsigned char* op = smem + L::kOperandBase + os * L::kOperandStage;
        const uint64_t ahi = kmajor_desc(smem_u32(op + L::kAHi));
        const uint64_t alo = kmajor_desc(smem_u32(op + L::kALo));
        const uint64_t bhi = kmajor_desc(smem_u32(op + L::kBHi));
        const uint64_t blo = kmajor_desc(smem_u32(op + L::kBLo));
        const uint32_t d = tm + static_cast<uint32_t>(s_chunks[c].row0 * kTcPitch);
        mma_tf32(d, ahi, bhi, idesc);
        mma_tf32(d, ahi, blo, idesc);
        mma_tf32(d, alo, bhi, idesc);
        mma_commit(smem_u32(&op_empty_bar[os]));
        issued_mmas = c + 1;
      }
    }
  } else {
    // Converters.
    const int team = (warp - 2) >> 1, t = tid - 64 - team * kTcTeamThreads;
    for (int c = team; c < n; c += kTcTeams) {
      const int cs = c % kTcCopyStages, os = c % kTcOperandStages;
      if (!mbar_wait(smem_u32(&full_bar[cs]), static_cast<uint32_t>(c / kTcCopyStages) & 1u, abort_flag)) break;
      if (c >= kTcOperandStages &&
          !mbar_wait(smem_u32(&op_empty_bar[os]), static_cast<uint32_t>(c / kTcOperandStages - 1) & 1u, abort_flag)) {
        break;
      }
      tc_convert<W>(s_chunks[c], smem + cs * L::kCopyStage, smem + L::kOperandBase + os * L::kOperandStage, t);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(smem_u32(&op_full_bar[os]));
      mbar_arrive(smem_u32(&copy_free_bar[cs]));
    }
  }

  // Drain: the producer waits for the copies it issued to land, the MMA
  // issuer for its last commit (which covers every MMA before it).
  bool drained = true;
  if (warp == 0 && lane == 0) {
    for (int c = max(0, issued_copies - kTcCopyStages); c < issued_copies; ++c) {
      drained = mbar_wait(smem_u32(&full_bar[c % kTcCopyStages]), static_cast<uint32_t>(c / kTcCopyStages) & 1u,
                          nullptr) && drained;
    }
  }
  if (warp == 1 && lane == 0 && issued_mmas > 0) {
    drained = mbar_wait(smem_u32(&op_empty_bar[(issued_mmas - 1) % kTcOperandStages]),
                        static_cast<uint32_t>((issued_mmas - 1) / kTcOperandStages) & 1u, nullptr);
    if (issued_mmas < n) drained = false;
  }
  if (!drained) *abort_flag = 1;
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const bool good = *abort_flag == 0;
  if (warp >= 2) {
    // Accumulator row m = 32 (w % 4) + lane (vector m / 2, real part when m
    // is even) goes to scratch[part][cell][group][m]: a warp stores 128
    // contiguous bytes per cell.
    const int q = warp & 3, half = (warp - 2) >> 2;
    const int m = q * 32 + lane;
    const int pad_y = sp.pad[1];
    const int rows_half = (pad_y + 1) / 2;
    const int r_begin = half * rows_half, r_end = min(pad_y, r_begin + rows_half);
    const int64_t cell_stride = static_cast<int64_t>(groups) * kTcRows;
    float* out = scratch + (static_cast<int64_t>(part) * sp.padded_cells * groups + group) * kTcRows + m;
    const uint32_t lane_base = tm + (static_cast<uint32_t>(q * 32) << 16);
    for (int r = r_begin; r < r_end; ++r) {
      uint32_t v[kTcPitch];
      const uint32_t addr = lane_base + static_cast<uint32_t>(r * kTcPitch);
      tmem_ld8(addr, v);
      tmem_ld8(addr + 8, v + 8);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (good) {
#pragma unroll
        for (int x = 0; x < L::kPadX; ++x) out[(r * L::kPadX + x) * cell_stride] = __uint_as_float(v[x]);
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tm), "r"(kTcColumns));
  }
  if (tid == 0 && !good) atomicAdd(error_flag, 1u);
}

// Every fine-grid cell of 8 consecutive vectors as the fixed-order sum of
// the padded tiles and parts that cover it (the order of fold_tiles_kernel).
__global__ void __launch_bounds__(256) tc_fold_kernel(SpreadParams sp, int batch, int groups,
                                                      const float* __restrict__ scratch,
                                                      const uint32_t* __restrict__ part_start, int64_t part_limit,
                                                      const int2* __restrict__ candidates,
                                                      float2* __restrict__ fine) {
  const int64_t cell = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (cell >= sp.grid.fine_count) return;
  const int b0 = blockIdx.y * 8;
  const int group = b0 / kTcVectors;
  const int row0 = 2 * (b0 % kTcVectors);
  const int x = static_cast<int>(cell % sp.grid.fine[0]);
  const int y = static_cast<int>(cell / sp.grid.fine[0]);
  const int2* c0 = candidates + sp.candidate_base[0] + static_cast<int64_t>(x) * sp.candidate_count[0];
  const int2* c1 = candidates + sp.candidate_base[1] + static_cast<int64_t>(y) * sp.candidate_count[1];
  float4 sum[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) sum[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  for (int k1 = 0; k1 < sp.candidate_count[1]; ++k1) {
    const int2 e1 = c1[k1];
    if (e1.x < 0) break;
    for (int k0 = 0; k0 < sp.candidate_count[0]; ++k0) {
      const int2 e0 = c0[k0];
      if (e0.x < 0) break;
      const int64_t tile = e0.x + static_cast<int64_t>(sp.ntiles[0]) * e1.x;
      const int local = e0.y + sp.pad[0] * e1.y;
      const uint32_t p_first = part_start[tile];
      const uint32_t p_last = min(part_start[tile + 1], static_cast<uint32_t>(part_limit));
      for (uint32_t p = p_first; p < p_last; ++p) {
        const float4* v = reinterpret_cast<const float4*>(
            scratch + ((static_cast<int64_t>(p) * sp.padded_cells + local) * groups + group) * kTcRows + row0);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const float4 a = v[i];
          sum[i].x += a.x;
          sum[i].y += a.y;
          sum[i].z += a.z;
          sum[i].w += a.w;
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int b = b0 + 2 * i;
    if (b < batch) fine[static_cast<int64_t>(b) * sp.grid.fine_count + cell] = make_float2(sum[i].x, sum[i].y);
    if (b + 1 < batch) fine[static_cast<int64_t>(b + 1) * sp.grid.fine_count + cell] = make_float2(sum[i].z, sum[i].w);
  }
}

template <int W>
void launch_tc_width(const SpreadParams& sp, const TcLaunch& l, cudaStream_t stream) {
  static_assert(TcLayout<W>::kBytes <= static_cast<int>(kTcSharedBytes), "stages exceed shared memory");
  static_assert(TcLayout<W>::kPadX <= kTcPitch, "padded tile row exceeds the accumulator pitch");
  auto kernel = tc_spread_kernel<W>;
  check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(kTcSharedBytes)),
             "tensor-core spread shared memory");
  const int groups = (l.batch + kTcVectors - 1) / kTcVectors;
  const dim3 grid(static_cast<unsigned>(l.part_upper_bound), static_cast<unsigned>(groups));
  kernel<<<grid, kTcThreads, kTcSharedBytes, stream>>>(sp, l.packed, l.count, l.weights, l.chunks,
                                                        l.tile_chunk_start, l.part_start, groups,
                                                        reinterpret_cast<float*>(l.scratch), l.error_flag);
  note_launch();
}

template <int W>
void launch_tc_weights(const SpreadParams& sp, const TcPrepare& p, cudaStream_t stream) {
  const unsigned blocks = static_cast<unsigned>((p.count + 255) / 256);
  tc_weights_kernel<W><<<blocks, 256, 0, stream>>>(sp.grid, p.sorted_points, p.count, p.perm, p.weights,
                                                   p.inverse);
  note_launch();
}

}  // namespace

int64_t tc_chunk_bound(const SpreadParams& sp, int64_t count) {
  return count / kTcChunkPoints + 1 + sp.tile_count * static_cast<int64_t>(sp.tile[1]) * (kTcTileX / 8);
}

void tc_prepare(const SpreadParams& sp, const TcPrepare& p, cudaStream_t stream, StageTimer* timer) {
  StageScope scope(timer, kStageTileParts, stream);
  if (p.count > 0) {
    switch (sp.grid.width) {
      case 2: launch_tc_weights<2>(sp, p, stream); break;
      case 3: launch_tc_weights<3>(sp, p, stream); break;
      case 4: launch_tc_weights<4>(sp, p, stream); break;
      case 5: launch_tc_weights<5>(sp, p, stream); break;
      case 6: launch_tc_weights<6>(sp, p, stream); break;
      case 7: launch_tc_weights<7>(sp, p, stream); break;
      default: launch_tc_weights<8>(sp, p, stream); break;
    }
  }
  const unsigned blocks = static_cast<unsigned>((sp.tile_count + 255) / 256);
  tc_tile_chunks_kernel<<<blocks, 256, 0, stream>>>(sp, p.offsets, p.tile_chunks, p.parts);
  note_launch();
  exclusive_scan_u32(p.tile_chunks, sp.tile_count, p.tile_chunk_start, stream);
  exclusive_scan_u32(p.parts, sp.tile_count, p.part_start, stream);
  tc_chunk_fill_kernel<<<blocks, 256, 0, stream>>>(sp, p.offsets, p.tile_chunk_start, p.chunks);
  note_launch();
}

void tc_spread_execute(const SpreadParams& sp, const TcLaunch& l, cudaStream_t stream, StageTimer* timer) {
  const int groups = (l.batch + kTcVectors - 1) / kTcVectors;
  {
    StageScope scope(timer, kStageStrengthScale, stream);
    const dim3 grid(static_cast<unsigned>((l.count + 63) / 64), static_cast<unsigned>(groups));
    tc_pack_kernel<<<grid, 256, 0, stream>>>(l.strengths, l.count, l.batch, l.inverse, l.packed);
    note_launch();
  }
  {
    StageScope scope(timer, kStageSpread, stream);
    switch (sp.grid.width) {
      case 2: launch_tc_width<2>(sp, l, stream); break;
      case 3: launch_tc_width<3>(sp, l, stream); break;
      case 4: launch_tc_width<4>(sp, l, stream); break;
      case 5: launch_tc_width<5>(sp, l, stream); break;
      case 6: launch_tc_width<6>(sp, l, stream); break;
      case 7: launch_tc_width<7>(sp, l, stream); break;
      default: launch_tc_width<8>(sp, l, stream); break;
    }
  }
  StageScope scope(timer, kStageFold, stream);
  const dim3 grid(static_cast<unsigned>((sp.grid.fine_count + 255) / 256), static_cast<unsigned>((l.batch + 7) / 8));
  tc_fold_kernel<<<grid, 256, 0, stream>>>(sp, l.batch, groups, reinterpret_cast<const float*>(l.scratch),
                                           l.part_start, l.part_upper_bound, l.candidates, l.fine);
  note_launch();
}

}  // namespace b200nufft
