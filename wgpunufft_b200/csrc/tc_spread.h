// Batched 2D type-1 spreading on the tcgen05 tensor cores (tc_spread.cu).
//
// When many strength vectors share one point set, spreading one tile of the
// fine grid is a dense contraction: the strengths of 64 vectors (128 rows:
// real and imaginary parts) times the separable window weights of the
// tile's points. Tiles are 8 cells wide and padded rows are 16 columns apart
// in tensor memory, so the w window rows of points starting in one bin row
// are one contiguous run of 16 w accumulator columns. Points are taken eight
// at a time (one tf32 MMA of K = 8): a chunk holds up to eight points of one
// bin row of a tile and is one MMA of M = 128, N = 16 w, K = 8 into the
// padded-tile accumulator held in tensor memory. Each product is split into
// 3 tf32 MMAs (hi*hi + hi*lo + lo*hi) to keep FP32 accuracy; the MMA order is
// fixed, so results are bitwise repeatable.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device.h"
#include "spread.h"

namespace b200nufft {

constexpr int kTcVectors = 64;        // strength vectors per CTA (M = 128 rows)
constexpr int kTcRows = 2 * kTcVectors;
constexpr int kTcChunkPoints = 8;     // points per chunk: the K of one tf32 MMA
constexpr int kTcChunksPerPart = 256; // chunks per CTA at most
constexpr int kTcPitch = 16;          // tensor-memory columns per padded tile row
constexpr int kTcTileX = 8;           // tile width in cells (one column group)
constexpr int kTcMaxWidth = 8;        // widest window (weights stored per point)
constexpr int kTcMinBatch = 16;       // active batches below this use the CUDA-core spreader
constexpr int kTcColumns = 256;       // tensor-memory columns a CTA allocates (two CTAs per SM)

// One chunk: up to eight consecutive slots of one bin row of a tile.
struct TcChunk {
  uint32_t slot;
  uint16_t count;
  uint8_t row0;  // padded-tile row of the bin row
  uint8_t x0;    // padded-tile column of the column group
};

// The window of one point in slot order: its wrapped support start, its y
// weights, and its x weights placed at their padded-tile columns
// (wxs[c] = wx[c - sx mod 8]); zero for points outside the fold reach.
struct __align__(16) TcWeights {
  int32_t sx, sy;
  int32_t unused[2];
  float wy[kTcMaxWidth];
  float wxs[2 * kTcTileX];
};
static_assert(sizeof(TcWeights) == 112, "TcWeights is copied in 16-byte units");

// Tile rows of the tensor-core geometry for window width w.
inline int tc_tile_rows(int width) { return kTcColumns / kTcPitch - width + 1; }

// Upper bound on the chunks of a point set of `count` points.
int64_t tc_chunk_bound(const SpreadParams& sp, int64_t count);

// Prepared per point set: window records in slot order, the slot of every
// point, chunk tables, and the parts of every tile (tile_count + 1 words of
// part_start).
struct TcPrepare {
  const float* sorted_points;
  int64_t count;
  const uint32_t* perm;
  const uint32_t* offsets;
  TcWeights* weights;
  uint32_t* inverse;
  uint32_t* tile_chunks;       // tile_count words
  uint32_t* tile_chunk_start;  // tile_count + 1 words
  TcChunk* chunks;
  uint32_t* parts;             // tile_count words
  uint32_t* part_start;        // tile_count + 1 words
};
void tc_prepare(const SpreadParams& sp, const TcPrepare& p, cudaStream_t stream, StageTimer* timer);

struct TcLaunch {
  const float2* strengths;  // batch x count, caller order
  int64_t count;
  int batch;
  const uint32_t* inverse;
  const TcWeights* weights;
  const TcChunk* chunks;
  const uint32_t* tile_chunk_start;
  const uint32_t* part_start;
  int64_t part_upper_bound;
  float* packed;            // groups x count x 128 floats
  float2* scratch;          // part_upper_bound x padded_cells x groups x 64 complex values
  const int2* candidates;
  float2* fine;
  uint32_t* error_flag;     // incremented when a tensor-core wait gives up
};
// Spreads `batch` vectors onto `fine` (every cell written).
void tc_spread_execute(const SpreadParams& sp, const TcLaunch& l, cudaStream_t stream, StageTimer* timer);

}  // namespace b200nufft
