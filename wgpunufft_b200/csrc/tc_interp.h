// Batched 2D type-2 interpolation on the tcgen05 tensor cores (tc_interp.cu).
//
// When many coefficient vectors share one point set, interpolating the
// points whose support starts in one band of 4 rows of an 8-cell column group
// is a dense contraction: the fine-grid values of 64 vectors over the w + 3
// window rows of the band and 16 columns of the group (128 rows: real and
// imaginary parts; K = 16 cells per row) times each point's separable window
// weights over the same cells (N = the points, zero outside each window).
// Such a group of points is a chunk of at most 128 points; it is w + 3 MMA
// steps of M = 128, N = 16 .. 128, K = 16, each split into 3 f16 MMAs
// (hi*hi + hi*lo + lo*hi of power-of-two-scaled values) that keep FP32
// accuracy, in a fixed order, so results are bitwise repeatable.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "device.h"
#include "tc_spread.h"

namespace b200nufft {

constexpr int kTi2Vectors = 64;        // vectors per CTA (M = 128 rows)
constexpr int kTi2ChunkPoints = 128;   // points per chunk at most (N = 16 .. 128)
constexpr int kTi2GroupX = 8;          // cells per column group (chunk starts)
constexpr int kTi2Pitch = 16;          // region columns per window row (K per row)
constexpr int kTi2MaxWidth = 7;        // widest window
constexpr int kTi2BandRows = 4;        // rows of one chunk band (support starts): 1, 2 or 4
constexpr int kTi2TileRows = 128;      // rows of one tile (a multiple of the band rows)
static_assert(kTi2BandRows == 1 || kTi2BandRows == 2 || kTi2BandRows == 4, "bands of 1, 2 or 4 rows");
constexpr int kTi2ChunksPerPart = 256; // chunks per CTA at most

// One chunk: up to 128 consecutive slots of one (band, column group) bin.
struct Ti2Chunk {
  uint32_t slot;
  uint16_t count;
  uint16_t row;  // first row of the band relative to the tile's first row
};

// Whether a plan of this fine grid and window can interpolate on the tensor cores.
bool tc_interp_supported(const GridParams& g);

// The bin geometry of the tensor-core order: bins of 8 x 4 cells keyed by
// the exact support start (a copy of `g` with those shifts and strides).
GridParams tc_interp_bins(const GridParams& g, uint64_t* bins);

struct Ti2Prepare {
  const float* points;       // caller's coordinates (point-major)
  int64_t count;
  const uint32_t* perm;      // tensor-core slot -> original point
  const uint32_t* offsets;   // bins + 1 slot offsets of the tensor-core order
  TcWeights* weights;        // per slot
  uint32_t* inverse;         // original point -> slot
  int64_t tile_count;
  uint32_t* tile_chunks;     // tile_count words
  uint32_t* tile_chunk_start;// tile_count + 1 words
  Ti2Chunk* chunks;
  uint32_t* parts;           // tile_count words
  uint32_t* part_start;      // tile_count + 1 words
};
int64_t tc_interp_tiles(const GridParams& g);
int64_t tc_interp_chunk_bound(const GridParams& g, int64_t count);
void tc_interp_prepare(const GridParams& g, const Ti2Prepare& p, cudaStream_t stream);

struct Ti2Launch {
  const float2* fine;        // batch x fine_count
  int batch;
  int64_t count;
  const TcWeights* weights;
  const Ti2Chunk* chunks;
  const uint32_t* tile_chunk_start;
  const uint32_t* part_start;
  int64_t part_upper_bound;
  const uint32_t* inverse;
  float2* staged;            // count x groups x 64 values, tensor-core slot order
  float2* output;            // batch x count, caller's point order
  uint32_t* vector_max;      // batch words of scratch: largest |re|, |im| of every vector's fine grid
  uint32_t* error_flag;      // incremented when a wait gives up
};
void tc_interp_execute(const GridParams& g, const Ti2Launch& l, cudaStream_t stream);

}  // namespace b200nufft
