// Device memory, launch accounting and the parameter blocks that the host
// passes to the kernels.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <string>

#include "es_kernel.h"
#include "fold.cuh"
#include "stage_timer.h"
#include "status.h"

namespace b200nufft {

// Throws NufftFailure for a failed CUDA runtime call.
void check_cuda(cudaError_t error, const char* what);

// Counts this library's kernel launches (b200nufft_launch_count).
void note_launch(int count = 1);

// A grow-only device allocation, the analogue of the reference's
// GrowOnlyBuffer (src/gpu_point_bins.rs:53-90).
class DeviceBuffer {
 public:
  DeviceBuffer() = default;
  DeviceBuffer(const DeviceBuffer&) = delete;
  DeviceBuffer& operator=(const DeviceBuffer&) = delete;
  ~DeviceBuffer();
  // Ensures at least `bytes` bytes; contents are lost when it grows.
  void* reserve(size_t bytes, const char* label);
  void* get() const { return ptr_; }
  size_t size() const { return bytes_; }
  void release();

 private:
  void* ptr_ = nullptr;
  size_t bytes_ = 0;
};

// Fine-grid geometry and window of an F32 plan as the kernels see it.
// The f32 window as per-tap polynomials (src/kernel.rs Horner panels, fitted
// in f64 and rounded to f32): rows of highest degree first, w + 3 rows for a
// w-point window with unused leading rows zero.
constexpr int kHornerRows32 = 19;   // horner32_window (fold.cuh) assumes 19 x 16
constexpr int kHornerWidth32 = 16;

// Per slot of an f32 plan: the wrapped support start and the offset
// (start - position, in [-w/2, 1 - w/2)) of every axis; start[0] < 0 marks a
// point outside the fold reach, which the reference weighs zero.
template <int D>
struct alignas(D == 3 ? 32 : 16) PreparedWindow {
  int32_t start[D == 3 ? 4 : 2];
  float offset[D == 3 ? 4 : 2];
};

struct GridParams {
  int32_t dimensions;
  int32_t width;
  float half_width;
  float beta;
  FoldAxis axis[3];
  int64_t fine[3];       // fine-grid cells per axis
  int64_t fine_count;    // cells of one transform's grid
  // f64 plans: the native fold and the Horner table of the window.
  FoldAxis64 axis64[3];
  double half_width64;
  const double* horner;  // device, rows x width
  int32_t horner_rows;
  float horner32[kHornerRows32][kHornerWidth32];
};

// Prepared windows of `count` f32 points in slot order (coordinates in slot order).
void prepare_windows(const float* sorted_points, int64_t count, const GridParams& grid, void* windows,
                     cudaStream_t stream);
size_t prepared_window_bytes(int dimensions);
// inverse[perm[s]] = s for s < count.
void invert_permutation(const uint32_t* perm, int64_t count, uint32_t* inverse, cudaStream_t stream);

// Stable sort of the points by bin key. Launches on `stream`; all pointers
// are device pointers owned by the caller.
struct SortBuffers {
  uint32_t* keys_a;
  uint32_t* keys_b;
  uint32_t* vals_b;
  uint32_t* vals_a;
  uint32_t* hist;        // 4 passes x 256 counts
  uint32_t* status;      // tiles x 256 look-back words
  uint32_t* counters;    // 4 tile tickets + 1 error flag
};

// Key kinds: the reference's type-1 stable bins of support starts
// (src/gpu_nd_bins.rs:474-554), or its type-2 grouped bins of plain-f32
// position cells (src/gpu_point_bins.rs:422-465).
// SupportStartValidFirst: the support-start keys of the points within the
// fold's reach, and key `bins` (after every bin) for the others, which no
// spreading tile then reaches; the reference's order, with those points in
// bin 0, is rebuilt on request (reference_bin_order).
enum class KeyKind { SupportStart, ApproximateCell, SupportStartValidFirst };

// Sorts `count` points; on return `*perm` and `*sorted_keys` point into the
// buffers at the permutation and the sorted keys. Writes bin offsets
// (bins + 1 words) to `offsets`.
void sort_points(const float* points, int64_t count, const GridParams& grid, KeyKind kind,
                 uint64_t bins, SortBuffers buffers, uint32_t* offsets, uint32_t** perm,
                 uint32_t** sorted_keys, cudaStream_t stream, StageTimer* timer = nullptr);

// With KeyKind::SupportStartValidFirst the sort runs over bins + 1 keys and
// writes bins + 2 offsets (offsets[bins] = points within reach), and
// `valid_mask` (ceil(count / 32) words, bit i % 32 of word i / 32) marks the
// points within reach in the caller's order.
void sort_points_valid_first(const float* points, int64_t count, const GridParams& grid, uint64_t bins,
                             SortBuffers buffers, uint32_t* offsets, uint32_t* valid_mask, uint32_t** perm,
                             uint32_t** sorted_keys, cudaStream_t stream, StageTimer* timer = nullptr);

// The same for f64 coordinates folded in native f64 (support-start keys);
// with `valid_mask` non-null the points outside the fold's reach sort after
// every bin as above.
void sort_points64(const double* points, int64_t count, const GridParams& grid, uint64_t bins,
                   SortBuffers buffers, uint32_t* offsets, uint32_t** perm, uint32_t** sorted_keys,
                   cudaStream_t stream, StageTimer* timer = nullptr, uint32_t* valid_mask = nullptr);

// The reference's order from a valid-first sort: the points outside the
// fold's reach merged into bin 0 by original index, and bin offsets that
// count them in bin 0 (bins + 1 words). `ref_keys` receives the sorted keys.
void reference_bin_order(const uint32_t* perm, const uint32_t* keys, const uint32_t* offsets, int64_t count,
                         uint64_t bins, uint32_t* ref_perm, uint32_t* ref_keys, uint32_t* ref_offsets,
                         cudaStream_t stream);

// The coordinates of `count` points in the bin order `perm`.
void gather_sorted_points(const float* points, const uint32_t* perm, int64_t count, int dimensions,
                          float* sorted, cudaStream_t stream, StageTimer* timer = nullptr);
void gather_sorted_points64(const double* points, const uint32_t* perm, int64_t count,
                            int dimensions, double* sorted, cudaStream_t stream,
                            StageTimer* timer = nullptr);
// The inverse for 3D coordinates: points[perm[i]] = sorted[i] (float, double).
template <typename T>
void scatter_points3(const T* sorted, const uint32_t* perm, int64_t count, T* points, cudaStream_t stream);

// Df64 storage (a (hi, lo) pair of floats per scalar, the reference's
// double-float format) to and from f64, `count` scalars.
void df64_to_f64(const float* pairs, int64_t count, double* out, cudaStream_t stream);
void f64_to_df64(const double* values, int64_t count, float* pairs, cudaStream_t stream);

// Points per tile of the sort's radix passes; each tile publishes 256
// look-back words (one per digit) per pass.
constexpr int kSortTilePoints = 4096;
constexpr int kSortDigits = 256;

// Bytes of look-back status words a sort of `count` points needs.
size_t sort_status_bytes(int64_t count);

// Reference-layout prepared slots of the stable type-1 binning.
void prepare_reference_slots(const float* points, int64_t count, const GridParams& grid,
                             const uint32_t* perm, const uint32_t* sorted_keys, int32_t* starts,
                             float* offsets, cudaStream_t stream);

}  // namespace b200nufft
