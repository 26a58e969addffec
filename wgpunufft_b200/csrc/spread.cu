// Type-1 spreading: bin subproblems accumulated in shared memory.
//
// The reference spreads with an output-stationary block spreader that sums
// every cell's points in a fixed order, with no floating-point atomics, so
// that outputs are bitwise repeatable (src/gpu_nd_spread.rs:1-35). Here each
// CTA takes one subproblem: the points whose support starts in one tile of the
// fine grid (or one part of a crowded tile), read from the bins of the stable
// sort. Every point evaluates its window per axis into registers and adds
// its w^d contributions to a padded copy of the tile in shared memory. The
// contributions are accumulated as fixed-point integers, scaled by a power of
// two derived from the largest strength (f32 plans: each rounded to a 32-bit
// integer and summed exactly in two 32-bit halves; f64 plans: 64-bit integers
// with 2^-50 resolution), so the sum of a cell is the exact integer sum of its
// rounded contributions whatever order the threads add them in: the
// accumulation is deterministic without ordering the threads, and it carries
// more bits than a floating-point sum. Each padded tile is then converted back
// to floating point and written out, and a fold pass adds, for every
// fine-grid cell, the padded tiles and parts that cover it in a fixed order
// (halos wrap periodically). Nothing is accumulated with floating-point
// atomics.
#include <cuda_runtime.h>

#include <algorithm>

#include "device.h"
#include "spread.h"

namespace b200nufft {

namespace {

constexpr int kSpreadThreads = 256;

// ---------------------------------------------------------------------------
// Precision traits: coordinates, window, fixed-point accumulator.

struct F32Traits {
  static constexpr bool kPreparedWindows = true;
  using Real = float;
  using Complex = float2;
  using Bits = uint32_t;
  // Shared-memory words per padded cell: re lo, re hi, im lo, im hi.
  static constexpr int kWordsPerCell = 4;
  using Word = uint32_t;

  static __device__ __forceinline__ Bits magnitude_bits(float v) {
    return __float_as_uint(v) & 0x7fffffffu;
  }
  // S so that every contribution, at most the largest strength, scales below
  // 2^30: each then rounds to a 32-bit integer with a resolution of 2^-30 of
  // the largest strength. Non-finite strengths leave the outputs unspecified
  // but the exponent bounded.
  static __device__ __forceinline__ int exponent(Bits max_bits) {
    if (max_bits == 0u) return 0;
    const int e = max_bits >= 0x7f800000u ? 128 : ilogbf(__uint_as_float(max_bits)) + 1;
    return 30 - e;
  }
  static __device__ __forceinline__ bool in_reach(float x) { return in_fold_reach(x); }
  static __device__ __forceinline__ void window(float x, const GridParams& g, int a, int32_t& wrapped,
                                                float* w, int W) {
    int32_t start;
    Df64 off;
    support_of(x, g.axis[a], g.half_width, start, off);
    wrapped = wrap_start(start, g.axis[a].length);
    const float width_f = static_cast<float>(W);
    for (int j = 0; j < W; ++j) {
      const float d = __fadd_rn(__fadd_rn(static_cast<float>(j), off.hi), off.lo);
      w[j] = es_weight(d, g.beta, width_f);
    }
  }
  static __device__ __forceinline__ float power_of_two(int e) { return ldexpf(1.0f, e); }
  // Adds a contribution (|v| < 2^31 after rounding) as two exact 32-bit sums:
  // its low 16 bits, unsigned, and its arithmetic high part. Both stay exact
  // for up to 2^16 contributions per cell; the cell's value is hi 2^16 + lo.
  static __device__ __forceinline__ void add(Word* acc, int padded, int part, int c, float value) {
    const int32_t v = __float2int_rn(value);
    atomicAdd(&acc[(2 * part) * padded + c], static_cast<uint32_t>(v) & 0xFFFFu);
    atomicAdd(reinterpret_cast<int32_t*>(&acc[(2 * part + 1) * padded + c]), v >> 16);
  }
  static __device__ __forceinline__ float value(const Word* acc, int padded, int part, int c, int S) {
    const uint32_t lo = acc[(2 * part) * padded + c];
    const int32_t hi = static_cast<int32_t>(acc[(2 * part + 1) * padded + c]);
    const long long total = static_cast<long long>(hi) * 65536ll + static_cast<long long>(lo);
    return ldexpf(__ll2float_rn(total), -S);
  }
};

struct F64Traits {
  static constexpr bool kPreparedWindows = false;
  using Real = double;
  using Complex = double2;
  using Bits = unsigned long long;
  // Shared-memory words per padded cell: re, im (64-bit).
  static constexpr int kWordsPerCell = 2;
  using Word = unsigned long long;

  static __device__ __forceinline__ Bits magnitude_bits(double v) {
    return static_cast<unsigned long long>(__double_as_longlong(v)) & 0x7fffffffffffffffull;
  }
  // S so that every contribution scales below 2^50; a part of at most 4096
  // records then sums below 2^62 in every cell, with a resolution of 2^-50 of
  // the largest strength.
  static __device__ __forceinline__ int exponent(Bits max_bits) {
    if (max_bits == 0ull) return 0;
    const int e = max_bits >= 0x7ff0000000000000ull ? 1024 : ilogb(__longlong_as_double(static_cast<long long>(max_bits))) + 1;
    return 50 - e;
  }
  static __device__ __forceinline__ bool in_reach(double x) { return in_fold_reach64(x); }
  static __device__ __forceinline__ void window(double x, const GridParams& g, int a,
                                                int32_t& wrapped, double* w, int W) {
    int32_t start;
    double offset;
    support_of64(x, g.axis64[a], g.half_width64, start, offset);
    wrapped = wrap_start(start, g.axis[a].length);
    for (int j = 0; j < W; ++j) w[j] = horner_weight(offset, j, W, g.horner, g.horner_rows);
  }
  static __device__ __forceinline__ double power_of_two(int e) { return ldexp(1.0, e); }
  static __device__ __forceinline__ void add(Word* acc, int padded, int part, int c, double value) {
    atomicAdd(&acc[part * padded + c], static_cast<unsigned long long>(__double2ll_rn(value)));
  }
  static __device__ __forceinline__ double value(const Word* acc, int padded, int part, int c, int S) {
    return ldexp(__ll2double_rn(static_cast<long long>(acc[part * padded + c])), -S);
  }
};

template <typename T>
struct SpreadLaunchT {
  const typename T::Real* points;
  const void* windows;
  const typename T::Complex* strengths;
  int64_t point_count;
  int batch;
  const uint32_t* perm;
  const uint32_t* offsets;
  const uint32_t* part_start;
  int64_t part_upper_bound;
  typename T::Bits* max_bits;
  typename T::Complex* scratch;
  const int2* candidates;
  typename T::Complex* fine;
  const uint32_t* valid_mask;
};

// Records per part of this point set.
__device__ __forceinline__ int32_t part_cap_of(const SpreadParams& sp) {
  return sp.part_cap_device != nullptr ? *sp.part_cap_device : sp.part_cap;
}

// The part cap from the number of points within reach (SpreadParams).
__global__ void part_cap_kernel(SpreadParams sp, const uint32_t* __restrict__ offsets) {
  const long long valid = offsets[sp.cap_bins];
  const long long ctas = valid >= sp.crowded_points ? sp.cap_ctas_crowded : sp.cap_ctas;
  long long cap = ((valid > 1 ? valid : 1ll) + ctas - 1) / ctas;
  cap = (cap + 255) / 256 * 256;
  cap = cap < 256 ? 256 : cap;
  cap = cap > sp.cap_max ? static_cast<long long>(sp.cap_max) : cap;
  *sp.part_cap_device = static_cast<int32_t>(cap);
}

// Largest |re| or |im| of every strength vector, as magnitude bits, over
// the points within reach when a mask is given (others get zero weight, so
// their strengths must not change the fixed-point scale). A thread takes
// four consecutive values per step (two 16-byte loads for f32 vectors that
// start 16-byte aligned) and the mask bits of those four points; the block
// reduces its warps' maxima and adds one atomicMax (thousands of per-warp
// atomics on one word serialize at its L2 slice).
template <typename T>
__global__ void __launch_bounds__(256) strength_magnitude_kernel(const typename T::Complex* __restrict__ values,
                                                                 int64_t count, int batch,
                                                                 typename T::Bits* __restrict__ max_bits,
                                                                 const uint32_t* __restrict__ valid_mask) {
  using Bits = typename T::Bits;
  __shared__ Bits warp_max[8];
  const int b = blockIdx.y;
  const typename T::Complex* v = values + static_cast<int64_t>(b) * count;
  Bits m = 0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x * 4;
  const bool vector16 =
      sizeof(typename T::Complex) == 8 && (reinterpret_cast<uintptr_t>(v) & 15) == 0;
  for (int64_t i = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) * 4; i < count; i += stride) {
    const uint32_t bits = valid_mask != nullptr ? (__ldg(&valid_mask[i >> 5]) >> (i & 31)) : 0xFu;
    if (vector16 && i + 4 <= count) {
      const float4 p = __ldg(reinterpret_cast<const float4*>(v + i));
      const float4 q = __ldg(reinterpret_cast<const float4*>(v + i) + 1);
      const float r[8] = {p.x, p.y, p.z, p.w, q.x, q.y, q.z, q.w};
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if ((bits >> k) & 1u) {
          m = max(m, static_cast<Bits>(__float_as_uint(r[2 * k]) & 0x7fffffffu));
          m = max(m, static_cast<Bits>(__float_as_uint(r[2 * k + 1]) & 0x7fffffffu));
        }
      }
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (i + k < count && ((bits >> k) & 1u)) {
          const typename T::Complex s = v[i + k];
          m = max(m, T::magnitude_bits(s.x));
          m = max(m, T::magnitude_bits(s.y));
        }
      }
    }
  }
#pragma unroll
  for (int offset = 16; offset > 0; offset >>= 1) m = max(m, __shfl_xor_sync(0xFFFFFFFFu, m, offset));
  if ((threadIdx.x & 31) == 0) warp_max[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < static_cast<int>(blockDim.x >> 5); ++w) m = max(m, warp_max[w]);
    if (m) atomicMax(&max_bits[b], m);
  }
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
  const uint32_t cap = static_cast<uint32_t>(part_cap_of(sp));
  parts[t] = static_cast<uint32_t>((count + cap - 1) / cap);
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

// Records per register run of a thread: one for 3D and for windows whose
// w^2 complex accumulators would not fit in registers.
constexpr int kRunBits = 6;
template <int D, int W, typename T>
__host__ __device__ constexpr int spread_run() {
  return (D == 1 || (D == 2 && 2 * W * W * sizeof(typename T::Real) < 400)) ? (1 << kRunBits) : 1;
}

// Record r of the tile's bin rows: its support start relative to the tile,
// its window weights and its strength. False when the point lies outside the
// fold reach (weighed zero by the reference) or starts in another tile (a bin
// wider than the tile).
template <int D, int W, typename T>
__device__ __forceinline__ bool tile_record(const SpreadParams& sp, const typename T::Real* points,
                                            const void* windows, const typename T::Complex* sv,
                                            const uint32_t* perm, const uint32_t* row_begin,
                                            const uint32_t* row_prefix, int rows, const int* origin,
                                            uint32_t r, int& row, int* local_start,
                                            typename T::Real (*w)[W], typename T::Complex& s) {
  using Real = typename T::Real;
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
  if constexpr (T::kPreparedWindows) {
    // f32 plans: the window start and offset prepared at set_points.
    const PreparedWindow<D> win = static_cast<const PreparedWindow<D>*>(windows)[slot];
    if (win.start[0] < 0) return false;  // outside the fold reach: weighed zero
    bool inside = true;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      local_start[a] = win.start[a] - origin[a];
      inside = inside && local_start[a] >= 0 && local_start[a] < sp.tile[a];
    }
    if (!inside) return false;  // a bin wider than the tile: another tile owns it
#pragma unroll
    for (int a = 0; a < D; ++a) horner32_window<W>(win.offset[a], sp.grid.horner32, w[a]);
    s = sv[perm[slot]];
    return true;
  }
  Real p[D];
#pragma unroll
  for (int a = 0; a < D; ++a) p[a] = points[static_cast<int64_t>(slot) * D + a];
  bool reach = true;
#pragma unroll
  for (int a = 0; a < D; ++a) reach = reach && T::in_reach(p[a]);
  if (!reach) return false;
  bool inside = true;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    int32_t wrapped;
    T::window(p[a], sp.grid, a, wrapped, w[a], W);
    local_start[a] = wrapped - origin[a];
    inside = inside && local_start[a] >= 0 && local_start[a] < sp.tile[a];
  }
  if (!inside) return false;
  s = sv[perm[slot]];
  return true;
}

// Slot of record r of the tile's bin rows (rows are visited in order).
__device__ __forceinline__ uint32_t record_slot(uint32_t r, int& row, const uint32_t* row_begin,
                                                const uint32_t* row_prefix, int rows) {
  if (r >= row_prefix[row + 1] || r < row_prefix[row]) {
    int low = 0, high = rows - 1;
    while (low < high) {
      const int mid = (low + high + 1) >> 1;
      if (row_prefix[mid] <= r) low = mid; else high = mid - 1;
    }
    row = low;
  }
  return row_begin[row] + (r - row_prefix[row]);
}

// A prepared f32 record: its start relative to the tile and its window
// weights; false when it lies outside the fold reach or starts in another tile.
template <int D, int W>
__device__ __forceinline__ bool prepared_record(const SpreadParams& sp, const PreparedWindow<D>& win,
                                                const int* origin, int* local_start, float (*w)[W]) {
  if (win.start[0] < 0) return false;
  bool inside = true;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    local_start[a] = win.start[a] - origin[a];
    inside = inside && local_start[a] >= 0 && local_start[a] < sp.tile[a];
  }
  if (!inside) return false;
#pragma unroll
  for (int a = 0; a < D; ++a) horner32_window<W>(win.offset[a], sp.grid.horner32, w[a]);
  return true;
}

// Adds a run's register sums (already in the fixed-point scale) to the tile
// and clears them.
template <int D, int W, typename T>
__device__ __forceinline__ void flush_run(typename T::Word* acc, int padded, int pad0, int x, int y,
                                          typename T::Complex (*a)[W]) {
  constexpr int R = D == 2 ? W : 1;
#pragma unroll
  for (int j = 0; j < R; ++j) {
    const int base = (y + j) * pad0 + x;
#pragma unroll
    for (int i = 0; i < W; ++i) {
      T::add(acc, padded, 0, base + i, a[j][i].x);
      T::add(acc, padded, 1, base + i, a[j][i].y);
      a[j][i].x = a[j][i].y = typename T::Real(0);
    }
  }
}

// 2D register windows slide along x: when a thread's next record starts
// d columns to the right in the same row, the d leftmost window columns are
// complete (no later record of the thread's range reaches them), so they
// are added to the tile and the window shifts left, instead of adding all
// w^2 cells at every change of start. Records of one-cell bins come in
// (row, column) order, so a thread's range of consecutive records flushes
// about one column per distinct start.
template <int W, typename T>
__device__ __forceinline__ void flush_first_column(typename T::Word* acc, int padded, int pad0, int x, int y,
                                                   typename T::Complex (*a)[W]) {
#pragma unroll
  for (int j = 0; j < W; ++j) {
    const int c = (y + j) * pad0 + x;
    T::add(acc, padded, 0, c, a[j][0].x);
    T::add(acc, padded, 1, c, a[j][0].y);
#pragma unroll
    for (int i = 0; i + 1 < W; ++i) a[j][i] = a[j][i + 1];
    a[j][W - 1].x = a[j][W - 1].y = typename T::Real(0);
  }
}

// 3D f32 tiles of widths 5 to 8 are spread by whole warps, one record at a
// time. The padded tile lives in shared memory with pitches chosen so that
// the window's segments (L consecutive cells of one x row) start in
// distinct banks, and lane l owns the segments that start in bank l: every
// add instruction of the warp touches 32 different banks, whatever the
// record. Lanes sum the records of a run with one support start in float
// registers (a fixed order: the record order) and add the run to the
// fixed-point tile once, rounded, when the start changes or after
// 2^kWarpRunBits records.
//
// In crowded tiles (at least one record per start cell) each part's records
// are first bucketed by their start in shared memory by a stable counting
// sort, so that runs are as long as the data allows; otherwise the records
// are taken in bin order. Points outside the fold reach or starting in
// another tile are skipped.
constexpr int kWarpRunBits = 5;
constexpr int kWarpMaxRecords = 2048;  // the 3D part cap
constexpr int kWarpGroup = 8;          // records staged per warp at a time
constexpr int kStageStride = 28;       // wx[8] wy[8] wz[8] re im base -
constexpr int kSpreadWarps = kSpreadThreads / 32;

template <int D, int W, typename T>
__host__ __device__ constexpr bool warp_capable() {
  return D == 3 && T::kPreparedWindows && W >= kWarpMinWidth && W <= kWarpMaxWidth;
}

template <int W>
__device__ void spread_warp3(const SpreadParams& sp, const PreparedWindow<3>* win3, const float2* sv,
                             const uint32_t* perm, const uint32_t* row_begin, const uint32_t* row_prefix,
                             int rows, const int* origin, uint32_t record_begin, uint32_t record_end,
                             bool bucket, uint32_t* acc, int span, uint32_t* sorted,
                             float (*stage)[kWarpGroup][kStageStride], int exponent, int& S) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int t0 = sp.tile[0], t1 = sp.tile[1];
  const int cells = t0 * t1 * sp.tile[2];
  const int pitch0 = sp.pitch0, pitch01 = sp.pitch01;
  auto slot_of = [&](uint32_t r, int& row) {
    if (r >= row_prefix[row + 1] || r < row_prefix[row]) {
      int low = 0, high = rows - 1;
      while (low < high) {
        const int mid = (low + high + 1) >> 1;
        if (row_prefix[mid] <= r) low = mid; else high = mid - 1;
      }
      row = low;
    }
    return row_begin[row] + (r - row_prefix[row]);
  };
  // Local start of a record; false when it is skipped.
  auto local_of = [&](const PreparedWindow<3>& win, int& x, int& y, int& z) {
    if (win.start[0] < 0) return false;
    x = win.start[0] - origin[0];
    y = win.start[1] - origin[1];
    z = win.start[2] - origin[2];
    return x >= 0 && x < t0 && y >= 0 && y < t1 && z >= 0 && z < sp.tile[2];
  };
  const uint32_t n = record_end - record_begin;
  uint32_t spread_count = n;
  if (bucket) {
    // count[key * warps + warp]: each warp's records per start (the last key
    // collects the skipped records), in the tile region, cleared below.
    uint32_t* count = acc;
    const int entries = (cells + 1) * kSpreadWarps;
    for (int c = tid; c < entries; c += kSpreadThreads) count[c] = 0u;
    __syncthreads();
    auto key_of = [&](const PreparedWindow<3>& win) {
      int x, y, z;
      return local_of(win, x, y, z) ? x + t0 * (y + t1 * z) : cells;
    };
    // Warp w sorts the consecutive records [warp_begin, warp_end).
    const uint32_t per_warp = (n + kSpreadWarps - 1) / kSpreadWarps;
    const uint32_t warp_begin = record_begin + min(n, per_warp * warp);
    const uint32_t warp_end = record_begin + min(n, per_warp * (warp + 1));
    int row = 0;
    for (uint32_t r = warp_begin + lane; r < warp_end; r += 32) {
      atomicAdd(&count[key_of(win3[slot_of(r, row)]) * kSpreadWarps + warp], 1u);
    }
    __syncthreads();
    // Exclusive scan of the entries, key-major: a contiguous block per
    // thread, the block sums in the front of `sorted`, filled afterwards.
    uint32_t* block_sums = sorted;
    const int per = (entries + kSpreadThreads - 1) / kSpreadThreads;
    const int c0 = min(entries, tid * per), c1 = min(entries, c0 + per);
    uint32_t sum = 0;
    for (int c = c0; c < c1; ++c) sum += count[c];
    block_sums[tid] = sum;
    __syncthreads();
    if (warp == 0) {
      constexpr int kPer = kSpreadThreads / 32;
      uint32_t v[kPer];
      uint32_t mine = 0;
#pragma unroll
      for (int k = 0; k < kPer; ++k) {
        v[k] = block_sums[lane * kPer + k];
        mine += v[k];
      }
      uint32_t x = mine;
#pragma unroll
      for (int offset = 1; offset < 32; offset <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, offset);
        if (lane >= offset) x += y;
      }
      uint32_t running = x - mine;
#pragma unroll
      for (int k = 0; k < kPer; ++k) {
        block_sums[lane * kPer + k] = running;
        running += v[k];
      }
    }
    __syncthreads();
    uint32_t running = block_sums[tid];
    for (int c = c0; c < c1; ++c) {
      const uint32_t v = count[c];
      count[c] = running;
      running += v;
    }
    __syncthreads();
    spread_count = count[cells * kSpreadWarps];
    __syncthreads();  // every thread has read the count before the scatter moves the counters
    // Stable scatter: each warp walks its records in order, 32 at a time;
    // equal keys in one step take consecutive places in lane order.
    row = 0;
    const unsigned lower = (1u << lane) - 1u;
    for (uint32_t first = warp_begin; first < warp_end; first += 32) {
      const uint32_t r = first + lane;
      int key = -1;
      uint32_t slot = 0;
      if (r < warp_end) {
        slot = slot_of(r, row);
        key = key_of(win3[slot]);
      }
      const unsigned same = __match_any_sync(0xFFFFFFFFu, key);
      uint32_t* counter = &count[(key < 0 ? 0 : key) * kSpreadWarps + warp];
      const uint32_t place = key < 0 ? 0u : *counter + __popc(same & lower);
      __syncwarp();
      if (key >= 0) {
        sorted[place] = slot;
        if ((same & lower) == 0u) *counter += __popc(same);
      }
      __syncwarp();
    }
    __syncthreads();
    for (int c = tid; c < 4 * span; c += kSpreadThreads) acc[c] = 0u;
    __syncthreads();
  }
  S = exponent - kWarpRunBits;
  const float scale_lo = ldexpf(1.0f, S / 2);
  const float scale_hi = ldexpf(1.0f, S - S / 2);

  constexpr int L = warp_segment_cells(W);
  constexpr int R = warp_rounds(W);
  // Staged x weights: one block of up to 8, or (w = 6) the two 3-cell
  // segments at offsets 0 and 4, so a lane reads its segment with one
  // aligned load from an offset fixed for the part.
  constexpr bool kSplitX = W / L == 2;
  static_assert(W / L == 1 || (kSplitX && L <= 4), "x segments are one block or two aligned halves");
  uint32_t desc[R];
  int xo[R], yo[R], zo[R];  // the lane's stage offsets of each round: x segment, wy[j], wz[k]
#pragma unroll
  for (int r = 0; r < R; ++r) {
    desc[r] = sp.warp_segments[r * 32 + lane];
    xo[r] = 4 * static_cast<int>((desc[r] >> 16) & 15);
    yo[r] = 8 + static_cast<int>((desc[r] >> 20) & 15);
    zo[r] = 16 + static_cast<int>((desc[r] >> 24) & 15);
  }
  float2 a2[R][L];  // (re, im) register sums of the run
#pragma unroll
  for (int r = 0; r < R; ++r) {
#pragma unroll
    for (int t = 0; t < L; ++t) a2[r][t] = make_float2(0.0f, 0.0f);
  }
  int run = -1, run_length = 0;
  auto flush = [&]() {
#pragma unroll
    for (int r = 0; r < R; ++r) {
      if (desc[r] & kSegmentValid) {
        const int c = run + static_cast<int>(desc[r] & 0xFFFFu);
#pragma unroll
        for (int t = 0; t < L; ++t) {
          F32Traits::add(acc, span, 0, c + t, a2[r][t].x);
          F32Traits::add(acc, span, 1, c + t, a2[r][t].y);
        }
      }
#pragma unroll
      for (int t = 0; t < L; ++t) a2[r][t] = make_float2(0.0f, 0.0f);
    }
  };
  float (*my_stage)[kStageStride] = stage[warp];
  // Warp w spreads the consecutive records [spread_begin, spread_end) of the
  // bucketed order (or of the bin order), so runs continue across groups.
  const uint32_t per_warp = (spread_count + kSpreadWarps - 1) / kSpreadWarps;
  const uint32_t spread_begin = min(spread_count, per_warp * warp);
  const uint32_t spread_end = min(spread_count, per_warp * (warp + 1));
  int row = 0;
  // Lane 3 g + a stages axis a of record g of each group; its record's
  // window and point index are loaded two groups ahead and the strength one
  // group ahead, so the loads overlap the spreading of earlier groups.
  const int stage_g = lane / 3, stage_a = lane - 3 * stage_g;
  const bool stager = lane < 3 * kWarpGroup;
  PreparedWindow<3> win0{}, win1{};
  win0.start[0] = win1.start[0] = -1;
  uint32_t point1 = 0;
  float2 c0 = make_float2(0.0f, 0.0f);
  auto fetch = [&](uint32_t r, PreparedWindow<3>& win, uint32_t& point) {
    win.start[0] = -1;
    if (stager && r < spread_end) {
      const uint32_t slot = bucket ? sorted[r] : slot_of(record_begin + r, row);
      win = win3[slot];
      if (stage_a == 0) point = perm[slot];
    }
  };
  {
    uint32_t point0 = 0;
    fetch(spread_begin + stage_g, win0, point0);
    if (stager && stage_a == 0 && spread_begin + stage_g < spread_end) c0 = sv[point0];
    fetch(spread_begin + kWarpGroup + stage_g, win1, point1);
  }
  for (uint32_t first = spread_begin; first < spread_end; first += kWarpGroup) {
    const PreparedWindow<3> win = win0;
    const float2 c = c0;
    if (stager && stage_a == 0 && first + kWarpGroup + stage_g < spread_end) c0 = sv[point1];
    win0 = win1;
    fetch(first + 2 * kWarpGroup + stage_g, win1, point1);
    // Stage the group: lane 3 g + a evaluates axis a of record g; lane 3 g
    // also stages the scaled strength and the start's tile offset (-1: skip).
    if (stager) {
      const int g = stage_g, a = stage_a;
      const uint32_t r = first + g;
      int base = -1;
      float w[W];
#pragma unroll
      for (int j = 0; j < W; ++j) w[j] = 0.0f;
      if (r < spread_end) {
        int x, y, z;
        if (local_of(win, x, y, z)) {
          base = x + y * pitch0 + z * pitch01;
          const float offset = a == 0 ? win.offset[0] : (a == 1 ? win.offset[1] : win.offset[2]);
          horner32_window<W>(offset, sp.grid.horner32, w);
          if (a == 0) {
            my_stage[g][24] = (c.x * scale_lo) * scale_hi;
            my_stage[g][25] = (c.y * scale_lo) * scale_hi;
          }
        }
      }
      if (kSplitX && a == 0) {
#pragma unroll
        for (int j = 0; j < 8; ++j) my_stage[g][j] = (j & 3) < L ? w[(j >> 2) * L + (j & 3)] : 0.0f;
      } else {
#pragma unroll
        for (int j = 0; j < 8; ++j) my_stage[g][a * 8 + j] = j < W ? w[j] : 0.0f;
      }
      if (a == 0) my_stage[g][26] = __int_as_float(base);
    }
    __syncwarp();
#pragma unroll 1
    for (int g = 0; g < kWarpGroup; ++g) {
      const float* st = my_stage[g];
      const int base = __float_as_int(st[26]);
      if (base < 0) continue;
      if (base != run || run_length == (1 << kWarpRunBits)) {
        if (run >= 0) flush();
        run = base;
        run_length = 0;
      }
      ++run_length;
      const float2 c = *reinterpret_cast<const float2*>(st + 24);
      float wx[8];
      if (!kSplitX) {
        const float4 x_lo = *reinterpret_cast<const float4*>(st);
        const float4 x_hi = *reinterpret_cast<const float4*>(st + 4);
        wx[0] = x_lo.x; wx[1] = x_lo.y; wx[2] = x_lo.z; wx[3] = x_lo.w;
        wx[4] = x_hi.x; wx[5] = x_hi.y; wx[6] = x_hi.z; wx[7] = x_hi.w;
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const float wyz = st[yo[r]] * st[zo[r]];
        const float2 wc = cscale(c, wyz);
        float wxs[L];
        if (kSplitX) {
          const float4 seg = *reinterpret_cast<const float4*>(st + xo[r]);
          const float v[4] = {seg.x, seg.y, seg.z, seg.w};
#pragma unroll
          for (int t = 0; t < L; ++t) wxs[t] = v[t];
        } else {
#pragma unroll
          for (int t = 0; t < L; ++t) wxs[t] = wx[t];
        }
#pragma unroll
        for (int t = 0; t < L; ++t) a2[r][t] = cfma(wc, wxs[t], a2[r][t]);
      }
    }
    __syncwarp();
  }
  if (run >= 0) flush();
}

// 2D f64 tiles (windows of 5 taps or more, too wide for a thread's register
// run) are spread by whole warps, one record at a time: lanes 0 .. 2w-1
// evaluate one window tap each (axis a = lane / w), and lane l owns the
// window cells u = l + 32 q (x = u mod w, y = u / w), summing a run of
// records with one support start in f64 registers in record order. A run
// reaches the 64-bit fixed-point tile once, when its start changes; the tile
// of a part of at most 4096 records stays below 2^62 in every cell whatever
// the runs, so the scale is the record-by-record one.
template <int W>
__device__ void spread_warp2_f64(const SpreadParams& sp, const double* points, const double2* sv,
                                 const uint32_t* perm, const uint32_t* row_begin, const uint32_t* row_prefix,
                                 int rows, const int* origin, uint32_t record_begin, uint32_t record_end,
                                 unsigned long long* acc, int padded, double (*stage)[2][W], double scale_lo,
                                 double scale_hi) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int R = (W * W + 31) / 32;
  double ar[R], ai[R];
#pragma unroll
  for (int q = 0; q < R; ++q) ar[q] = ai[q] = 0.0;
  int run_x = -1, run_y = 0;
  const int pad0 = sp.pad[0];
  auto flush = [&]() {
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int u = lane + 32 * q;
      if (u < W * W) {
        const int c = (run_y + u / W) * pad0 + run_x + u % W;
        F64Traits::add(acc, padded, 0, c, ar[q]);
        F64Traits::add(acc, padded, 1, c, ai[q]);
      }
      ar[q] = ai[q] = 0.0;
    }
  };
  // Warp w spreads the consecutive records [warp_begin, warp_end).
  const uint32_t n = record_end - record_begin;
  const uint32_t per_warp = (n + kSpreadWarps - 1) / kSpreadWarps;
  const uint32_t warp_begin = record_begin + min(n, per_warp * warp);
  const uint32_t warp_end = record_begin + min(n, per_warp * (warp + 1));
  const int axis = lane < W ? 0 : 1, tap = lane < W ? lane : lane - W;
  double* my_tap = &stage[warp][axis][tap];
  int row = 0;
  // The next record's coordinates and point index are loaded one record
  // ahead, and the strength as soon as its index is known.
  double next_x = 0.0, next_y = 0.0;
  uint32_t next_point = 0;
  if (warp_begin < warp_end) {
    const uint32_t slot = record_slot(warp_begin, row, row_begin, row_prefix, rows);
    next_x = points[static_cast<int64_t>(slot) * 2];
    next_y = points[static_cast<int64_t>(slot) * 2 + 1];
    next_point = perm[slot];
  }
  for (uint32_t r = warp_begin; r < warp_end; ++r) {
    const double x = next_x, y = next_y;
    const double2 c = sv[next_point];
    if (r + 1 < warp_end) {
      const uint32_t slot = record_slot(r + 1, row, row_begin, row_prefix, rows);
      next_x = points[static_cast<int64_t>(slot) * 2];
      next_y = points[static_cast<int64_t>(slot) * 2 + 1];
      next_point = perm[slot];
    }
    if (!F64Traits::in_reach(x) || !F64Traits::in_reach(y)) continue;
    int32_t start[2];
    double offset[2];
    support_of64(x, sp.grid.axis64[0], sp.grid.half_width64, start[0], offset[0]);
    support_of64(y, sp.grid.axis64[1], sp.grid.half_width64, start[1], offset[1]);
    const int lx = wrap_start(start[0], sp.grid.axis[0].length) - origin[0];
    const int ly = wrap_start(start[1], sp.grid.axis[1].length) - origin[1];
    if (lx < 0 || lx >= sp.tile[0] || ly < 0 || ly >= sp.tile[1]) continue;  // another tile owns it
    __syncwarp();  // the previous record's taps are read
    if (lane < 2 * W) {
      *my_tap = horner_weight(axis == 0 ? offset[0] : offset[1], tap, W, sp.grid.horner, sp.grid.horner_rows);
    }
    __syncwarp();
    if (lx != run_x || ly != run_y) {
      if (run_x >= 0) flush();
      run_x = lx;
      run_y = ly;
    }
    const double sr = (c.x * scale_lo) * scale_hi, si = (c.y * scale_lo) * scale_hi;
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int u = lane + 32 * q;
      if (u < W * W) {
        const double weight = stage[warp][0][u % W] * stage[warp][1][u / W];
        ar[q] = fma(sr, weight, ar[q]);
        ai[q] = fma(si, weight, ai[q]);
      }
    }
  }
  if (run_x >= 0) flush();
}

// 3D f64 tiles (windows of 5 taps or more) are spread by whole warps, one
// record at a time: the lanes evaluate the 3w window taps (tap t on axis
// t / w), and lane l adds the contributions of window cells
// u = l + 32 q (x = u mod w, y = (u / w) mod w, z = u / w^2) straight to the
// 64-bit fixed-point tile; the 32 lanes of an add touch 32 different cells.
template <int W>
__device__ void spread_warp3_f64(const SpreadParams& sp, const double* points, const double2* sv,
                                 const uint32_t* perm, const uint32_t* row_begin, const uint32_t* row_prefix,
                                 int rows, const int* origin, uint32_t record_begin, uint32_t record_end,
                                 unsigned long long* acc, int padded, double (*stage)[3][W], double scale_lo,
                                 double scale_hi) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int kCells = W * W * W;
  constexpr int R = (kCells + 31) / 32;
  const int pad0 = sp.pad[0], pad01 = sp.pad[0] * sp.pad[1];
  const uint32_t n = record_end - record_begin;
  const uint32_t per_warp = (n + kSpreadWarps - 1) / kSpreadWarps;
  const uint32_t warp_begin = record_begin + min(n, per_warp * warp);
  const uint32_t warp_end = record_begin + min(n, per_warp * (warp + 1));
  int row = 0;
  double next[3] = {0.0, 0.0, 0.0};
  uint32_t next_point = 0;
  if (warp_begin < warp_end) {
    const uint32_t slot = record_slot(warp_begin, row, row_begin, row_prefix, rows);
#pragma unroll
    for (int a = 0; a < 3; ++a) next[a] = points[static_cast<int64_t>(slot) * 3 + a];
    next_point = perm[slot];
  }
  for (uint32_t r = warp_begin; r < warp_end; ++r) {
    const double p[3] = {next[0], next[1], next[2]};
    const double2 c = sv[next_point];
    if (r + 1 < warp_end) {
      const uint32_t slot = record_slot(r + 1, row, row_begin, row_prefix, rows);
#pragma unroll
      for (int a = 0; a < 3; ++a) next[a] = points[static_cast<int64_t>(slot) * 3 + a];
      next_point = perm[slot];
    }
    if (!F64Traits::in_reach(p[0]) || !F64Traits::in_reach(p[1]) || !F64Traits::in_reach(p[2])) continue;
    int local[3];
    double offset[3];
    bool inside = true;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      int32_t start;
      support_of64(p[a], sp.grid.axis64[a], sp.grid.half_width64, start, offset[a]);
      local[a] = wrap_start(start, sp.grid.axis[a].length) - origin[a];
      inside = inside && local[a] >= 0 && local[a] < sp.tile[a];
    }
    if (!inside) continue;  // another tile owns it
    __syncwarp();  // the previous record's taps are read
    for (int t = lane; t < 3 * W; t += 32) {
      const int a = t / W, j = t - a * W;
      const double o = a == 0 ? offset[0] : (a == 1 ? offset[1] : offset[2]);
      stage[warp][a][j] = horner_weight(o, j, W, sp.grid.horner, sp.grid.horner_rows);
    }
    __syncwarp();
    const double sr = (c.x * scale_lo) * scale_hi, si = (c.y * scale_lo) * scale_hi;
    const int base = local[2] * pad01 + local[1] * pad0 + local[0];
#pragma unroll 4
    for (int q = 0; q < R; ++q) {
      const int u = lane + 32 * q;
      if (u < kCells) {
        const int i = u % W, j = (u / W) % W, k = u / (W * W);
        const double weight = stage[warp][0][i] * stage[warp][1][j] * stage[warp][2][k];
        const int cell = base + k * pad01 + j * pad0 + i;
        F64Traits::add(acc, padded, 0, cell, sr * weight);
        F64Traits::add(acc, padded, 1, cell, si * weight);
      }
    }
  }
}

// Resident CTAs per SM that the register budget is sized for: four for the
// 2D f64 warp spreader, three for narrow windows without register runs, two for
// register runs, other f64 windows and the 3D warp spreader.
template <int D, int W, typename T>
__host__ __device__ constexpr int spread_min_blocks() {
  if (D == 2 && sizeof(typename T::Real) == 8 && spread_run<D, W, T>() == 1 && W >= 5) return 4;
  return (spread_run<D, W, T>() > 1 || sizeof(typename T::Real) == 8 || warp_capable<D, W, T>()) ? 2 : 3;
}

// Spreads part `part` of vector `b` (one CTA): the part's records into a
// padded tile of fixed-point sums, written out in floating point. Called
// once per CTA by spread_tiles_kernel, and per work item by the persistent
// kernel of many problems (batch.cu), whose CTAs run it again and again.
template <int D, int W, typename T>
__device__ __forceinline__ void spread_part(
    const SpreadParams& sp, const typename T::Real* __restrict__ points, const void* __restrict__ windows,
    const typename T::Complex* __restrict__ strengths, int64_t point_count, int batch,
    const uint32_t* __restrict__ perm, const uint32_t* __restrict__ offsets,
    const uint32_t* __restrict__ part_start, const typename T::Bits* __restrict__ max_bits,
    typename T::Complex* __restrict__ scratch, uint32_t part, int b) {
  using Real = typename T::Real;
  using Word = typename T::Word;
  extern __shared__ __align__(16) unsigned char shared_bytes[];
  Word* acc = reinterpret_cast<Word*>(shared_bytes);
  __shared__ uint32_t row_begin[kMaxTileRows];
  __shared__ uint32_t row_prefix[kMaxTileRows + 1];
  __shared__ int64_t s_tile;
  __shared__ uint32_t warp_totals[kSpreadThreads / 32];

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
  // The shared tile: dense (span = padded) or with the warp path's pitches.
  constexpr bool kWarpCapable = warp_capable<D, W, T>();
  const bool warp_path = kWarpCapable && sp.span > 0;
  const int span = warp_path ? sp.span : padded;
  {
    // Cleared 16 bytes at a time (the tile's words are a multiple of 16 bytes).
    static_assert(T::kWordsPerCell * sizeof(Word) % 16 == 0, "tile words clear in 16-byte units");
    uint4* acc16 = reinterpret_cast<uint4*>(acc);
    const int units = static_cast<int>(T::kWordsPerCell * sizeof(Word) / 16) * span;
    for (int c = tid; c < units; c += kSpreadThreads) acc16[c] = make_uint4(0u, 0u, 0u, 0u);
  }
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
  const uint32_t part_cap = static_cast<uint32_t>(part_cap_of(sp));
  const uint32_t record_begin = part_in_tile * part_cap;
  const uint32_t record_end = min(tile_total, record_begin + part_cap);
  // Runs of records with one support start add up in registers first (a
  // fixed order within the run) and reach the fixed-point tile once per run,
  // which leaves that much headroom in the scale.
  constexpr int kRun = spread_run<D, W, T>();
  __shared__ uint32_t sorted[kWarpCapable ? kWarpMaxRecords : 1];
  __shared__ __align__(16) float stage[kWarpCapable ? kSpreadWarps : 1][kWarpGroup][kStageStride];
  const int tile_cells = sp.tile[0] * sp.tile[1] * sp.tile[2];
  const bool bucket = warp_path && record_end - record_begin <= static_cast<uint32_t>(kWarpMaxRecords) &&
                      (tile_cells + 1) * kSpreadWarps <= T::kWordsPerCell * span &&
                      tile_total >= static_cast<uint32_t>(tile_cells);
  int S = T::exponent(max_bits[b]) - (kRun > 1 ? kRunBits : 0);
  const Real scale_lo = T::power_of_two(S / 2);
  const Real scale_hi = T::power_of_two(S - S / 2);
  const typename T::Complex* sv = strengths + static_cast<int64_t>(b) * point_count;

  int row = 0;
  if constexpr (kWarpCapable) {
    if (warp_path) {
      spread_warp3<W>(sp, static_cast<const PreparedWindow<3>*>(windows), sv, perm, row_begin, row_prefix, rows,
                      origin, record_begin, record_end, bucket, acc, span, sorted, stage,
                      T::exponent(max_bits[b]), S);
    }
  }
  constexpr bool kWarp64 = D >= 2 && sizeof(Real) == 8 && kRun == 1 && W >= 5;
  __shared__ double stage64[kWarp64 ? kSpreadWarps : 1][kWarp64 ? D : 1][kWarp64 ? W : 1];
  if constexpr (kWarp64 && D == 2) {
    spread_warp2_f64<W>(sp, reinterpret_cast<const double*>(points), reinterpret_cast<const double2*>(sv), perm,
                        row_begin, row_prefix, rows, origin, record_begin, record_end,
                        reinterpret_cast<unsigned long long*>(acc), padded, stage64, scale_lo, scale_hi);
  }
  if constexpr (kWarp64 && D == 3) {
    spread_warp3_f64<W>(sp, reinterpret_cast<const double*>(points), reinterpret_cast<const double2*>(sv), perm,
                        row_begin, row_prefix, rows, origin, record_begin, record_end,
                        reinterpret_cast<unsigned long long*>(acc), padded, stage64, scale_lo, scale_hi);
  }
  if constexpr (kRun == 1 && !kWarp64) {
    for (uint32_t r = record_begin + tid; !warp_path && r < record_end; r += kSpreadThreads) {
      int local_start[D];
      Real w[D][W];
      typename T::Complex s;
      if (!tile_record<D, W, T>(sp, points, windows, sv, perm, row_begin, row_prefix, rows, origin, r, row,
                                local_start, w, s)) {
        continue;
      }
      const Real sr = (s.x * scale_lo) * scale_hi;
      const Real si = (s.y * scale_lo) * scale_hi;
      if (D == 1) {
#pragma unroll
        for (int i = 0; i < W; ++i) {
          const int c = local_start[0] + i;
          T::add(acc, padded, 0, c, sr * w[0][i]);
          T::add(acc, padded, 1, c, si * w[0][i]);
        }
      } else if (D == 2) {
#pragma unroll
        for (int j = 0; j < W; ++j) {
          const Real wr = sr * w[1][j];
          const Real wi = si * w[1][j];
          const int base = (local_start[1] + j) * sp.pad[0] + local_start[0];
#pragma unroll
          for (int i = 0; i < W; ++i) {
            T::add(acc, padded, 0, base + i, wr * w[0][i]);
            T::add(acc, padded, 1, base + i, wi * w[0][i]);
          }
        }
      } else {
#pragma unroll 1
        for (int k = 0; k < W; ++k) {
#pragma unroll
          for (int j = 0; j < W; ++j) {
            const Real wyz = w[1][j] * w[2][k];
            const Real wr = sr * wyz;
            const Real wi = si * wyz;
            const int base =
                ((local_start[2] + k) * sp.pad[1] + local_start[1] + j) * sp.pad[0] + local_start[0];
#pragma unroll
            for (int i = 0; i < W; ++i) {
              T::add(acc, padded, 0, base + i, wr * w[0][i]);
              T::add(acc, padded, 1, base + i, wi * w[0][i]);
            }
          }
        }
      }
    }
  } else if constexpr (kRun > 1) {
    // Each thread takes runs of up to kRun consecutive records (consecutive
    // slots of one bin row share starts when bins are one cell wide), sized so
    // that every pass gives every thread the same number of records.
    constexpr int R = D == 2 ? W : 1;
    const uint32_t count = record_end - record_begin;
    const uint32_t per_thread = (count + kSpreadThreads - 1) / kSpreadThreads;
    const uint32_t passes = (per_thread + kRun - 1) / kRun;
    const uint32_t run = passes ? (count + kSpreadThreads * passes - 1) / (kSpreadThreads * passes) : 1u;
    for (uint32_t first = record_begin + tid * run; first < record_end; first += kSpreadThreads * run) {
      const uint32_t stop = min(first + run, record_end);
      typename T::Complex a2[R][W];  // (re, im) register sums of the run
#pragma unroll
      for (int j = 0; j < R; ++j) {
#pragma unroll
        for (int i = 0; i < W; ++i) a2[j][i].x = a2[j][i].y = Real(0);
      }
      int run0 = -1, run1 = 0;
      // f32: records are loaded ahead of their use, so the load latency
      // overlaps the work on earlier records: the window and point index two
      // records ahead and the strength one ahead (one and zero ahead for
      // windows wider than 6, whose accumulators leave no registers for it).
      constexpr bool kTwoAhead = 2 * W * W * sizeof(Real) < 392;
      PreparedWindow<D> win0{}, win1{};
      uint32_t point0 = 0, point1 = 0;
      typename T::Complex s0{};
      if constexpr (T::kPreparedWindows) {
        if (first < stop) {
          const uint32_t slot = record_slot(first, row, row_begin, row_prefix, rows);
          win0 = static_cast<const PreparedWindow<D>*>(windows)[slot];
          point0 = perm[slot];
          if (kTwoAhead) s0 = sv[point0];
        }
        if (kTwoAhead && first + 1 < stop) {
          const uint32_t slot = record_slot(first + 1, row, row_begin, row_prefix, rows);
          win1 = static_cast<const PreparedWindow<D>*>(windows)[slot];
          point1 = perm[slot];
        }
      }
      for (uint32_t r = first; r < stop; ++r) {
        int local_start[D];
        Real w[D][W];
        typename T::Complex s;
        if constexpr (T::kPreparedWindows) {
          const PreparedWindow<D> win = win0;
          if constexpr (kTwoAhead) {
            s = s0;
            if (r + 1 < stop) s0 = sv[point1];
            win0 = win1;
            if (r + 2 < stop) {
              const uint32_t slot = record_slot(r + 2, row, row_begin, row_prefix, rows);
              win1 = static_cast<const PreparedWindow<D>*>(windows)[slot];
              point1 = perm[slot];
            }
          } else {
            const uint32_t point = point0;
            if (r + 1 < stop) {
              const uint32_t slot = record_slot(r + 1, row, row_begin, row_prefix, rows);
              win0 = static_cast<const PreparedWindow<D>*>(windows)[slot];
              point0 = perm[slot];
            }
            s = sv[point];
          }
          if (!prepared_record<D, W>(sp, win, origin, local_start, w)) continue;
        } else {
          if (!tile_record<D, W, T>(sp, points, windows, sv, perm, row_begin, row_prefix, rows, origin, r,
                                    row, local_start, w, s)) {
            continue;
          }
        }
        // The strength in the fixed-point scale (a power of two: exact), so
        // the run sums reach the tile without another product.
        s = cscale(cscale(s, scale_lo), scale_hi);
        const int l1 = D == 2 ? local_start[D - 1] : 0;
        if constexpr (D == 2) {
          const int l0 = local_start[0];
          if (run0 >= 0 && l1 == run1 && l0 > run0 && l0 < run0 + W) {
            // Same row, a few columns on: flush and drop the passed columns.
            for (; run0 < l0; ++run0) flush_first_column<W, T>(acc, padded, sp.pad[0], run0, run1, a2);
          } else if (l0 != run0 || l1 != run1) {
            if (run0 >= 0) flush_run<D, W, T>(acc, padded, sp.pad[0], run0, run1, a2);
            run0 = l0;
            run1 = l1;
          }
        } else if (local_start[0] != run0 || l1 != run1) {
          if (run0 >= 0) flush_run<D, W, T>(acc, padded, sp.pad[0], run0, run1, a2);
          run0 = local_start[0];
          run1 = l1;
        }
#pragma unroll
        for (int j = 0; j < R; ++j) {
          const typename T::Complex wj = D == 2 ? cscale(s, w[D - 1][j]) : s;
#pragma unroll
          for (int i = 0; i < W; ++i) a2[j][i] = cfma(wj, w[0][i], a2[j][i]);
        }
      }
      if (run0 >= 0) flush_run<D, W, T>(acc, padded, sp.pad[0], run0, run1, a2);
    }
  }
  __syncthreads();
  typename T::Complex* out = scratch + (static_cast<int64_t>(part) * batch + b) * padded;
  if (warp_path) {
    // The thread's cells c = tid + k kSpreadThreads: (x, y, z) stepped by
    // the stride's own coordinates with one carry per axis, not divided.
    const int pad0 = sp.pad[0], pad1 = sp.pad[1], pad01 = sp.pad[0] * sp.pad[1];
    int z = tid / pad01, y = (tid - z * pad01) / pad0;
    int x = tid - z * pad01 - y * pad0;
    const int step_z = kSpreadThreads / pad01, step_y = (kSpreadThreads - step_z * pad01) / pad0;
    const int step_x = kSpreadThreads - step_z * pad01 - step_y * pad0;
    for (int c = tid; c < padded; c += kSpreadThreads) {
      const int at = x + y * sp.pitch0 + z * sp.pitch01;
      typename T::Complex v;
      v.x = T::value(acc, span, 0, at, S);
      v.y = T::value(acc, span, 1, at, S);
      out[c] = v;
      x += step_x;
      y += step_y;
      z += step_z;
      if (x >= pad0) {
        x -= pad0;
        ++y;
      }
      if (y >= pad1) {
        y -= pad1;
        ++z;
      }
    }
    return;
  }
  for (int c = tid; c < padded; c += kSpreadThreads) {
    typename T::Complex v;
    v.x = T::value(acc, padded, 0, c, S);
    v.y = T::value(acc, padded, 1, c, S);
    out[c] = v;
  }
}

// One CTA per (part, vector).
template <int D, int W, typename T>
__global__ void __launch_bounds__(kSpreadThreads, spread_min_blocks<D, W, T>()) spread_tiles_kernel(
    SpreadParams sp, const typename T::Real* __restrict__ points, const void* __restrict__ windows,
    const typename T::Complex* __restrict__ strengths, int64_t point_count, int batch,
    const uint32_t* __restrict__ perm, const uint32_t* __restrict__ offsets,
    const uint32_t* __restrict__ part_start, const typename T::Bits* __restrict__ max_bits,
    typename T::Complex* __restrict__ scratch) {
  spread_part<D, W, T>(sp, points, windows, strengths, point_count, batch, perm, offsets, part_start, max_bits,
                       scratch, blockIdx.x, blockIdx.y);
}

constexpr int kFoldThreads = 256;

// Every fine-grid cell as the sum, in a fixed order, of the padded tiles and
// parts that cover it.
template <int D, int BB, typename Complex>
__global__ void fold_tiles_kernel(SpreadParams sp, int batch, const Complex* __restrict__ scratch,
                                  const uint32_t* __restrict__ part_start, int64_t part_limit,
                                  const int2* __restrict__ candidates,
                                  Complex* __restrict__ fine) {
  // Each thread sums one cell of BB consecutive vectors, so the candidate
  // lookups are shared and the vectors' loads are independent. A CTA covers
  // kFoldThreads consecutive cells of one x row: the row and its (y, z) are
  // found once per CTA with 32-bit arithmetic.
  const uint32_t chunks = (static_cast<uint32_t>(sp.grid.fine[0]) + kFoldThreads - 1) / kFoldThreads;
  const uint32_t row = blockIdx.x / chunks;
  const int x = static_cast<int>((blockIdx.x - row * chunks) * kFoldThreads + threadIdx.x);
  if (x >= sp.grid.fine[0]) return;
  const int64_t cell = x + sp.grid.fine[0] * static_cast<int64_t>(row);
  const int b0 = blockIdx.y * BB;
  int coord[3] = {x, 0, 0};
  if (D == 2) coord[1] = static_cast<int>(row);
  if (D == 3) {
    const uint32_t f1 = static_cast<uint32_t>(sp.grid.fine[1]);
    coord[2] = static_cast<int>(row / f1);
    coord[1] = static_cast<int>(row - static_cast<uint32_t>(coord[2]) * f1);
  }
  const int2* c0 = candidates + sp.candidate_base[0] + coord[0] * sp.candidate_count[0];
  const int2* c1 = D > 1 ? candidates + sp.candidate_base[1] + coord[1] * sp.candidate_count[1] : nullptr;
  const int2* c2 = D > 2 ? candidates + sp.candidate_base[2] + coord[2] * sp.candidate_count[2] : nullptr;
  const int k2n = D > 2 ? sp.candidate_count[2] : 1;
  const int k1n = D > 1 ? sp.candidate_count[1] : 1;
  const int active = min(BB, batch - b0);
  Complex sum[BB];
#pragma unroll
  for (int i = 0; i < BB; ++i) {
    sum[i].x = 0;
    sum[i].y = 0;
  }
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
        for (uint32_t p = first; p < last; ++p) {
          const Complex* v = scratch + (static_cast<int64_t>(p) * batch + b0) * sp.padded_cells + local;
#pragma unroll
          for (int i = 0; i < BB; ++i) {
            if (i < active) {
              const Complex x = v[static_cast<int64_t>(i) * sp.padded_cells];
              sum[i].x += x.x;
              sum[i].y += x.y;
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int i = 0; i < BB; ++i) {
    if (i < active) fine[static_cast<int64_t>(b0 + i) * sp.grid.fine_count + cell] = sum[i];
  }
}

// The fold per destination tile (SpreadParams::dest_fold): a CTA of 256
// threads takes kDestCells planes of a 16 x 16-cell tile plane stack, a
// thread the cells (x, y, z0 .. z0 + kDestCells - 1). The CTA walks the
// covering source tiles in the order of the candidates of the tile's first
// cell along each axis (z outermost) and each source tile's parts in order;
// a thread adds a part's value to each of its cells that the source tile
// covers. Every cell's candidates are an ordered part of those lists, so each
// cell gets the row fold's sums in the row fold's order, bit for bit; the
// thread's loads of one part are independent of one another.
constexpr int kDestCells = 4;

template <typename Complex>
__global__ void __launch_bounds__(256) fold_dest_kernel(SpreadParams sp, int batch,
                                                        const Complex* __restrict__ scratch,
                                                        const uint32_t* __restrict__ part_start, int64_t part_limit,
                                                        const int2* __restrict__ candidates,
                                                        Complex* __restrict__ fine) {
  const int slices = sp.tile[2] / kDestCells;
  const uint32_t tile = blockIdx.x / static_cast<uint32_t>(slices);
  const int slice = static_cast<int>(blockIdx.x - tile * static_cast<uint32_t>(slices));
  const int b = blockIdx.y;
  const uint32_t n0t = static_cast<uint32_t>(sp.ntiles[0]), n1t = static_cast<uint32_t>(sp.ntiles[1]);
  const int t0 = static_cast<int>(tile % n0t);
  const int t1 = static_cast<int>((tile / n0t) % n1t);
  const int t2 = static_cast<int>(tile / (n0t * n1t));
  const int x = t0 * 16 + static_cast<int>(threadIdx.x & 15);
  const int y = t1 * 16 + static_cast<int>(threadIdx.x >> 4);
  const int z0 = t2 * sp.tile[2] + slice * kDestCells;
  const int n0 = sp.grid.fine[0], n1 = sp.grid.fine[1], n2 = sp.grid.fine[2];
  // The source tiles of each axis: the candidates of the tile's first cell.
  int src[3][2];
  const int first_cell[3] = {t0 * 16, t1 * 16, t2 * sp.tile[2]};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const int2* c = candidates + sp.candidate_base[a] + static_cast<int64_t>(first_cell[a]) * sp.candidate_count[a];
    src[a][0] = c[0].x;
    src[a][1] = sp.candidate_count[a] > 1 ? c[1].x : -1;
  }
  // A cell's local offset in each source tile along an axis; -1 where that
  // tile does not cover it.
  auto offsets = [&](int a, int cell, int& o0, int& o1) {
    o0 = -1;
    o1 = -1;
    const int2* c = candidates + sp.candidate_base[a] + static_cast<int64_t>(cell) * sp.candidate_count[a];
    const int k = sp.candidate_count[a] > 1 ? 2 : 1;
    for (int i = 0; i < k; ++i) {
      const int2 e = c[i];
      if (e.x < 0) break;
      if (e.x == src[a][0]) o0 = e.y;
      else if (e.x == src[a][1]) o1 = e.y;
    }
  };
  const bool xy_inside = x < n0 && y < n1;
  int ox[2] = {-1, -1}, oy[2] = {-1, -1};
  if (xy_inside) {
    offsets(0, x, ox[0], ox[1]);
    offsets(1, y, oy[0], oy[1]);
  }
  int oz[kDestCells][2];
#pragma unroll
  for (int k = 0; k < kDestCells; ++k) {
    oz[k][0] = -1;
    oz[k][1] = -1;
    if (z0 + k < n2) offsets(2, z0 + k, oz[k][0], oz[k][1]);
  }
  Complex sum[kDestCells];
#pragma unroll
  for (int k = 0; k < kDestCells; ++k) {
    sum[k].x = 0;
    sum[k].y = 0;
  }
  const int plane = sp.pad[0] * sp.pad[1];
#pragma unroll
  for (int u2 = 0; u2 < 2; ++u2) {
    if (src[2][u2] < 0) continue;
    bool any_z = false;
#pragma unroll
    for (int k = 0; k < kDestCells; ++k) any_z = any_z || oz[k][u2] >= 0;
    if (!any_z) continue;  // the same for the whole CTA
#pragma unroll
    for (int u1 = 0; u1 < 2; ++u1) {
      if (src[1][u1] < 0) continue;
#pragma unroll
      for (int u0 = 0; u0 < 2; ++u0) {
        if (src[0][u0] < 0) continue;
        const int64_t source = src[0][u0] + static_cast<int64_t>(sp.ntiles[0]) *
                                                (src[1][u1] + static_cast<int64_t>(sp.ntiles[1]) * src[2][u2]);
        const uint32_t first = part_start[source];
        const uint32_t last = min(part_start[source + 1], static_cast<uint32_t>(part_limit));
        const bool covered = ox[u0] >= 0 && oy[u1] >= 0;
        const int base = ox[u0] + sp.pad[0] * oy[u1];
        int at[kDestCells];
        bool take[kDestCells];
#pragma unroll
        for (int k = 0; k < kDestCells; ++k) {
          take[k] = covered && oz[k][u2] >= 0;
          at[k] = base + plane * oz[k][u2];
        }
        for (uint32_t p = first; p < last; ++p) {
          const Complex* v = scratch + (static_cast<int64_t>(p) * batch + b) * sp.padded_cells;
          Complex got[kDestCells];
#pragma unroll
          for (int k = 0; k < kDestCells; ++k) {
            if (take[k]) got[k] = v[at[k]];
          }
#pragma unroll
          for (int k = 0; k < kDestCells; ++k) {
            if (take[k]) {
              sum[k].x += got[k].x;
              sum[k].y += got[k].y;
            }
          }
        }
      }
    }
  }
  if (!xy_inside) return;
#pragma unroll
  for (int k = 0; k < kDestCells; ++k) {
    if (z0 + k < n2) {
      fine[static_cast<int64_t>(b) * sp.grid.fine_count + x + static_cast<int64_t>(n0) * (y + static_cast<int64_t>(n1) * (z0 + k))] = sum[k];
    }
  }
}

// Grids of at most kWarpFoldCells cells fold a cell per warp. Small grids
// holding many points have hundreds of parts per tile, and a thread walking
// them one after another would leave the GPU idle: here the lanes take every
// 32nd part of each covering tile, in order, and a fixed butterfly adds the
// 32 lane sums (every lane ends with the same bits). The order depends on the
// grid alone, so single vectors and batches agree bit for bit.
constexpr int kWarpFoldThreads = 256;

template <int D, typename Complex>
__global__ void __launch_bounds__(kWarpFoldThreads) fold_cells_warp_kernel(
    SpreadParams sp, int batch, const Complex* __restrict__ scratch, const uint32_t* __restrict__ part_start,
    int64_t part_limit, const int2* __restrict__ candidates, Complex* __restrict__ fine) {
  const int lane = threadIdx.x & 31;
  const int64_t cell = (static_cast<int64_t>(blockIdx.x) * kWarpFoldThreads + threadIdx.x) >> 5;
  if (cell >= sp.grid.fine_count) return;  // the whole warp leaves together
  int coord[3] = {0, 0, 0};
  int64_t rest = cell;
  for (int a = 0; a < D; ++a) {
    coord[a] = static_cast<int>(rest % sp.grid.fine[a]);
    rest /= sp.grid.fine[a];
  }
  const int2* c0 = candidates + sp.candidate_base[0] + coord[0] * sp.candidate_count[0];
  const int2* c1 = D > 1 ? candidates + sp.candidate_base[1] + coord[1] * sp.candidate_count[1] : nullptr;
  const int2* c2 = D > 2 ? candidates + sp.candidate_base[2] + coord[2] * sp.candidate_count[2] : nullptr;
  const int k2n = D > 2 ? sp.candidate_count[2] : 1;
  const int k1n = D > 1 ? sp.candidate_count[1] : 1;
  for (int b = blockIdx.y; b < batch; b += gridDim.y) {
    Complex sum;
    sum.x = 0;
    sum.y = 0;
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
          for (uint32_t p = first + lane; p < last; p += 32) {
            const Complex v = scratch[(static_cast<int64_t>(p) * batch + b) * sp.padded_cells + local];
            sum.x += v.x;
            sum.y += v.y;
          }
        }
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sum.x += __shfl_xor_sync(0xffffffffu, sum.x, o);
      sum.y += __shfl_xor_sync(0xffffffffu, sum.y, o);
    }
    if (lane == 0) fine[static_cast<int64_t>(b) * sp.grid.fine_count + cell] = sum;
  }
}

template <typename Complex>
void launch_warp_fold(const SpreadParams& sp, int batch, const Complex* scratch, const uint32_t* part_start,
                      int64_t part_limit, const int2* candidates, Complex* fine, cudaStream_t stream) {
  constexpr int kCellsPerCta = kWarpFoldThreads / 32;
  const dim3 grid(static_cast<unsigned>((sp.grid.fine_count + kCellsPerCta - 1) / kCellsPerCta),
                  static_cast<unsigned>(std::min(batch, 65535)));
  switch (sp.grid.dimensions) {
    case 1:
      fold_cells_warp_kernel<1, Complex><<<grid, kWarpFoldThreads, 0, stream>>>(sp, batch, scratch, part_start,
                                                                                part_limit, candidates, fine);
      break;
    case 2:
      fold_cells_warp_kernel<2, Complex><<<grid, kWarpFoldThreads, 0, stream>>>(sp, batch, scratch, part_start,
                                                                                part_limit, candidates, fine);
      break;
    default:
      fold_cells_warp_kernel<3, Complex><<<grid, kWarpFoldThreads, 0, stream>>>(sp, batch, scratch, part_start,
                                                                                part_limit, candidates, fine);
      break;
  }
  note_launch();
}

template <int BB, typename Complex>
void launch_fold(const SpreadParams& sp, int batch, const Complex* scratch, const uint32_t* part_start,
                 int64_t part_limit, const int2* candidates, Complex* fine, cudaStream_t stream) {
  // One CTA per kFoldThreads cells of an x row.
  int64_t rows = 1;
  for (int a = 1; a < sp.grid.dimensions; ++a) rows *= sp.grid.fine[a];
  const int64_t chunks = (sp.grid.fine[0] + kFoldThreads - 1) / kFoldThreads;
  const dim3 grid(static_cast<unsigned>(rows * chunks), static_cast<unsigned>((batch + BB - 1) / BB));
  switch (sp.grid.dimensions) {
    case 1:
      fold_tiles_kernel<1, BB, Complex><<<grid, kFoldThreads, 0, stream>>>(sp, batch, scratch, part_start,
                                                                           part_limit, candidates, fine);
      break;
    case 2:
      fold_tiles_kernel<2, BB, Complex><<<grid, kFoldThreads, 0, stream>>>(sp, batch, scratch, part_start,
                                                                           part_limit, candidates, fine);
      break;
    default:
      fold_tiles_kernel<3, BB, Complex><<<grid, kFoldThreads, 0, stream>>>(sp, batch, scratch, part_start,
                                                                           part_limit, candidates, fine);
      break;
  }
  note_launch();
}

// Vectors per fold thread: one for a single vector, eight for batches.
template <typename Complex>
void fold_any(const SpreadParams& sp, int batch, const Complex* scratch, const uint32_t* part_start,
              int64_t part_limit, const int2* candidates, Complex* fine, cudaStream_t stream) {
  if (sp.grid.fine_count <= kWarpFoldCells) {
    launch_warp_fold(sp, batch, scratch, part_start, part_limit, candidates, fine, stream);
  } else if (sp.dest_fold && batch < 8) {
    const dim3 grid(static_cast<unsigned>(sp.tile_count * (sp.tile[2] / kDestCells)), static_cast<unsigned>(batch));
    fold_dest_kernel<Complex><<<grid, 256, 0, stream>>>(sp, batch, scratch, part_start, part_limit, candidates, fine);
    note_launch();
  } else if (batch >= 8) {
    launch_fold<8>(sp, batch, scratch, part_start, part_limit, candidates, fine, stream);
  } else {
    launch_fold<1>(sp, batch, scratch, part_start, part_limit, candidates, fine, stream);
  }
}

template <int D, int W, typename T>
void launch_spread_width(const SpreadParams& sp, const SpreadLaunchT<T>& l, cudaStream_t stream) {
  const int span = warp_capable<D, W, T>() && sp.span > 0 ? sp.span : sp.padded_cells;
  const size_t smem = static_cast<size_t>(T::kWordsPerCell) * span * sizeof(typename T::Word);
  auto kernel = spread_tiles_kernel<D, W, T>;
  check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  static_cast<int>(smem)),
             "spread shared memory");
  const dim3 grid(static_cast<unsigned>(l.part_upper_bound), static_cast<unsigned>(l.batch));
  kernel<<<grid, kSpreadThreads, smem, stream>>>(sp, l.points, l.windows, l.strengths, l.point_count, l.batch,
                                                 l.perm, l.offsets, l.part_start, l.max_bits,
                                                 l.scratch);
  note_launch();
}

template <int D, typename T>
void launch_spread_dim(const SpreadParams& sp, const SpreadLaunchT<T>& l, cudaStream_t stream) {
  switch (sp.grid.width) {
    case 2: launch_spread_width<D, 2, T>(sp, l, stream); break;
    case 3: launch_spread_width<D, 3, T>(sp, l, stream); break;
    case 4: launch_spread_width<D, 4, T>(sp, l, stream); break;
    case 5: launch_spread_width<D, 5, T>(sp, l, stream); break;
    case 6: launch_spread_width<D, 6, T>(sp, l, stream); break;
    case 7: launch_spread_width<D, 7, T>(sp, l, stream); break;
    case 8: launch_spread_width<D, 8, T>(sp, l, stream); break;
    case 9: launch_spread_width<D, 9, T>(sp, l, stream); break;
    case 10: launch_spread_width<D, 10, T>(sp, l, stream); break;
    case 11: launch_spread_width<D, 11, T>(sp, l, stream); break;
    case 12: launch_spread_width<D, 12, T>(sp, l, stream); break;
    case 13: launch_spread_width<D, 13, T>(sp, l, stream); break;
    case 14: launch_spread_width<D, 14, T>(sp, l, stream); break;
    case 15: launch_spread_width<D, 15, T>(sp, l, stream); break;
    default: launch_spread_width<D, 16, T>(sp, l, stream); break;
  }
}

template <typename T>
void spread_execute_impl(const SpreadParams& sp, const SpreadLaunchT<T>& l, cudaStream_t stream,
                         StageTimer* timer) {
  if (l.point_count > 0) {
    {
      StageScope scope(timer, kStageStrengthScale, stream);
      check_cuda(cudaMemsetAsync(l.max_bits, 0, sizeof(typename T::Bits) * l.batch, stream),
                 "clear maxima");
      const unsigned blocks =
          static_cast<unsigned>(std::min<int64_t>((l.point_count + 1023) / 1024, 148 * 8));
      strength_magnitude_kernel<T><<<dim3(blocks, l.batch), 256, 0, stream>>>(
          l.strengths, l.point_count, l.batch, l.max_bits, l.valid_mask);
      note_launch();
    }
    StageScope scope(timer, kStageSpread, stream);
    switch (sp.grid.dimensions) {
      case 1: launch_spread_dim<1, T>(sp, l, stream); break;
      case 2: launch_spread_dim<2, T>(sp, l, stream); break;
      default: launch_spread_dim<3, T>(sp, l, stream); break;
    }
  }
  // A null fine grid leaves the padded tiles for a fused fold (fused_fft.cu).
  if (l.fine == nullptr) return;
  StageScope scope(timer, kStageFold, stream);
  fold_any(sp, l.batch, l.scratch, l.part_start, l.part_upper_bound, l.candidates, l.fine, stream);
}

// ---------------------------------------------------------------------------
// Many independent problems from one persistent launch.

// Work list: work[p] = first item of problem p (its parts, in order), work[count]
// = all items; work[count + 1] = the queue counter. Clears the scale words.
__global__ void __launch_bounds__(1024) batch_work_kernel(const BatchProblem* __restrict__ problems, int count,
                                                          uint32_t* __restrict__ work) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t carry_shared;
  if (threadIdx.x == 0) carry_shared = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base = 0; base < count; base += 1024) {
    const int p = base + threadIdx.x;
    uint32_t v = 0;
    if (p < count) {
      const BatchProblem& bp = problems[p];
      v = bp.point_count > 0 ? bp.part_start[bp.sp.tile_count] : 0u;
      *bp.max_bits = 0u;
    }
    uint32_t x = v;
#pragma unroll
    for (int offset = 1; offset < 32; offset <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, offset);
      if (lane >= offset) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t t = warp_sums[lane];
#pragma unroll
      for (int offset = 1; offset < 32; offset <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, t, offset);
        if (lane >= offset) t += y;
      }
      warp_sums[lane] = t;
    }
    __syncthreads();
    const uint32_t carry = carry_shared;
    const uint32_t inclusive = x + (warp > 0 ? warp_sums[warp - 1] : 0u);
    if (p < count) work[p] = carry + inclusive - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry_shared = carry + inclusive;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    work[count] = carry_shared;
    work[count + 1] = 0u;
  }
}

// Largest |re| or |im| of every problem's strengths over its points within
// reach (blockIdx.y = problem).
__global__ void batch_magnitude_kernel(const BatchProblem* __restrict__ problems, const __grid_constant__ BatchStrengths strengths) {
  const BatchProblem& bp = problems[blockIdx.y];
  const float2* v = strengths.ptr[blockIdx.y];
  const int64_t count = bp.point_count;
  const uint32_t* valid_mask = bp.valid_mask;
  uint32_t m = 0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < count; i += stride) {
    if (valid_mask != nullptr && !((__ldg(&valid_mask[i >> 5]) >> (i & 31)) & 1u)) continue;
    const float2 s = v[i];
    m = max(m, F32Traits::magnitude_bits(s.x));
    m = max(m, F32Traits::magnitude_bits(s.y));
  }
#pragma unroll
  for (int offset = 16; offset > 0; offset >>= 1) m = max(m, __shfl_xor_sync(0xFFFFFFFFu, m, offset));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(bp.max_bits, m);
}

// Persistent spreading: every CTA takes the next (problem, part) item from
// the queue counter until none is left, copies that problem's parameters
// into shared memory and spreads the part as spread_tiles_kernel does, so
// each problem's padded tiles are the same bits as from its own launch.
template <int W, bool Has2D, bool Has3D>
__global__ void __launch_bounds__(kSpreadThreads, 1) batch_spread_kernel(const BatchProblem* __restrict__ problems,
                                                                         const __grid_constant__ BatchStrengths strengths,
                                                                         int count, uint32_t* __restrict__ work) {
  __shared__ __align__(16) SpreadParams s_sp;
  __shared__ uint32_t s_item;
  const uint32_t total = work[count];
  for (;;) {
    __syncthreads();  // the previous item's tile and parameters are no longer read
    if (threadIdx.x == 0) s_item = atomicAdd(&work[count + 1], 1u);
    __syncthreads();
    const uint32_t item = s_item;
    if (item >= total) break;
    // The problem whose items include `item` (last start at or below it).
    int low = 0, high = count - 1;
    while (low < high) {
      const int mid = (low + high + 1) >> 1;
      if (work[mid] <= item) low = mid; else high = mid - 1;
    }
    const BatchProblem* bp = problems + low;
    {
      const uint32_t* src = reinterpret_cast<const uint32_t*>(&bp->sp);
      uint32_t* dst = reinterpret_cast<uint32_t*>(&s_sp);
      for (int i = threadIdx.x; i < static_cast<int>(sizeof(SpreadParams) / 4); i += kSpreadThreads) dst[i] = src[i];
    }
    __syncthreads();
    const uint32_t part = item - work[low];
    if constexpr (Has2D) {
      if (s_sp.grid.dimensions == 2) {
        spread_part<2, W, F32Traits>(s_sp, nullptr, bp->windows, strengths.ptr[low], bp->point_count, 1, bp->perm,
                                     bp->offsets, bp->part_start, bp->max_bits, bp->scratch, part, 0);
      }
    }
    if constexpr (Has3D) {
      if (s_sp.grid.dimensions == 3) {
        spread_part<3, W, F32Traits>(s_sp, nullptr, bp->windows, strengths.ptr[low], bp->point_count, 1, bp->perm,
                                     bp->offsets, bp->part_start, bp->max_bits, bp->scratch, part, 0);
      }
    }
  }
}

template <int W>
void launch_batch_spread(const BatchProblem* problems, const BatchStrengths& strengths, int count, bool has_2d,
                         bool has_3d, size_t shared_bytes, uint32_t* work, cudaStream_t stream) {
  auto launch = [&](auto kernel) {
    check_cuda(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    static_cast<int>(shared_bytes)),
               "batch spread shared memory");
    int per_sm = 0;
    check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kSpreadThreads, shared_bytes),
               "batch spread occupancy");
    int sms = 0, device = 0;
    check_cuda(cudaGetDevice(&device), "current device");
    check_cuda(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
    const unsigned grid = static_cast<unsigned>(std::max(1, per_sm) * sms);
    kernel<<<grid, kSpreadThreads, shared_bytes, stream>>>(problems, strengths, count, work);
    note_launch();
  };
  if (has_2d && has_3d) {
    launch(batch_spread_kernel<W, true, true>);
  } else if (has_3d) {
    launch(batch_spread_kernel<W, false, true>);
  } else {
    launch(batch_spread_kernel<W, true, false>);
  }
}

}  // namespace

void batch_spread(const BatchProblem* problems, const BatchStrengths& strengths, int count, int width, bool has_2d,
                  bool has_3d, size_t shared_bytes, uint32_t* work, cudaStream_t stream) {
  if (count <= 0) return;
  if (count > kMaxBatchProblems) throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "too many problems in one batch"};
  batch_work_kernel<<<1, 1024, 0, stream>>>(problems, count, work);
  batch_magnitude_kernel<<<dim3(16, static_cast<unsigned>(count)), 256, 0, stream>>>(problems, strengths);
  note_launch(2);
  switch (width) {
    case 2: launch_batch_spread<2>(problems, strengths, count, has_2d, has_3d, shared_bytes, work, stream); break;
    case 3: launch_batch_spread<3>(problems, strengths, count, has_2d, has_3d, shared_bytes, work, stream); break;
    case 4: launch_batch_spread<4>(problems, strengths, count, has_2d, has_3d, shared_bytes, work, stream); break;
    case 5: launch_batch_spread<5>(problems, strengths, count, has_2d, has_3d, shared_bytes, work, stream); break;
    case 6: launch_batch_spread<6>(problems, strengths, count, has_2d, has_3d, shared_bytes, work, stream); break;
    case 7: launch_batch_spread<7>(problems, strengths, count, has_2d, has_3d, shared_bytes, work, stream); break;
    default: launch_batch_spread<8>(problems, strengths, count, has_2d, has_3d, shared_bytes, work, stream); break;
  }
}

void spread_fold(const SpreadParams& sp, const SpreadLaunch& l, cudaStream_t stream) {
  fold_any(sp, l.batch, l.scratch, l.part_start, l.part_upper_bound, l.candidates, l.fine, stream);
}

size_t spread_shared_bytes(const SpreadParams& sp) {
  const int w = sp.grid.width;
  const bool warp = sp.grid.dimensions == 3 && w >= kWarpMinWidth && w <= kWarpMaxWidth && sp.span > 0;
  return static_cast<size_t>(F32Traits::kWordsPerCell) * (warp ? sp.span : sp.padded_cells) * sizeof(uint32_t);
}

void spread_count_parts(const SpreadParams& sp, const uint32_t* offsets, uint32_t* parts,
                        uint32_t* part_start, cudaStream_t stream, StageTimer* timer) {
  StageScope scope(timer, kStageTileParts, stream);
  if (sp.part_cap_device != nullptr) {
    part_cap_kernel<<<1, 1, 0, stream>>>(sp, offsets);
    note_launch();
  }
  const unsigned blocks = static_cast<unsigned>((sp.tile_count + 255) / 256);
  switch (sp.grid.dimensions) {
    case 1: tile_records_kernel<1><<<blocks, 256, 0, stream>>>(sp, offsets, parts); break;
    case 2: tile_records_kernel<2><<<blocks, 256, 0, stream>>>(sp, offsets, parts); break;
    default: tile_records_kernel<3><<<blocks, 256, 0, stream>>>(sp, offsets, parts); break;
  }
  part_scan_kernel<<<1, 1024, 0, stream>>>(parts, sp.tile_count, part_start);
  note_launch(2);
}

void exclusive_scan_u32(const uint32_t* in, int64_t n, uint32_t* out, cudaStream_t stream) {
  part_scan_kernel<<<1, 1024, 0, stream>>>(in, n, out);
  note_launch();
}

void spread_execute(const SpreadParams& sp, const SpreadLaunch& l, cudaStream_t stream,
                    StageTimer* timer) {
  SpreadLaunchT<F32Traits> t{l.points,   l.windows,  l.strengths,        l.point_count, l.batch,
                             l.perm,     l.offsets,          l.part_start,  l.part_upper_bound,
                             l.max_bits, l.scratch,          l.candidates,  l.fine, l.valid_mask};
  spread_execute_impl<F32Traits>(sp, t, stream, timer);
}

bool spread_warp_layout(int width, const int32_t pad[3], int32_t& pitch0, int32_t& pitch01,
                        uint32_t* table) {
  if (width < kWarpMinWidth || width > kWarpMaxWidth) return false;
  const int L = warp_segment_cells(width);
  const int R = warp_rounds(width);
  const int per_row = width / L;
  int best_banks = 1 << 30;
  int64_t best_cells = 0;
  for (int d0 = 0; d0 < 16; ++d0) {
    for (int d1 = 0; d1 < 32; ++d1) {
      const int p0 = pad[0] + d0;
      const int p01 = p0 * pad[1] + d1;
      int banks[32] = {};
      for (int k = 0; k < width; ++k) {
        for (int j = 0; j < width; ++j) {
          for (int s = 0; s < per_row; ++s) ++banks[(s * L + j * p0 + k * p01) & 31];
        }
      }
      int most = 0;
      for (int v : banks) most = std::max(most, v);
      const int64_t cells = static_cast<int64_t>(p01) * pad[2];
      if (most < best_banks || (most == best_banks && cells < best_cells)) {
        best_banks = most;
        best_cells = cells;
        pitch0 = p0;
        pitch01 = p01;
      }
    }
  }
  if (best_banks > R) return false;
  const int last = (width - 1) * (1 + pitch0 + pitch01);
  if (last > 0xFFFF) return false;
  for (int i = 0; i < R * 32; ++i) table[i] = 0u;
  int filled[32] = {};
  for (int k = 0; k < width; ++k) {
    for (int j = 0; j < width; ++j) {
      for (int s = 0; s < per_row; ++s) {
        const int offset = s * L + j * pitch0 + k * pitch01;
        const int lane = offset & 31;
        table[filled[lane] * 32 + lane] = kSegmentValid | static_cast<uint32_t>(offset) |
                                          (static_cast<uint32_t>(s) << 16) | (static_cast<uint32_t>(j) << 20) |
                                          (static_cast<uint32_t>(k) << 24);
        ++filled[lane];
      }
    }
  }
  return true;
}

void spread_execute64(const SpreadParams& sp, const SpreadLaunch64& l, cudaStream_t stream,
                      StageTimer* timer) {
  SpreadLaunchT<F64Traits> t{l.points,   nullptr,    l.strengths,        l.point_count, l.batch,
                             l.perm,     l.offsets,          l.part_start,  l.part_upper_bound,
                             l.max_bits, l.scratch,          l.candidates,  l.fine, l.valid_mask};
  spread_execute_impl<F64Traits>(sp, t, stream, timer);
}

}  // namespace b200nufft
