// Stable binning of the nonuniform points.
//
// The reference bins points with u32 atomics, a prefix scan, a scatter, a
// merge sort of bins above 64 points and an O(bin^2) ranking of the smaller
// ones (src/gpu_nd_bins.rs:336-709, src/gpu_bin_sort.rs, src/gpu_scan.rs);
// its result is the points sorted by bin key, ties in original index order,
// plus the exclusive scan of the bin counts with a trailing total. Here the
// same order comes from a least-significant-digit radix sort whose passes are
// single kernels with a decoupled look-back across tiles (one pass per 8 key
// bits), which is stable by construction, so no bin needs a second sort
// however clustered the points are. Bin offsets then follow from the sorted
// keys without atomics: the first slot of every bin is where its key begins.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>

#include "device.h"

namespace b200nufft {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortWarps = kSortThreads / 32;
constexpr int kItemsPerThread = 16;
constexpr int kSortTile = kSortThreads * kItemsPerThread;
constexpr int kRadix = 256;
static_assert(kSortTile == kSortTilePoints && kRadix == kSortDigits,
              "sort_status_bytes and fixed scratch sizes assume 4096-point tiles of 256 digits");
constexpr uint32_t kFlagAggregate = 1u << 30;
constexpr uint32_t kFlagInclusive = 2u << 30;
constexpr uint32_t kValueMask = (1u << 30) - 1;
// Polls of a predecessor's look-back word before a tile gives up and flags
// an error (about a second with the back-off below).
constexpr uint32_t kLookbackPollLimit = 1u << 24;

// ---------------------------------------------------------------------------
// Keys.

// Bin key of a point from its support starts (src/gpu_nd_bins.rs:474-554):
// every axis's start is computed only when all coordinates lie within the
// fold's reach; otherwise the point lands in bin 0 of every axis.
template <int D>
__device__ __forceinline__ uint32_t support_start_key(const float* p, const GridParams& g) {
  bool reach = true;
#pragma unroll
  for (int a = 0; a < D; ++a) reach = reach && in_fold_reach(p[a]);
  uint32_t key = 0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    int32_t start = 0;
    if (reach) {
      Df64 offset;
      support_of(p[a], g.axis[a], g.half_width, start, offset);
    }
    const int32_t wrapped = wrap_start(start, g.axis[a].length);
    key += (static_cast<uint32_t>(wrapped) >> g.axis[a].shift) * g.axis[a].stride;
  }
  return key;
}

// Grid cell of a coordinate folded in plain f32 and clamped onto the grid
// (approximate_cell, src/gpu_point_bins.rs:460-464), with the reference's
// operations kept separate.
__device__ __forceinline__ uint32_t approximate_cell(float x, const FoldAxis& a) {
  const float position = __fadd_rn(__fmul_rn(x, a.scale_hi), a.origin);
  const float wrapped =
      __fsub_rn(position, __fmul_rn(a.length_f, floorf(__fdiv_rn(position, a.length_f))));
  const float clamped = fmaxf(wrapped, 0.0f);
  uint32_t cell = clamped >= 4294967040.0f ? 0xFFFFFFFFu : static_cast<uint32_t>(clamped);
  const uint32_t last = static_cast<uint32_t>(a.length - 1);
  return cell < last ? cell : last;
}

template <int D>
__device__ __forceinline__ uint32_t approximate_cell_key(const float* p, const GridParams& g) {
  uint32_t key = 0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    key += (approximate_cell(p[a], g.axis[a]) >> g.axis[a].shift) * g.axis[a].stride;
  }
  return key;
}

// Computes every point's key and the digit histograms of all passes. A warp
// takes 32 consecutive points per iteration; with valid-first keys its
// ballot of the points within reach is one word of `valid_mask`.
template <int D, KeyKind K>
__global__ void __launch_bounds__(256) bin_keys_kernel(const float* __restrict__ points,
                                                       int64_t count, GridParams g,
                                                       uint32_t* __restrict__ keys,
                                                       uint32_t* __restrict__ hist, int passes,
                                                       uint32_t invalid_key, uint32_t* __restrict__ valid_mask) {
  __shared__ uint32_t local[4][kRadix];
  for (int i = threadIdx.x; i < 4 * kRadix; i += blockDim.x) (&local[0][0])[i] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31); base < count;
       base += stride) {
    const int64_t i = base + lane;
    const bool inside = i < count;
    bool reach = false;
    uint32_t key = 0;
    if (inside) {
      float p[D];
#pragma unroll
      for (int a = 0; a < D; ++a) p[a] = points[i * D + a];
      if constexpr (K == KeyKind::ApproximateCell) {
        key = approximate_cell_key<D>(p, g);
      } else {
        key = support_start_key<D>(p, g);
        reach = true;
#pragma unroll
        for (int a = 0; a < D; ++a) reach = reach && in_fold_reach(p[a]);
        if (K == KeyKind::SupportStartValidFirst && !reach) key = invalid_key;
      }
    }
    if constexpr (K == KeyKind::SupportStartValidFirst) {
      const uint32_t ballot = __ballot_sync(0xFFFFFFFFu, reach);
      if (lane == 0) valid_mask[base >> 5] = ballot;
    }
    if (inside) {
      keys[i] = key;
      for (int pass = 0; pass < passes; ++pass) {
        atomicAdd(&local[pass][(key >> (8 * pass)) & 0xFF], 1u);
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x) {
    const uint32_t v = (&local[0][0])[i];
    if (v) atomicAdd(&hist[i], v);
  }
}

// Bin keys of f64 coordinates: the support starts of the native f64 fold,
// with the same reach rule and wrapping as the f32 keys.
template <int D>
__global__ void __launch_bounds__(256) bin_keys64_kernel(const double* __restrict__ points,
                                                         int64_t count, GridParams g,
                                                         uint32_t* __restrict__ keys,
                                                         uint32_t* __restrict__ hist, int passes,
                                                         uint32_t invalid_key, uint32_t* __restrict__ valid_mask) {
  __shared__ uint32_t local[4][kRadix];
  for (int i = threadIdx.x; i < 4 * kRadix; i += blockDim.x) (&local[0][0])[i] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t base = static_cast<int64_t>(blockIdx.x) * blockDim.x + (threadIdx.x & ~31); base < count;
       base += stride) {
    const int64_t i = base + lane;
    const bool inside = i < count;
    bool reach = inside;
    uint32_t key = 0;
    if (inside) {
      double p[D];
#pragma unroll
      for (int a = 0; a < D; ++a) {
        p[a] = points[i * D + a];
        reach = reach && in_fold_reach64(p[a]);
      }
#pragma unroll
      for (int a = 0; a < D; ++a) {
        int32_t start = 0;
        if (reach) {
          double offset;
          support_of64(p[a], g.axis64[a], g.half_width64, start, offset);
        }
        const int32_t wrapped = wrap_start(start, g.axis[a].length);
        key += (static_cast<uint32_t>(wrapped) >> g.axis[a].shift) * g.axis[a].stride;
      }
      if (valid_mask != nullptr && !reach) key = invalid_key;
    }
    if (valid_mask != nullptr) {
      const uint32_t ballot = __ballot_sync(0xFFFFFFFFu, reach);
      if (lane == 0) valid_mask[base >> 5] = ballot;
    }
    if (inside) {
      keys[i] = key;
      for (int pass = 0; pass < passes; ++pass) {
        atomicAdd(&local[pass][(key >> (8 * pass)) & 0xFF], 1u);
      }
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * kRadix; i += blockDim.x) {
    const uint32_t v = (&local[0][0])[i];
    if (v) atomicAdd(&hist[i], v);
  }
}

// Exclusive scan of every pass's 256 digit counts, in place.
__global__ void digit_scan_kernel(uint32_t* hist, int passes) {
  __shared__ uint32_t buffer[kRadix];
  for (int pass = 0; pass < passes; ++pass) {
    const uint32_t v = hist[pass * kRadix + threadIdx.x];
    buffer[threadIdx.x] = v;
    __syncthreads();
    for (int offset = 1; offset < kRadix; offset <<= 1) {
      const uint32_t add = threadIdx.x >= offset ? buffer[threadIdx.x - offset] : 0u;
      __syncthreads();
      buffer[threadIdx.x] += add;
      __syncthreads();
    }
    hist[pass * kRadix + threadIdx.x] = buffer[threadIdx.x] - v;
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// One stable counting pass over 8 key bits.
//
// Tiles take their index from a ticket so that every earlier tile has already
// started; each tile ranks its items within warps (match on the digit, in
// item order), publishes its digit counts, then adds its predecessors'
// counts by looking back until it meets an inclusive prefix. Items go
// through shared memory so that the global stores of one digit are
// contiguous.
__global__ void __launch_bounds__(kSortThreads) onesweep_pass_kernel(
    const uint32_t* __restrict__ keys_in, const uint32_t* __restrict__ vals_in,
    uint32_t* __restrict__ keys_out, uint32_t* __restrict__ vals_out, int64_t count, int shift,
    const uint32_t* __restrict__ digit_base, uint32_t* status, uint32_t* ticket,
    uint32_t* error_flag, int write_keys) {
  __shared__ uint32_t s_tile;
  __shared__ uint32_t warp_counts[kSortWarps][kRadix];
  __shared__ uint32_t s_local_start[kRadix];
  __shared__ uint32_t s_global_start[kRadix];
  __shared__ uint32_t s_keys[kSortTile];
  __shared__ uint32_t s_vals[kSortTile];

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  if (tid == 0) s_tile = atomicAdd(ticket, 1u);
  for (int i = tid; i < kSortWarps * kRadix; i += kSortThreads) (&warp_counts[0][0])[i] = 0;
  __syncthreads();
  const uint32_t tile = s_tile;
  const int64_t tile_base = static_cast<int64_t>(tile) * kSortTile;
  const int64_t warp_base = tile_base + static_cast<int64_t>(warp) * 32 * kItemsPerThread;

  uint32_t key[kItemsPerThread];
  uint32_t val[kItemsPerThread];
  uint32_t rank[kItemsPerThread];
#pragma unroll
  for (int i = 0; i < kItemsPerThread; ++i) {
    const int64_t index = warp_base + i * 32 + lane;
    const bool valid = index < count;
    key[i] = valid ? keys_in[index] : 0u;
    val[i] = valid ? (vals_in ? vals_in[index] : static_cast<uint32_t>(index)) : 0u;
  }
  const uint32_t lane_below = (1u << lane) - 1u;
#pragma unroll
  for (int i = 0; i < kItemsPerThread; ++i) {
    const int64_t index = warp_base + i * 32 + lane;
    const bool valid = index < count;
    const uint32_t active = __ballot_sync(0xFFFFFFFFu, valid);
    const uint32_t digit = (key[i] >> shift) & 0xFFu;
    uint32_t peers = 0, before = 0;
    if (valid) {
      peers = __match_any_sync(active, digit);
      before = warp_counts[warp][digit];
      rank[i] = before + __popc(peers & lane_below);
    }
    __syncwarp();
    if (valid && (31 - __clz(peers)) == lane) warp_counts[warp][digit] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();

  // Per digit: the tile's count, and each warp's exclusive prefix.
  const int digit = tid;
  uint32_t total = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) {
    const uint32_t c = warp_counts[w][digit];
    warp_counts[w][digit] = total;
    total += c;
  }
  // Publish the aggregate (or the inclusive prefix of the first tile).
  volatile uint32_t* my_status = status + static_cast<size_t>(tile) * kRadix + digit;
  if (tile == 0) {
    *my_status = kFlagInclusive | total;
  } else {
    *my_status = kFlagAggregate | total;
  }
  // Exclusive scan of the tile's digit counts: where each digit starts in the
  // tile's shared-memory order.
  s_local_start[digit] = total;
  __syncthreads();
  for (int offset = 1; offset < kRadix; offset <<= 1) {
    const uint32_t add = digit >= offset ? s_local_start[digit - offset] : 0u;
    __syncthreads();
    s_local_start[digit] += add;
    __syncthreads();
  }
  const uint32_t local_start = s_local_start[digit] - total;
  __syncthreads();
  s_local_start[digit] = local_start;

  // Look back over the predecessors.
  uint32_t exclusive = 0;
  if (tile > 0) {
    int64_t j = static_cast<int64_t>(tile) - 1;
    uint32_t polls = 0;
    bool failed = false;
    while (j >= 0) {
      const uint32_t word = *(volatile uint32_t*)(status + static_cast<size_t>(j) * kRadix + digit);
      const uint32_t flag = word & ~kValueMask;
      if (flag == 0u) {
        if (++polls > kLookbackPollLimit) {
          failed = true;
          break;
        }
        __nanosleep(64);
        continue;
      }
      exclusive += word & kValueMask;
      if (flag == kFlagInclusive) break;
      --j;
    }
    if (failed) atomicExch(error_flag, 1u);
    __threadfence();
    *my_status = kFlagInclusive | ((exclusive + total) & kValueMask);
  }
  s_global_start[digit] = digit_base[digit] + exclusive;
  __syncthreads();

#pragma unroll
  for (int i = 0; i < kItemsPerThread; ++i) {
    const int64_t index = warp_base + i * 32 + lane;
    if (index < count) {
      const uint32_t d = (key[i] >> shift) & 0xFFu;
      const uint32_t position = s_local_start[d] + warp_counts[warp][d] + rank[i];
      s_keys[position] = key[i];
      s_vals[position] = val[i];
    }
  }
  __syncthreads();
  const int64_t remaining = count - tile_base;
  const int valid_items = remaining < kSortTile ? static_cast<int>(remaining) : kSortTile;
  for (int p = tid; p < valid_items; p += kSortThreads) {
    const uint32_t k = s_keys[p];
    const uint32_t d = (k >> shift) & 0xFFu;
    const uint32_t out = s_global_start[d] + (p - s_local_start[d]);
    if (out >= count) {  // only after a look-back that gave up
      atomicExch(error_flag, 1u);
      continue;
    }
    if (write_keys) keys_out[out] = k;
    vals_out[out] = s_vals[p];
  }
}

// First slot of every bin from the sorted keys: bins (key[i-1], key[i]]
// start at slot i, and bins past the last key start at `count`. A thread
// writes its own short range; ranges of 32 bins or more (the empty stretches
// between clusters) are written by the whole warp, one range after another,
// so that no lane walks a long stretch while the others wait. Launched with
// whole warps (blockDim a multiple of 32): every lane takes the ballot.
__global__ void bin_offsets_kernel(const uint32_t* __restrict__ keys, int64_t count,
                                   uint64_t bins, uint32_t* __restrict__ offsets) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int lane = static_cast<int>(threadIdx.x & 31u);
  uint64_t low = 1, high = 0;  // empty unless this thread owns a slot
  if (i <= count) {
    low = i == 0 ? 0ull : static_cast<uint64_t>(keys[i - 1]) + 1ull;
    high = i == count ? bins : static_cast<uint64_t>(keys[i]);
    high = high < bins ? high : bins;
  }
  const bool wide = low <= high && high - low >= 32;
  if (!wide) {
    for (uint64_t b = low; b <= high; ++b) offsets[b] = static_cast<uint32_t>(i);
  }
  unsigned pending = __ballot_sync(0xffffffffu, wide);
  while (pending != 0) {
    const int source = __ffs(pending) - 1;
    pending &= pending - 1;
    const uint64_t first = __shfl_sync(0xffffffffu, static_cast<unsigned long long>(low), source);
    const uint64_t last = __shfl_sync(0xffffffffu, static_cast<unsigned long long>(high), source);
    const uint32_t slot = static_cast<uint32_t>(__shfl_sync(0xffffffffu, static_cast<long long>(i), source));
    for (uint64_t b = first + static_cast<uint64_t>(lane); b <= last; b += 32) offsets[b] = slot;
  }
}

// The same offsets a bin at a time, for bins far outnumbering the points:
// offsets[b] = the number of keys below b, by binary search, so that no
// thread walks a long run of empty bins.
__global__ void bin_offsets_search_kernel(const uint32_t* __restrict__ keys, int64_t count, uint64_t bins,
                                          uint32_t* __restrict__ offsets) {
  const uint64_t b = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b > bins) return;
  int64_t low = 0, high = count;
  while (low < high) {
    const int64_t mid = (low + high) >> 1;
    if (static_cast<uint64_t>(keys[mid]) < b) low = mid + 1; else high = mid;
  }
  offsets[b] = static_cast<uint32_t>(low);
}

// Coordinates in bin order: sorted[slot] = points[perm[slot]], so that the
// spreading and interpolation kernels read them contiguously.
template <int D, typename T>
__global__ void gather_points_kernel(const T* __restrict__ points,
                                     const uint32_t* __restrict__ perm, int64_t count,
                                     T* __restrict__ sorted) {
  const int64_t slot = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (slot >= count) return;
  const int64_t point = perm[slot];
#pragma unroll
  for (int a = 0; a < D; ++a) sorted[slot * D + a] = points[point * D + a];
}

// The inverse of gather_points_kernel: the coordinates of slot i back at the
// point perm[i].
template <int D, typename T>
__global__ void scatter_points_kernel(const T* __restrict__ sorted, const uint32_t* __restrict__ perm,
                                      int64_t count, T* __restrict__ points) {
  const int64_t slot = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (slot >= count) return;
  const int64_t point = perm[slot];
#pragma unroll
  for (int a = 0; a < D; ++a) points[point * D + a] = sorted[slot * D + a];
}

__global__ void identity_kernel(uint32_t* __restrict__ perm, uint32_t* __restrict__ keys,
                                int64_t count) {
  const int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < count) {
    perm[i] = static_cast<uint32_t>(i);
    keys[i] = 0u;
  }
}

// Reference start_in_bin (src/gpu_nd_bins.rs:658-670): a start binned one
// cell across the edge of its bin is moved to the nearest start of the bin.
__device__ __forceinline__ int32_t start_in_bin(int32_t start, int32_t low, int32_t side,
                                                int32_t n) {
  const int32_t span = min(low + side, n) - 1 - low;
  int32_t delta = (start < 0 ? start + n : start) - low;
  if (delta < 0) delta += n;
  if (delta > span && n - delta < delta - span) delta -= n;
  const int32_t clamped = delta < 0 ? 0 : (delta > span ? span : delta);
  return start + clamped - delta;
}

template <int D>
__global__ void prepare_slots_kernel(const float* __restrict__ points, int64_t count, GridParams g,
                                     const uint32_t* __restrict__ perm,
                                     const uint32_t* __restrict__ sorted_keys,
                                     int32_t* __restrict__ starts, float* __restrict__ offsets) {
  const int64_t slot = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (slot >= count) return;
  const uint32_t point = perm[slot];
  float p[D];
#pragma unroll
  for (int a = 0; a < D; ++a) p[a] = points[static_cast<int64_t>(point) * D + a];
  bool reach = true;
#pragma unroll
  for (int a = 0; a < D; ++a) reach = reach && in_fold_reach(p[a]);
  uint32_t rest = sorted_keys[slot];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    uint32_t bin_a;
    if (a == D - 1) {
      bin_a = rest;
    } else {
      bin_a = rest % g.axis[a].bins;
      rest /= g.axis[a].bins;
    }
    const int32_t side = 1 << g.axis[a].shift;
    int32_t start = 0;
    Df64 offset{1024.0f, 0.0f};
    if (reach) support_of(p[a], g.axis[a], g.half_width, start, offset);
    start = start_in_bin(start, static_cast<int32_t>(bin_a) * side, side, g.axis[a].length);
    starts[(D + 1) * slot + a] = start;
    offsets[2 * (D * slot + a)] = offset.hi;
    offsets[2 * (D * slot + a) + 1] = offset.lo;
  }
  starts[(D + 1) * slot + D] = static_cast<int32_t>(point);
}

template <int D>
void launch_keys(const float* points, int64_t count, const GridParams& g, KeyKind kind,
                 uint32_t* keys, uint32_t* hist, int passes, uint32_t invalid_key, uint32_t* valid_mask,
                 cudaStream_t stream) {
  const int blocks = static_cast<int>(std::min<int64_t>((count + 255) / 256, 148 * 16));
  if (kind == KeyKind::SupportStart) {
    bin_keys_kernel<D, KeyKind::SupportStart>
        <<<blocks, 256, 0, stream>>>(points, count, g, keys, hist, passes, 0u, nullptr);
  } else if (kind == KeyKind::SupportStartValidFirst) {
    bin_keys_kernel<D, KeyKind::SupportStartValidFirst>
        <<<blocks, 256, 0, stream>>>(points, count, g, keys, hist, passes, invalid_key, valid_mask);
  } else {
    bin_keys_kernel<D, KeyKind::ApproximateCell>
        <<<blocks, 256, 0, stream>>>(points, count, g, keys, hist, passes, 0u, nullptr);
  }
  note_launch();
}

// The reference order from a valid-first order: with a = points in bin 0,
// v = points within reach (offsets[bins]) and M points, slot s < a (bin 0)
// and slot s >= v (outside the reach, after every bin) hold two index-sorted
// runs merged into the reference's bin 0; slots a <= s < v move up by M - v.
__global__ void reference_order_kernel(const uint32_t* __restrict__ perm, const uint32_t* __restrict__ keys,
                                       const uint32_t* __restrict__ offsets, int64_t count, uint64_t bins,
                                       uint32_t* __restrict__ ref_perm, uint32_t* __restrict__ ref_keys) {
  const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= count) return;
  const int64_t a = offsets[1 < bins ? 1 : bins];
  const int64_t v = offsets[bins];
  const int64_t invalid = count - v;
  const uint32_t x = perm[s];
  int64_t dst;
  if (s < a || s >= v) {
    // Rank among the other run: the number of its indices below x.
    const bool first_run = s < a;
    int64_t low = first_run ? v : 0, high = first_run ? count : a;
    const int64_t begin = low;
    while (low < high) {
      const int64_t mid = (low + high) >> 1;
      if (perm[mid] < x) low = mid + 1; else high = mid;
    }
    dst = (first_run ? s : s - v) + (low - begin);
    ref_keys[dst] = 0u;
  } else {
    dst = s + invalid;
    ref_keys[dst] = keys[s];
  }
  ref_perm[dst] = x;
}

__global__ void reference_offsets_kernel(const uint32_t* __restrict__ offsets, int64_t count, uint64_t bins,
                                         uint32_t* __restrict__ ref_offsets) {
  const int64_t b = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b > static_cast<int64_t>(bins)) return;
  const uint32_t invalid = static_cast<uint32_t>(count) - offsets[bins];
  ref_offsets[b] = b == 0 ? 0u : offsets[b] + invalid;
}

}  // namespace

void gather_sorted_points(const float* points, const uint32_t* perm, int64_t count, int dimensions,
                          float* sorted, cudaStream_t stream, StageTimer* timer) {
  if (count == 0) return;
  StageScope scope(timer, kStageBinOffsets, stream);
  const unsigned blocks = static_cast<unsigned>((count + 255) / 256);
  switch (dimensions) {
    case 1: gather_points_kernel<1, float><<<blocks, 256, 0, stream>>>(points, perm, count, sorted); break;
    case 2: gather_points_kernel<2, float><<<blocks, 256, 0, stream>>>(points, perm, count, sorted); break;
    default: gather_points_kernel<3, float><<<blocks, 256, 0, stream>>>(points, perm, count, sorted); break;
  }
  note_launch();
}

namespace {

template <int D>
__global__ void prepare_windows_kernel(const float* __restrict__ sorted, int64_t count, GridParams g,
                                       PreparedWindow<D>* __restrict__ windows) {
  const int64_t slot = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (slot >= count) return;
  float p[D];
#pragma unroll
  for (int a = 0; a < D; ++a) p[a] = sorted[slot * D + a];
  bool reach = true;
#pragma unroll
  for (int a = 0; a < D; ++a) reach = reach && in_fold_reach(p[a]);
  PreparedWindow<D> w;
#pragma unroll
  for (int a = 0; a < (D == 3 ? 4 : 2); ++a) {
    w.start[a] = 0;
    w.offset[a] = 0.0f;
  }
  if (reach) {
#pragma unroll
    for (int a = 0; a < D; ++a) {
      int32_t start;
      Df64 off;
      support_of(p[a], g.axis[a], g.half_width, start, off);
      w.start[a] = wrap_start(start, g.axis[a].length);
      w.offset[a] = __fadd_rn(off.hi, off.lo);
    }
  } else {
    w.start[0] = -1;
  }
  windows[slot] = w;
}

}  // namespace

namespace {
__global__ void invert_permutation_kernel(const uint32_t* __restrict__ perm, int64_t count,
                                          uint32_t* __restrict__ inverse) {
  const int64_t s = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s < count) inverse[perm[s]] = static_cast<uint32_t>(s);
}
}  // namespace

void invert_permutation(const uint32_t* perm, int64_t count, uint32_t* inverse, cudaStream_t stream) {
  if (count == 0) return;
  invert_permutation_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, stream>>>(perm, count, inverse);
  note_launch();
}

size_t prepared_window_bytes(int dimensions) {
  return dimensions == 3 ? sizeof(PreparedWindow<3>) : sizeof(PreparedWindow<2>);
}

void prepare_windows(const float* sorted_points, int64_t count, const GridParams& grid, void* windows,
                     cudaStream_t stream) {
  if (count == 0) return;
  const unsigned blocks = static_cast<unsigned>((count + 255) / 256);
  switch (grid.dimensions) {
    case 1:
      prepare_windows_kernel<1><<<blocks, 256, 0, stream>>>(sorted_points, count, grid,
                                                            static_cast<PreparedWindow<1>*>(windows));
      break;
    case 2:
      prepare_windows_kernel<2><<<blocks, 256, 0, stream>>>(sorted_points, count, grid,
                                                            static_cast<PreparedWindow<2>*>(windows));
      break;
    default:
      prepare_windows_kernel<3><<<blocks, 256, 0, stream>>>(sorted_points, count, grid,
                                                            static_cast<PreparedWindow<3>*>(windows));
      break;
  }
  note_launch();
}

size_t sort_status_bytes(int64_t count) {
  const int64_t tiles = (count + kSortTile - 1) / kSortTile;
  return static_cast<size_t>(std::max<int64_t>(tiles, 1)) * kRadix * sizeof(uint32_t);
}

namespace {

int radix_passes(uint64_t bins) {
  int key_bits = 0;
  while (key_bits < 32 && (uint64_t(1) << key_bits) < bins) ++key_bits;
  return (key_bits + 7) / 8;
}

// The radix passes and bin offsets once buf.keys_a and buf.hist hold the
// keys and their digit histograms.
void sort_from_keys(int64_t count, uint64_t bins, int passes, SortBuffers buf, uint32_t* offsets,
                    uint32_t** perm, uint32_t** sorted_keys, cudaStream_t stream,
                    StageTimer* timer);

}  // namespace

void sort_points64(const double* points, int64_t count, const GridParams& g, uint64_t bins,
                   SortBuffers buf, uint32_t* offsets, uint32_t** perm, uint32_t** sorted_keys,
                   cudaStream_t stream, StageTimer* timer, uint32_t* valid_mask) {
  // Valid-first keys add one key after the bins.
  const uint64_t keys_range = valid_mask != nullptr ? bins + 1 : bins;
  const int passes = radix_passes(keys_range);
  if (count == 0) {
    check_cuda(cudaMemsetAsync(offsets, 0, (keys_range + 1) * sizeof(uint32_t), stream), "clear offsets");
    *perm = buf.vals_a;
    *sorted_keys = buf.keys_a;
    return;
  }
  {
    StageScope scope(timer, kStageBinKeys, stream);
    check_cuda(cudaMemsetAsync(buf.hist, 0, 4 * kRadix * sizeof(uint32_t), stream), "clear histogram");
    check_cuda(cudaMemsetAsync(buf.counters, 0, 7 * sizeof(uint32_t), stream), "clear tickets");
    const int blocks = static_cast<int>(std::min<int64_t>((count + 255) / 256, 148 * 16));
    const uint32_t invalid_key = static_cast<uint32_t>(bins);
    switch (g.dimensions) {
      case 1:
        bin_keys64_kernel<1><<<blocks, 256, 0, stream>>>(points, count, g, buf.keys_a, buf.hist, passes,
                                                         invalid_key, valid_mask);
        break;
      case 2:
        bin_keys64_kernel<2><<<blocks, 256, 0, stream>>>(points, count, g, buf.keys_a, buf.hist, passes,
                                                         invalid_key, valid_mask);
        break;
      default:
        bin_keys64_kernel<3><<<blocks, 256, 0, stream>>>(points, count, g, buf.keys_a, buf.hist, passes,
                                                         invalid_key, valid_mask);
        break;
    }
    note_launch();
  }
  sort_from_keys(count, keys_range, passes, buf, offsets, perm, sorted_keys, stream, timer);
}

namespace {

void sort_points_kind(const float* points, int64_t count, const GridParams& g, KeyKind kind, uint64_t bins,
                      SortBuffers buf, uint32_t* offsets, uint32_t* valid_mask, uint32_t** perm,
                      uint32_t** sorted_keys, cudaStream_t stream, StageTimer* timer) {
  // Valid-first keys add one key after the bins.
  const uint64_t keys_range = kind == KeyKind::SupportStartValidFirst ? bins + 1 : bins;
  const int passes = radix_passes(keys_range);
  if (count == 0) {
    check_cuda(cudaMemsetAsync(offsets, 0, (keys_range + 1) * sizeof(uint32_t), stream), "clear offsets");
    *perm = buf.vals_a;
    *sorted_keys = buf.keys_a;
    return;
  }
  {
    StageScope scope(timer, kStageBinKeys, stream);
    check_cuda(cudaMemsetAsync(buf.hist, 0, 4 * kRadix * sizeof(uint32_t), stream), "clear histogram");
    check_cuda(cudaMemsetAsync(buf.counters, 0, 7 * sizeof(uint32_t), stream), "clear tickets");
    const uint32_t invalid_key = static_cast<uint32_t>(bins);
    switch (g.dimensions) {
      case 1: launch_keys<1>(points, count, g, kind, buf.keys_a, buf.hist, passes, invalid_key, valid_mask, stream); break;
      case 2: launch_keys<2>(points, count, g, kind, buf.keys_a, buf.hist, passes, invalid_key, valid_mask, stream); break;
      default: launch_keys<3>(points, count, g, kind, buf.keys_a, buf.hist, passes, invalid_key, valid_mask, stream); break;
    }
  }
  sort_from_keys(count, keys_range, passes, buf, offsets, perm, sorted_keys, stream, timer);
}

}  // namespace

void sort_points(const float* points, int64_t count, const GridParams& g, KeyKind kind,
                 uint64_t bins, SortBuffers buf, uint32_t* offsets, uint32_t** perm,
                 uint32_t** sorted_keys, cudaStream_t stream, StageTimer* timer) {
  sort_points_kind(points, count, g, kind, bins, buf, offsets, nullptr, perm, sorted_keys, stream, timer);
}

void sort_points_valid_first(const float* points, int64_t count, const GridParams& g, uint64_t bins,
                             SortBuffers buf, uint32_t* offsets, uint32_t* valid_mask, uint32_t** perm,
                             uint32_t** sorted_keys, cudaStream_t stream, StageTimer* timer) {
  sort_points_kind(points, count, g, KeyKind::SupportStartValidFirst, bins, buf, offsets, valid_mask, perm,
                   sorted_keys, stream, timer);
}

void reference_bin_order(const uint32_t* perm, const uint32_t* keys, const uint32_t* offsets, int64_t count,
                         uint64_t bins, uint32_t* ref_perm, uint32_t* ref_keys, uint32_t* ref_offsets,
                         cudaStream_t stream) {
  if (count > 0) {
    reference_order_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, stream>>>(
        perm, keys, offsets, count, bins, ref_perm, ref_keys);
    note_launch();
  }
  reference_offsets_kernel<<<static_cast<unsigned>((bins + 1 + 255) / 256), 256, 0, stream>>>(offsets, count, bins,
                                                                                              ref_offsets);
  note_launch();
}

namespace {

void sort_from_keys(int64_t count, uint64_t bins, int passes, SortBuffers buf, uint32_t* offsets,
                    uint32_t** perm, uint32_t** sorted_keys, cudaStream_t stream,
                    StageTimer* timer) {
  if (passes == 0) {
    identity_kernel<<<static_cast<unsigned>((count + 255) / 256), 256, 0, stream>>>(buf.vals_a,
                                                                                 buf.keys_a, count);
    note_launch();
    *perm = buf.vals_a;
    *sorted_keys = buf.keys_a;
  } else {
    {
      StageScope scope(timer, kStageDigitScan, stream);
      digit_scan_kernel<<<1, kRadix, 0, stream>>>(buf.hist, passes);
      note_launch();
    }
    StageScope scope(timer, kStageRadixPasses, stream);
    const int64_t tiles = (count + kSortTile - 1) / kSortTile;
    uint32_t* keys_in = buf.keys_a;
    uint32_t* vals_in = nullptr;
    uint32_t* keys_out = buf.keys_b;
    uint32_t* vals_out = buf.vals_b;
    for (int pass = 0; pass < passes; ++pass) {
      check_cuda(cudaMemsetAsync(buf.status, 0, static_cast<size_t>(tiles) * kRadix * sizeof(uint32_t),
                                 stream),
                 "clear look-back words");
      onesweep_pass_kernel<<<static_cast<unsigned>(tiles), kSortThreads, 0, stream>>>(
          keys_in, vals_in, keys_out, vals_out, count, 8 * pass, buf.hist + pass * kRadix,
          buf.status, buf.counters + pass, buf.counters + 7, 1);
      note_launch();
      // Ping-pong: the next pass reads what this one wrote.
      uint32_t* next_keys_out = keys_in;
      uint32_t* next_vals_out = (vals_out == buf.vals_b) ? buf.vals_a : buf.vals_b;
      keys_in = keys_out;
      vals_in = vals_out;
      keys_out = next_keys_out;
      vals_out = next_vals_out;
    }
    *perm = vals_in;
    *sorted_keys = keys_in;
  }
  StageScope scope(timer, kStageBinOffsets, stream);
  if (bins > 2 * static_cast<uint64_t>(count)) {
    bin_offsets_search_kernel<<<static_cast<unsigned>((bins + 1 + 255) / 256), 256, 0, stream>>>(
        *sorted_keys, count, bins, offsets);
  } else {
    bin_offsets_kernel<<<static_cast<unsigned>((count + 1 + 255) / 256), 256, 0, stream>>>(
        *sorted_keys, count, bins, offsets);
  }
  note_launch();
}

}  // namespace

template <typename T>
void scatter_points3(const T* sorted, const uint32_t* perm, int64_t count, T* points, cudaStream_t stream) {
  if (count == 0) return;
  const unsigned blocks = static_cast<unsigned>((count + 255) / 256);
  scatter_points_kernel<3, T><<<blocks, 256, 0, stream>>>(sorted, perm, count, points);
  note_launch();
}
template void scatter_points3<float>(const float*, const uint32_t*, int64_t, float*, cudaStream_t);
template void scatter_points3<double>(const double*, const uint32_t*, int64_t, double*, cudaStream_t);

void gather_sorted_points64(const double* points, const uint32_t* perm, int64_t count,
                            int dimensions, double* sorted, cudaStream_t stream,
                            StageTimer* timer) {
  if (count == 0) return;
  StageScope scope(timer, kStageBinOffsets, stream);
  const unsigned blocks = static_cast<unsigned>((count + 255) / 256);
  switch (dimensions) {
    case 1: gather_points_kernel<1, double><<<blocks, 256, 0, stream>>>(points, perm, count, sorted); break;
    case 2: gather_points_kernel<2, double><<<blocks, 256, 0, stream>>>(points, perm, count, sorted); break;
    default: gather_points_kernel<3, double><<<blocks, 256, 0, stream>>>(points, perm, count, sorted); break;
  }
  note_launch();
}

void prepare_reference_slots(const float* points, int64_t count, const GridParams& g,
                             const uint32_t* perm, const uint32_t* sorted_keys, int32_t* starts,
                             float* offsets, cudaStream_t stream) {
  if (count == 0) return;
  const unsigned blocks = static_cast<unsigned>((count + 255) / 256);
  switch (g.dimensions) {
    case 1:
      prepare_slots_kernel<1><<<blocks, 256, 0, stream>>>(points, count, g, perm, sorted_keys,
                                                          starts, offsets);
      break;
    case 2:
      prepare_slots_kernel<2><<<blocks, 256, 0, stream>>>(points, count, g, perm, sorted_keys,
                                                          starts, offsets);
      break;
    default:
      prepare_slots_kernel<3><<<blocks, 256, 0, stream>>>(points, count, g, perm, sorted_keys,
                                                          starts, offsets);
      break;
  }
  note_launch();
}

}  // namespace b200nufft
