// Stable bin order without device allocation: b200nufft_bin_order_noalloc.
//
// Some callers cannot call cudaMalloc: code that runs while another
// framework owns every byte of device memory through its own pool, code in a
// real-time or callback context where an allocation may block or fail, and
// code that must not touch the allocator at all. For them this entry point
// computes the same stable bin order as b200nufft_set_points followed by
// b200nufft_copy_bin_order, but all of its scratch memory (keys, permutation
// buffers, digit histograms and look-back words of the radix sort) lives in
// one fixed array in this library's device image. The array is sized for at
// most B200NUFFT_NOALLOC_MAX_POINTS points. The CUDA driver places it on a
// GPU when it loads this file's module there: at the library's first kernel
// launch on that GPU with CUDA_MODULE_LOADING=EAGER, otherwise (lazy
// loading, CUDA 12's default) at this entry point's first call on that GPU,
// which looks up the array's address. So that first call (a call with no
// points does that set-up and writes zero bin offsets) must come before another framework takes
// the GPU's memory. From then on the GPU holds the array until the process
// exits.
//
// A look-back wait of the radix sort that gives up (bounded at about a
// second) cannot be reported by the return code, which is known before the
// GPU runs: the call then writes 0xFFFFFFFF to bin_offsets[bins], the
// trailing total that otherwise equals point_count.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "device.h"
#include "util.h"

namespace b200nufft {

namespace {

constexpr int64_t kMaxPoints = B200NUFFT_NOALLOC_MAX_POINTS;
constexpr size_t kWordBytes = sizeof(uint32_t);
constexpr size_t kBufferBytes = static_cast<size_t>(kMaxPoints) * kWordBytes;
constexpr size_t kHistBytes = 4 * 256 * kWordBytes;
constexpr size_t kStatusBytes =
    ((kMaxPoints + kSortTilePoints - 1) / kSortTilePoints) * kSortDigits * kWordBytes;
constexpr size_t kCounterBytes = 8 * kWordBytes;
constexpr size_t kScratchBytes = 4 * kBufferBytes + kHistBytes + kStatusBytes + kCounterBytes;
constexpr int kMaxDevices = 64;
constexpr double kTwoPi = 6.28318530717958647692;

// The scratch of every call on this device. In host code this name is only a
// stand-in for the symbol, not a device address: its address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

// Marks a sort whose look-back gave up: the trailing total of the bin
// offsets, which otherwise equals the point count, becomes 0xFFFFFFFF.
__global__ void mark_gave_up_kernel(const uint32_t* __restrict__ error_flag, uint32_t* __restrict__ total) {
  if (*error_flag != 0u) *total = 0xFFFFFFFFu;
}

std::mutex g_setup_mutex;
void* g_scratch_address[kMaxDevices] = {};

// The device address of the scratch array on the current device, looked up
// once per device (with that device current) and kept.
unsigned char* scratch_on_current_device() {
  int device = 0;
  check_cuda(cudaGetDevice(&device), "current device");
  if (device < 0 || device >= kMaxDevices) {
    throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "device ordinal out of range"};
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_address[device]) {
    void* address = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&address, g_noalloc_scratch);
    if (e != cudaSuccess || address == nullptr) {
      cudaGetLastError();
      throw NufftFailure{B200NUFFT_DEVICE_ERROR,
                         std::string("cannot resolve the scratch array on this device: ") +
                             cudaGetErrorString(e)};
    }
    g_scratch_address[device] = address;
  }
  return static_cast<unsigned char*>(g_scratch_address[device]);
}

}  // namespace

void bin_order_noalloc(int32_t dimensions, const int64_t* fine_shape, int32_t kernel_width,
                       const int32_t* bin_sides, int64_t point_count, const float* points,
                       uint32_t* permutation, uint32_t* bin_offsets, cudaStream_t stream) {
  if (dimensions < 1 || dimensions > 3) {
    throw NufftFailure{B200NUFFT_INVALID_DIMENSIONS, "dimensions must lie in 1..3"};
  }
  if (!fine_shape || !bin_sides || !bin_offsets) {
    throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null shape, bin sides or bin offsets"};
  }
  if (kernel_width < kMinWidth || kernel_width > kMaxWidth) {
    throw NufftFailure{B200NUFFT_INVALID_KERNEL_WIDTH, "kernel width outside 2..16"};
  }
  if (point_count < 0 || point_count > kMaxPoints) {
    throw NufftFailure{B200NUFFT_LENGTH_OVERFLOW,
                       "point count " + std::to_string(point_count) + " outside 0.." +
                           std::to_string(kMaxPoints) +
                           ", the capacity of the fixed scratch array"};
  }
  if (point_count > 0 && (!points || !permutation)) {
    throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "null points or permutation"};
  }
  GridParams g;
  std::memset(&g, 0, sizeof(g));
  g.dimensions = dimensions;
  g.width = kernel_width;
  g.half_width = 0.5f * static_cast<float>(kernel_width);
  uint64_t bins = 1;
  for (int a = 0; a < dimensions; ++a) {
    const int64_t n = fine_shape[a];
    const int32_t side = bin_sides[a];
    if (n < 2 * kernel_width || n % 2 != 0 || n > (int64_t(1) << 24) - kernel_width) {
      throw NufftFailure{B200NUFFT_INVALID_ARGUMENT,
                         "fine-grid axis " + std::to_string(a) + " of " + std::to_string(n) +
                             " cells is not an even length in 2w..2^24-w"};
    }
    if (side < 1 || (side & (side - 1)) != 0) {
      throw NufftFailure{B200NUFFT_INVALID_ARGUMENT, "bin sides must be powers of two"};
    }
    int shift = 0;
    while ((1 << shift) < side) ++shift;
    const uint64_t count = static_cast<uint64_t>((n + side - 1) / side);
    FoldAxis& axis = g.axis[a];
    const double scale = static_cast<double>(n) / kTwoPi;
    axis.scale_hi = static_cast<float>(scale);
    axis.scale_lo = static_cast<float>(scale - static_cast<double>(axis.scale_hi));
    axis.origin = static_cast<float>(n / 2);
    axis.length_f = static_cast<float>(n);
    axis.length = static_cast<int32_t>(n);
    axis.shift = shift;
    axis.bins = static_cast<uint32_t>(count);
    axis.stride = static_cast<uint32_t>(bins);
    bins *= count;
    if (bins > 0xFFFFFFFFull) throw NufftFailure{B200NUFFT_LENGTH_OVERFLOW, "bin count"};
    g.fine[a] = n;
  }
  g.fine_count = 1;
  for (int a = 0; a < dimensions; ++a) g.fine_count *= g.fine[a];
  if (sort_status_bytes(point_count) > kStatusBytes) {
    throw NufftFailure{B200NUFFT_INTERNAL, "look-back words exceed the fixed scratch array"};
  }

  unsigned char* base = scratch_on_current_device();
  SortBuffers buffers;
  buffers.keys_a = reinterpret_cast<uint32_t*>(base);
  buffers.keys_b = reinterpret_cast<uint32_t*>(base + kBufferBytes);
  buffers.vals_a = reinterpret_cast<uint32_t*>(base + 2 * kBufferBytes);
  buffers.vals_b = reinterpret_cast<uint32_t*>(base + 3 * kBufferBytes);
  buffers.hist = reinterpret_cast<uint32_t*>(base + 4 * kBufferBytes);
  buffers.status = reinterpret_cast<uint32_t*>(base + 4 * kBufferBytes + kHistBytes);
  buffers.counters = reinterpret_cast<uint32_t*>(base + 4 * kBufferBytes + kHistBytes + kStatusBytes);
  // The array keeps the previous call's contents: the tickets and the
  // look-back error word must start at zero (the sort clears the histograms
  // and look-back words itself).
  check_cuda(cudaMemsetAsync(buffers.counters, 0, kCounterBytes, stream), "clear sort tickets");
  uint32_t* perm = nullptr;
  uint32_t* sorted_keys = nullptr;
  sort_points(points, point_count, g, KeyKind::SupportStart, bins, buffers, bin_offsets, &perm,
              &sorted_keys, stream);
  if (point_count > 0) {
    check_cuda(cudaMemcpyAsync(permutation, perm, static_cast<size_t>(point_count) * kWordBytes,
                               cudaMemcpyDeviceToDevice, stream),
               "copy permutation");
    mark_gave_up_kernel<<<1, 1, 0, stream>>>(buffers.counters + 7, bin_offsets + bins);
    note_launch();
  }
  check_cuda(cudaGetLastError(), "bin order launch");
}

}  // namespace b200nufft

extern "C" int b200nufft_bin_order_noalloc(int32_t dimensions, const int64_t* fine_shape,
                                           int32_t kernel_width, const int32_t* bin_sides,
                                           int64_t point_count, const float* points,
                                           uint32_t* permutation, uint32_t* bin_offsets,
                                           void* stream) {
  try {
    b200nufft::bin_order_noalloc(dimensions, fine_shape, kernel_width, bin_sides, point_count, points,
                                 permutation, bin_offsets, static_cast<cudaStream_t>(stream));
    return B200NUFFT_SUCCESS;
  } catch (const b200nufft::NufftFailure& failure) {
    b200nufft::set_last_error(failure.message);
    return failure.code;
  } catch (...) {
    b200nufft::set_last_error("internal error");
    return B200NUFFT_INTERNAL;
  }
}
