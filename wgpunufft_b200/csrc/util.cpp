// Error reporting, launch accounting and grow-only device buffers.
#include <cuda_runtime.h>

#include <atomic>
#include <string>

#include "device.h"
#include "util.h"

namespace b200nufft {

namespace {
thread_local std::string g_last_error;
std::atomic<uint64_t> g_launches{0};
}  // namespace

void set_last_error(const std::string& message) { g_last_error = message; }
const char* last_error() { return g_last_error.c_str(); }

void check_cuda(cudaError_t error, const char* what) {
  if (error != cudaSuccess) {
    const int code = error == cudaErrorMemoryAllocation ? B200NUFFT_DEVICE_ALLOCATION_FAILED
                                                        : B200NUFFT_DEVICE_ERROR;
    throw NufftFailure{code, std::string(what) + ": " + cudaGetErrorString(error)};
  }
}

void note_launch(int count) { g_launches.fetch_add(static_cast<uint64_t>(count)); }
uint64_t launch_count() { return g_launches.load(); }

DeviceBuffer::~DeviceBuffer() { release(); }

void DeviceBuffer::release() {
  if (ptr_) cudaFree(ptr_);
  ptr_ = nullptr;
  bytes_ = 0;
}

void* DeviceBuffer::reserve(size_t bytes, const char* label) {
  if (bytes <= bytes_ && ptr_) return ptr_;
  release();
  const size_t rounded = bytes == 0 ? 256 : ((bytes + 255) / 256) * 256;
  void* p = nullptr;
  const cudaError_t e = cudaMalloc(&p, rounded);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw NufftFailure{B200NUFFT_DEVICE_ALLOCATION_FAILED,
                       std::string("device allocation of ") + std::to_string(rounded) +
                           " bytes for " + label + " failed: " + cudaGetErrorString(e)};
  }
  ptr_ = p;
  bytes_ = rounded;
  return ptr_;
}

}  // namespace b200nufft
