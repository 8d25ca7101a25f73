// Device-side helpers shared by the engines.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "host.h"

#define FMD_CUDA(call)                                                                   \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      throw ::fmd::Error(FMD_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define FMD_CUDA_LAUNCH() FMD_CUDA(cudaPeekAtLastError())

namespace fmd {

// Status bits a device kernel may raise for a system / replica.
enum : int32_t {
  kStatusOverflow = 1,   // neighbor list capacity exceeded
  kStatusNonFinite = 2,  // non-finite position / velocity / energy
  kStatusFeneStretch = 4,  // a FENE bond reached R0 (the reference clamps silently)
  kStatusCellCapacity = 8, // cell grid / cell occupancy capacity exceeded
  kStatusTimeout = 16,     // a bounded device wait expired
  kStatusStaleScalars = 32,  // a pre-force found no precomputed step scalars
};

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

template <typename T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void alloc(size_t count) {
    release();
    if (count == 0) count = 1;
    FMD_CUDA(cudaMalloc(&p, count * sizeof(T)));
    n = count;
  }
  void alloc_zero(size_t count) {
    alloc(count);
    FMD_CUDA(cudaMemset(p, 0, n * sizeof(T)));
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
  operator T*() const { return p; }
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
  return v;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, o);
  return v;
}

}  // namespace fmd
