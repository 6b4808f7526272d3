// Shared helpers for the NRG step kernels: error handling, a device arena,
// and a bounded grid barrier for cooperative persistent kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <stdexcept>
#include <string>
#include <vector>

namespace nrgb {

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};

#define NRGB_CUDA(call)                                                                   \
  do {                                                                                    \
    cudaError_t err__ = (call);                                                           \
    if (err__ != cudaSuccess)                                                             \
      throw ::nrgb::CudaError(std::string(#call) + ": " + cudaGetErrorString(err__) +     \
                              " (" + __FILE__ + ":" + std::to_string(__LINE__) + ")");    \
  } while (0)

// Bump allocator over one device allocation.  Every pointer it hands out is
// 256-byte aligned.  reset() releases everything at once; the backing store
// grows (with a device synchronize) when a request does not fit.
class DeviceArena {
 public:
  DeviceArena() = default;
  ~DeviceArena() { release(); }
  DeviceArena(const DeviceArena&) = delete;
  DeviceArena& operator=(const DeviceArena&) = delete;

  void reserve(size_t bytes) {
    if (bytes <= cap_) return;
    release();
    NRGB_CUDA(cudaMalloc(&base_, bytes));
    cap_ = bytes;
    off_ = 0;
  }
  // Allocation that must fit in the current reservation.
  void* alloc(size_t bytes) {
    size_t a = (off_ + 255) & ~size_t(255);
    if (a + bytes > cap_) throw CudaError("DeviceArena: out of reserved space");
    off_ = a + bytes;
    return static_cast<char*>(base_) + a;
  }
  template <class T>
  T* alloc_n(size_t n) { return static_cast<T*>(alloc(n * sizeof(T) + 8)); }
  size_t used() const { return off_; }
  size_t capacity() const { return cap_; }
  void reset() { off_ = 0; }
  void release() {
    if (base_) cudaFree(base_);
    base_ = nullptr;
    cap_ = off_ = 0;
  }

 private:
  void* base_ = nullptr;
  size_t cap_ = 0, off_ = 0;
};

// Size planner: accumulates aligned sizes so a caller can reserve an arena once.
struct ArenaPlan {
  size_t bytes = 0;
  template <class T>
  void add(size_t n) { bytes = ((bytes + 255) & ~size_t(255)) + n * sizeof(T) + 8; }
};

// Launch counting and optional per-kernel timing with CUDA events on the
// launching stream (used by the benchmark to time the dominant kernel
// inside a larger call).  One instance per process; not thread-safe.
class KernelStats {
 public:
  static KernelStats& get();
  void enable(bool on);              // resets all counters
  bool timing() const { return timing_; }
  // bracket one launch: begin() before, end() after (no-ops without timing)
  void begin(const char* name, cudaStream_t s);
  void end(cudaStream_t s);
  void count(const char* name, long n = 1);
  // launches and total milliseconds of `name` ("*" = all kernels); syncs events
  void query(const char* name, long* launches, double* ms);

 private:
  struct Rec { std::string name; cudaEvent_t a, b; };
  bool timing_ = false;
  std::vector<Rec> open_, done_;
  std::vector<cudaEvent_t> pool_;
  std::vector<std::pair<std::string, long>> counts_;
  std::vector<std::pair<std::string, double>> ms_;
  cudaEvent_t ev();
  void settle();
};

// Counts (and, when timing is on, times) one kernel launch statement.
#define NRGB_LAUNCH(name, stream, ...)                 \
  do {                                                 \
    ::nrgb::KernelStats& ks__ = ::nrgb::KernelStats::get(); \
    ks__.count(name);                                  \
    ks__.begin(name, stream);                          \
    __VA_ARGS__;                                       \
    ks__.end(stream);                                  \
  } while (0)

// Device-side state of a grid barrier (one per cooperative launch).
struct GridBarrier {
  unsigned int count;
  unsigned int gen;
  int error;     // set when a wait gave up
  int pad;
};

#ifdef __CUDACC__
// Sense-free generation barrier for co-resident CTAs (cooperative launch).
// Every wait is bounded: after ~2^26 polls the CTA records an error and
// continues; once the error is set all later barriers return immediately,
// so a broken launch ends instead of hanging the GPU.
__device__ __forceinline__ void grid_barrier(GridBarrier* b, unsigned int nblocks) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile GridBarrier* vb = b;
    if (vb->error == 0) {
      const unsigned int g = vb->gen;
      __threadfence();
      const unsigned int arrived = atomicAdd(&b->count, 1u) + 1u;
      if (arrived == nblocks) {
        b->count = 0;
        __threadfence();
        atomicAdd(&b->gen, 1u);
      } else {
        long long it = 0;
        while (vb->gen == g) {
          if (++it > (1ll << 26)) {
            atomicExch(&b->error, 1);
            break;
          }
          __nanosleep(20);
        }
      }
      __threadfence();
    }
  }
  __syncthreads();
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum; `scratch` holds >= 32 doubles.  All threads get the result.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double r = (threadIdx.x < nw) ? scratch[threadIdx.x] : 0.0;
  if (warp == 0) {
    r = warp_sum(r);
    if (lane == 0) scratch[0] = r;
  }
  __syncthreads();
  r = scratch[0];
  __syncthreads();
  return r;
}
#endif

}  // namespace nrgb
