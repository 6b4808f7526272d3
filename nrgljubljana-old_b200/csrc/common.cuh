// Shared helpers for the NRG step kernels: error handling, a device arena,
// and a bounded grid barrier for cooperative persistent kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <stdexcept>
#include <mutex>
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
  // byte offset of a pointer handed out by alloc()
  size_t offset_of(const void* p) const { return (size_t)(static_cast<const char*>(p) - static_cast<const char*>(base_)); }
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
// inside a larger call).  One instance per process, shared by every context
// and thread: all members are guarded by one mutex, and each bracketed
// launch carries its own record slot, so launches from several host threads
// may interleave.
class KernelStats {
 public:
  static KernelStats& get();
  // resets all counters; with `only` (a name, or a prefix ending in '*'),
  // only launches of that name are timed, the others are just counted
  void enable(bool on, const char* only = nullptr);
  bool timing() const { return timing_; }
  // bracket one launch: begin() before (counts it and, with timing on,
  // records the start event and returns a slot), end(slot) after
  int begin(const char* name, cudaStream_t s);
  void end(int slot, cudaStream_t s);
  void count(const char* name, long n = 1);
  // algorithmic work of launches of `name` (bytes for a memory-bound
  // kernel, flops for a contraction), stated by the launching host code
  void add_work(const char* name, double units);
  // launches and total milliseconds of `name` ("*" = all kernels); syncs events
  void query(const char* name, long* launches, double* ms);
  double work(const char* name);

 private:
  struct Rec { std::string name; cudaEvent_t a, b; };
  std::mutex m_;
  bool timing_ = false;
  std::string only_;  // empty: time every launch
  std::vector<Rec> open_, done_;
  std::vector<int> free_;
  std::vector<cudaEvent_t> pool_;
  std::vector<std::pair<std::string, long>> counts_;
  std::vector<std::pair<std::string, double>> ms_;
  std::vector<std::pair<std::string, double>> work_;
  cudaEvent_t ev();
  void count_locked(const char* name, long n);
  void settle();
};

// Counts (and, when timing is on, times) one kernel launch statement.
#define NRGB_LAUNCH(name, stream, ...)                      \
  do {                                                      \
    ::nrgb::KernelStats& ks__ = ::nrgb::KernelStats::get(); \
    const int slot__ = ks__.begin(name, stream);            \
    __VA_ARGS__;                                            \
    ks__.end(slot__, stream);                               \
  } while (0)

// Device-side state of a grid barrier.  The arrival counter and the
// generation word sit on separate 128-byte lines, so CTAs polling the
// generation do not contend with the atomics on the counter.
struct GridBarrier {
  unsigned int count;
  int error;     // set when a wait gave up
  unsigned int pad0[30];
  unsigned int gen;
  unsigned int pad1[31];
};

#ifdef __CUDACC__
__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];\n" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Generation barrier for co-resident CTAs (cooperative launch).  Thread 0
// of each CTA arrives with a release-acquire atomic and polls the
// generation with acquire loads and exponential back-off.  Every wait is
// bounded: after 2^limit_log2 polls (2^23, about a second, by default) the
// CTA records an error, and a waiting CTA that sees the error leaves too;
// once the error is set all later barriers return immediately.  Returns
// true (in every thread of the CTA) when the error is set, so that the
// caller can end the launch instead of computing on unsynchronised data.
__device__ __forceinline__ bool grid_barrier(GridBarrier* b, unsigned int nblocks, int limit_log2 = 23) {
  __shared__ int s_failed;
  __syncthreads();
  if (threadIdx.x == 0) {
    const long long limit = 1ll << limit_log2;
    if (*reinterpret_cast<volatile int*>(&b->error) == 0) {
      const unsigned int g = ld_acquire_u32(&b->gen);
      __threadfence();
      unsigned int arrived;
      asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], 1;\n" : "=r"(arrived) : "l"(&b->count) : "memory");
      if (arrived + 1u == nblocks) {
        b->count = 0;
        __threadfence();
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;\n" ::"l"(&b->gen) : "memory");
      } else {
        long long it = 0;
        unsigned ns = 8;
        while (ld_acquire_u32(&b->gen) == g) {
          if (++it > limit || *reinterpret_cast<volatile int*>(&b->error)) {
            atomicExch(&b->error, 1);
            break;
          }
          __nanosleep(ns);
          if (ns < 128) ns <<= 1;
        }
      }
      __threadfence();
    }
    s_failed = *reinterpret_cast<volatile int*>(&b->error);
  }
  __syncthreads();
  return s_failed != 0;
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
