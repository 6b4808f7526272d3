// Allocation-free variant of the operator basis change
//     out[o] = Z_bra[o]^T * op[o] * Z_ket[o]
// (the contraction of the recalculation step) for callers that must not see
// the library allocate device memory.
//
// Who needs it: a host that owns the whole device-memory budget (for example
// a serving loop that admits NRG runs by their projected footprint and
// cannot let a library call grow it), or a caller in a latency-critical loop
// that cannot afford the device-wide synchronisation cudaMalloc/cudaFree
// imply.  The regular entry points keep their intermediates in memory the
// context allocates; this one uses a fixed array that is part of the loaded
// library instead.
//
// The intermediate products op[o] * Z_ket[o] and the launch descriptors live
// in g_basis_scratch, a file-scope device array of NOALLOC_SCRATCH_BYTES
// (32 MiB) that every GPU which loads the library holds until the process
// exits.  All calls share it:
//   * nothing in it has to start at zero: each call writes every byte of the
//     scratch it later reads (descriptors, then intermediates with beta = 0);
//   * one call runs at a time per process: a process-wide lock serialises
//     the calls, and each call blocks until its work on `stream` has
//     finished, so two calls never have work on the array at the same time,
//     whichever streams or host threads they come from.  The price is that
//     the call is synchronous; callers that overlap streams get no
//     asynchrony from it.
// Host code never touches g_basis_scratch by name (on the host that name is
// only a stand-in for the device symbol): the device address comes from
// cudaGetSymbolAddress, once per device, with that device current, on the
// first call on that device.  Make that first call before any stream
// capture begins.  A call whose `stream` is capturing is refused (status 7)
// before anything is enqueued, so the caller's capture stays intact: the
// call's final stream synchronisation would otherwise end that capture.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/nrgb.h"
#include "common.cuh"
#include "gemm_f64.cuh"

namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(32) << 20;  // 32 MiB
constexpr int NOALLOC_MAX_OPS = 1024;
constexpr int NOALLOC_MAX_DEVICES = 64;

static __device__ __align__(256) unsigned char g_basis_scratch[NOALLOC_SCRATCH_BYTES];

// One call at a time per process: the host-side descriptor staging below is
// static (no heap), and calls on one device would race on the device array.
std::mutex g_call_mutex;
unsigned char* g_scratch_addr[NOALLOC_MAX_DEVICES] = {nullptr};
nrgb::GemmProb g_p1[NOALLOC_MAX_OPS], g_p2[NOALLOC_MAX_OPS];
nrgb::GemmSeg g_s1[NOALLOC_MAX_OPS], g_s2[NOALLOC_MAX_OPS];

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Device address of the scratch array for the current device (set-up on the
// first call per device).  Returns nullptr on failure.
unsigned char* scratch_address(int dev) {
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_basis_scratch) != cudaSuccess || p == nullptr) return nullptr;
    g_scratch_addr[dev] = static_cast<unsigned char*>(p);
  }
  return g_scratch_addr[dev];
}

}  // namespace

extern "C" int nrgb_basis_change_noalloc(int nops, const int* n_bra, const int* n_ket,
                                         const double* const* z_bra, const double* const* z_ket,
                                         const double* const* op, double* const* out, void* stream) {
  if (nops < 0 || (nops > 0 && (!n_bra || !n_ket || !z_bra || !z_ket || !op || !out))) return 1;
  if (nops > NOALLOC_MAX_OPS) return 5;
  // layout of the scratch: [stage-1 descriptors | stage-2 descriptors | intermediates]
  const size_t dbytes = align256(nops * sizeof(nrgb::GemmProb)) + align256(nops * sizeof(nrgb::GemmSeg));
  size_t need = 2 * dbytes;
  for (int o = 0; o < nops; ++o) {
    if (n_bra[o] < 0 || n_ket[o] < 0) return 1;
    need += align256((size_t)n_bra[o] * n_ket[o] * sizeof(double));
  }
  if (need > NOALLOC_SCRATCH_BYTES) return 5;  // larger than the static scratch
  if (nops == 0) return 0;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  {
    // the call ends with a stream synchronisation, which a capture forbids
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) return 6;
    if (cs != cudaStreamCaptureStatusNone) return 7;
  }
  std::lock_guard<std::mutex> lock(g_call_mutex);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= NOALLOC_MAX_DEVICES) return 6;
  unsigned char* base = scratch_address(dev);
  if (!base) return 6;

  unsigned char* d_p1 = base;
  unsigned char* d_s1 = d_p1 + align256(nops * sizeof(nrgb::GemmProb));
  unsigned char* d_p2 = base + dbytes;
  unsigned char* d_s2 = d_p2 + align256(nops * sizeof(nrgb::GemmProb));
  unsigned char* tmp = base + 2 * dbytes;

  int np = 0, t1 = 0, t2 = 0;
  for (int o = 0; o < nops; ++o) {
    const int nb = n_bra[o], nk = n_ket[o];
    double* T = reinterpret_cast<double*>(tmp);
    tmp += align256((size_t)nb * nk * sizeof(double));
    if (nb == 0 || nk == 0) continue;
    nrgb::GemmProb a{};
    a.C = T;  // T = op * Z_ket   (nb x nk)
    a.ldc = nb;
    a.m = nb;
    a.n = nk;
    a.beta = 0.0;
    a.seg0 = np;
    a.nseg = 1;
    a.tile0 = t1;
    a.tiles_n = (nk + nrgb::GEMM_BN - 1) / nrgb::GEMM_BN;
    t1 += ((nb + nrgb::GEMM_BM - 1) / nrgb::GEMM_BM) * a.tiles_n;
    g_p1[np] = a;
    g_s1[np] = nrgb::GemmSeg{op[o], z_ket[o], nb, nk, nk, 0, 0, 1.0};
    nrgb::GemmProb b = a;  // out = Z_bra^T * T
    b.C = out[o];
    b.tile0 = t2;
    t2 += ((nb + nrgb::GEMM_BM - 1) / nrgb::GEMM_BM) * b.tiles_n;
    g_p2[np] = b;
    g_s2[np] = nrgb::GemmSeg{z_bra[o], T, nb, nb, nb, 1, 0, 1.0};
    ++np;
  }
  if (np == 0) return 0;
  if (cudaMemcpyAsync(d_p1, g_p1, np * sizeof(g_p1[0]), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d_s1, g_s1, np * sizeof(g_s1[0]), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d_p2, g_p2, np * sizeof(g_p2[0]), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(d_s2, g_s2, np * sizeof(g_s2[0]), cudaMemcpyHostToDevice, st) != cudaSuccess)
    return 6;
  if (nrgb::gemm_grouped_launch_unaccounted(reinterpret_cast<nrgb::GemmProb*>(d_p1), np,
                                            reinterpret_cast<nrgb::GemmSeg*>(d_s1), t1, st) != cudaSuccess)
    return 6;
  if (nrgb::gemm_grouped_launch_unaccounted(reinterpret_cast<nrgb::GemmProb*>(d_p2), np,
                                            reinterpret_cast<nrgb::GemmSeg*>(d_s2), t2, st) != cudaSuccess)
    return 6;
  // the static host staging is reused by the next call: wait until the GPU is done
  if (cudaStreamSynchronize(st) != cudaSuccess) return 6;
  return 0;
}
