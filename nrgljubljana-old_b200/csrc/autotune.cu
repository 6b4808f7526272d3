// The schedule table (schedule.cuh) and the autotuner that fills it by
// measurement on the device at hand.
//
// GEMM tiles: grouped FP64 launches of square problems (edge 128 .. 2048,
// the block sizes of the workloads) are timed with 64 x 64 and with
// 128 x 128 tiles; gemm_large_from becomes the smallest edge from which the
// large tiles win by more than 3 % at every larger edge (0 when they never
// do).
//
// Cluster limit: one batched eigensolve of a mix of block sizes spread over
// the cluster kernel's range and beyond it (the sizes the served runs
// produce) is timed for several limits; the fastest limit is kept.  Blocks
// above the limit take cooperative panel launches until their trailing block
// fits.
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>

#include <algorithm>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "autotune.cuh"
#include "common.cuh"
#include "gemm_f64.cuh"
#include "schedule.cuh"

namespace nrgb {

Schedule& schedule_of(int device) {
  static Schedule table[64];
  if (device < 0 || device >= 64) device = 0;
  return table[device];
}

Schedule& schedule_here() {
  int dev = 0;
  cudaGetDevice(&dev);
  return schedule_of(dev);
}

namespace {

// deterministic symmetric test matrices: H[i, j] = H[j, i] in (-0.5, 0.5)
__global__ void fill_sym_kernel(double* H, int n, unsigned seed) {
  const size_t nn = (size_t)n * n;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < nn; t += (size_t)gridDim.x * blockDim.x) {
    const unsigned i = (unsigned)(t % n), j = (unsigned)(t / n);
    const unsigned a = i < j ? i : j, b = i < j ? j : i;
    unsigned h = seed ^ (a * 0x9E3779B1u) ^ (b * 0x85EBCA77u);
    h ^= h >> 15;
    h *= 0x2C1B3C6Du;
    h ^= h >> 12;
    h *= 0x297A2D39u;
    h ^= h >> 15;
    H[t] = (double)h / 4294967296.0 - 0.5;
  }
}

struct DevBuf {
  void* p = nullptr;
  explicit DevBuf(size_t bytes) { NRGB_CUDA(cudaMalloc(&p, bytes)); }
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

double time_ms(cudaStream_t st, int reps, const std::function<void()>& f) {
  cudaEvent_t a, b;
  NRGB_CUDA(cudaEventCreate(&a));
  NRGB_CUDA(cudaEventCreate(&b));
  f();  // warm-up
  double best = 1e30;
  for (int r = 0; r < reps; ++r) {
    NRGB_CUDA(cudaEventRecord(a, st));
    f();
    NRGB_CUDA(cudaEventRecord(b, st));
    NRGB_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    NRGB_CUDA(cudaEventElapsedTime(&ms, a, b));
    best = std::min(best, (double)ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return best;
}

}  // namespace

std::string autotune(EigSolver& syev, int cluster_capacity, cudaStream_t st) {
  Schedule& S = schedule_here();
  std::ostringstream rep;
  rep << "{\"gemm\": [";
  // ---- GEMM tiles ----
  const int edges[] = {128, 192, 256, 384, 512, 768, 1024, 1536, 2048};
  std::vector<std::pair<int, bool>> wins;
  {
    const int emax = 2048;
    DevBuf A((size_t)emax * emax * 8), B((size_t)emax * emax * 8);
    fill_sym_kernel<<<1184, 256, 0, st>>>(A.as<double>(), emax, 1u);
    fill_sym_kernel<<<1184, 256, 0, st>>>(B.as<double>(), emax, 2u);
    NRGB_CUDA(cudaGetLastError());
    const size_t cbytes = size_t(256) << 20;
    DevBuf Cb(cbytes);
    bool first = true;
    for (int e : edges) {
      // about 2 x 2048^3 x 2 flops per launch, output within 256 MB
      int np = std::max(1, (int)lround(2.0 * pow(2048.0 / e, 3)));
      np = std::min(np, (int)(cbytes / ((size_t)e * e * 8)));
      std::vector<GemmProb> P(np);
      std::vector<GemmSeg> G(np);
      int tiles = 0, stiles = 0;
      for (int p = 0; p < np; ++p) {
        G[p] = GemmSeg{A.as<double>(), B.as<double>(), emax, emax, e, 0, 0, 1.0};
        P[p] = GemmProb{};
        P[p].C = Cb.as<double>() + (size_t)p * e * e;
        P[p].ldc = e;
        P[p].m = P[p].n = e;
        P[p].beta = 0.0;
        P[p].seg0 = p;
        P[p].nseg = 1;
        gemm_assign_tiles(P[p], tiles, stiles);
      }
      DevBuf dP(sizeof(GemmProb) * np), dG(sizeof(GemmSeg) * np);
      NRGB_CUDA(cudaMemcpyAsync(dP.p, P.data(), sizeof(GemmProb) * np, cudaMemcpyHostToDevice, st));
      NRGB_CUDA(cudaMemcpyAsync(dG.p, G.data(), sizeof(GemmSeg) * np, cudaMemcpyHostToDevice, st));
      auto run = [&] {
        NRGB_CUDA(gemm_grouped_launch(dP.as<GemmProb>(), np, dG.as<GemmSeg>(), tiles, st, "autotune", stiles));
      };
      S.gemm_large_from.store(0);
      const double t_small = time_ms(st, 3, run);
      S.gemm_large_from.store(1);
      const double t_large = time_ms(st, 3, run);
      S.gemm_large_from.store(0);
      const double fl = 2.0 * e * (double)e * e * np;
      wins.push_back({e, t_large < 0.97 * t_small});
      rep << (first ? "" : ", ") << "{\"edge\": " << e << ", \"problems\": " << np << ", \"small_tf\": "
          << fl / t_small / 1e9 << ", \"large_tf\": " << fl / t_large / 1e9 << "}";
      first = false;
    }
  }
  int large_from = 0;
  for (int i = (int)wins.size() - 1; i >= 0 && wins[i].second; --i) large_from = wins[i].first;
  S.gemm_large_from.store(large_from);
  rep << "], \"gemm_large_from\": " << large_from << ", \"cluster\": [";
  // ---- cluster limit ----
  int best_limit = 0;
  if (cluster_capacity > 0) {
    std::vector<int> ns;
    for (int k = 0; k < 24; ++k) ns.push_back(40 + (int)lround(k * (1.4 * cluster_capacity - 40) / 23.0));
    size_t tot = 0, totn = 0;
    for (int n : ns) {
      tot += (size_t)n * n;
      totn += n;
    }
    DevBuf H0(tot * 8), H(tot * 8), Z(tot * 8), W(totn * 8 + 256);
    std::vector<SyevDesc> d;
    size_t o = 0, ow = 0;
    for (int n : ns) {
      fill_sym_kernel<<<256, 256, 0, st>>>(H0.as<double>() + o, n, 7u + n);
      d.push_back(SyevDesc{n, H.as<double>() + o, W.as<double>() + ow, Z.as<double>() + o});
      o += (size_t)n * n;
      ow += n;
    }
    NRGB_CUDA(cudaGetLastError());
    std::vector<int> limits = {cluster_capacity};
    for (int l : {600, 500, 400, 333, 237}) if (l < cluster_capacity) limits.push_back(l);
    double best = 1e30;
    bool first = true;
    for (int l : limits) {
      S.cluster_limit.store(l);
      auto run = [&] {
        NRGB_CUDA(cudaMemcpyAsync(H.p, H0.p, tot * 8, cudaMemcpyDeviceToDevice, st));
        syev.solve(d, st);
      };
      const double t = time_ms(st, 3, run);
      rep << (first ? "" : ", ") << "{\"limit\": " << l << ", \"ms\": " << t << "}";
      first = false;
      if (t < best * 0.97 || l == cluster_capacity) {
        if (t < best) {
          best = t;
          best_limit = l;
        }
      }
    }
  }
  S.cluster_limit.store(best_limit == cluster_capacity ? 0 : best_limit);
  S.tuned.store(1);
  rep << "], \"cluster_limit\": " << (best_limit == cluster_capacity ? 0 : best_limit)
      << ", \"cluster_capacity\": " << cluster_capacity << "}";
  return rep.str();
}

}  // namespace nrgb
