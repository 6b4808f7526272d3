// NRG iteration driver on the GPU (host side).
#pragma once
#include <cuda_runtime.h>

namespace nrgb {

class EigSolver;

// Per-run figures beyond the eight of nrgb_run's stats array.
struct RunExtra {
  double peak_bytes = 0;   // largest device memory held by the run's data at once
  double eig_calls = 0;    // solver calls (one per NRG step of sweep 1)
};

class NrgDriver {
 public:
  NrgDriver(cudaStream_t stream, EigSolver* eig);
  ~NrgDriver();
  // stats[8]: wall, diag, recalc, dm, spec seconds, launches, h2d, d2h bytes
  void run(const char* workdir, const char* outdir, double* stats, RunExtra* extra = nullptr);

 private:
  struct Impl;
  Impl* impl_;
};

}  // namespace nrgb
