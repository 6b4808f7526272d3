// NRG iteration driver on the GPU (host side).
#pragma once
#include <cuda_runtime.h>

namespace nrgb {

class SyevBatched;

class NrgDriver {
 public:
  NrgDriver(cudaStream_t stream, SyevBatched* syev);
  ~NrgDriver();
  void run(const char* workdir, const char* outdir, double* stats);

 private:
  struct Impl;
  Impl* impl_;
};

}  // namespace nrgb
