// The context behind the C ABI's nrgb_ctx handle (shared by the files that
// implement the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "syev.cuh"
#include "truncate.cuh"
#include "../host/driver.h"

namespace nrgb {

// The reference's structure on the GPU: one solver call per block
// (dsyev per invariant subspace, src/nrg.cc:2484-2507), for comparisons.
struct PerBlockSolver : EigSolver {
  SyevBatched* s = nullptr;
  int solve(const std::vector<SyevDesc>& probs, cudaStream_t st) override {
    int l = 0;
    for (const auto& p : probs) l += s->solve(std::vector<SyevDesc>{p}, st);
    return l;
  }
};

// Device matrices of the step-plan API, named by integer handles.
struct PlanMatrix {
  double* p = nullptr;
  int rows = 0, cols = 0;
};

struct PlanState {
  std::vector<PlanMatrix> mats;  // handle = index; p == nullptr: free slot
  std::vector<int> free_slots;
  TruncState trunc;              // splitting map of the current run
  void* twork = nullptr;
  size_t twork_bytes = 0;
  void* tail_dev = nullptr;
  size_t tail_bytes = 0;
  char* tail_pin = nullptr;
  size_t tail_pin_bytes = 0;
};

}  // namespace nrgb

struct nrgb_ctx {
  int device = 0;
  std::string err;
  cudaStream_t stream = nullptr;
  std::unique_ptr<nrgb::SyevBatched> syev;
  nrgb::PerBlockSolver per_block;
  int eig_mode = 0;
  nrgb::DeviceArena scratch;
  nrgb::DeviceArena io;
  std::unique_ptr<nrgb::NrgDriver> driver;
  nrgb::PlanState plan;
};

namespace nrgb {

// The solver nrgb_set_eig_mode selected for this context.
inline EigSolver* solver_of(nrgb_ctx* ctx) {
  if (ctx->eig_mode == 1) {
    ctx->per_block.s = ctx->syev.get();
    return &ctx->per_block;
  }
  return ctx->syev.get();
}

// Run f; a thrown error becomes status 2 with its text kept in the context.
template <class F>
int guarded(nrgb_ctx* ctx, F&& f) {
  if (!ctx) return 1;
  try {
    NRGB_CUDA(cudaSetDevice(ctx->device));
    f();
    ctx->err.clear();
    return 0;
  } catch (const std::exception& e) {
    ctx->err = e.what();
    return 2;
  }
}

// Release every matrix and buffer of the step-plan API.
void plan_release(nrgb_ctx* ctx);

}  // namespace nrgb
