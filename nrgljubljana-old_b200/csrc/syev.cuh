// Batched FP64 symmetric eigensolver for the invariant-subspace blocks of one
// NRG step (replaces the per-block LAPACK dsyev of src/diag.h:54-89).
//
// Each problem: A (n x n, column-major, both triangles filled) -> eigenvalues
// w (ascending) and orthonormal eigenvectors Z (n x n, column-major, column r
// is the eigenvector of w[r]; ldz == n).  A is destroyed.
//
// Pipeline (all problems of a batch advance together):
//   n <= 32 : one warp per problem, Householder + implicit QR in shared memory.
//   n  > 32 : 1) blocked Householder tridiagonalisation (panel of 32 columns
//                in a cooperative persistent kernel, trailing rank-64 update on
//                the DMMA GEMM),
//             2) divide and conquer on the tridiagonal (Cuppen splitting,
//                Gu-Eisenstat eigenvectors), merges of equal tree height of all
//                problems in the same launches,
//             3) back-transformation with blocked (WY) reflectors on the GEMM.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"

namespace nrgb {

struct SyevDesc {
  int n;
  double* A;   // n x n input (lda = n), destroyed
  double* w;   // n eigenvalues (ascending)
  double* Z;   // n x n eigenvectors (ld = n); must not alias A
};

// Diagonalises a batch of problems whose inputs are ordered on `stream`, and
// returns once the results are complete in device memory.  Implemented by
// the direct solver below and by a server's batcher, which merges the
// batches of several concurrent runs into one solver call.  Returns the
// number of kernel launches made for the batch.  Throws CudaError on failure.
class EigSolver {
 public:
  virtual ~EigSolver() = default;
  virtual int solve(const std::vector<SyevDesc>& probs, cudaStream_t stream) = 0;
  // A run brackets the part of its work that calls solve() (its first
  // sweep); a merging solver waits only for runs inside that part.
  virtual void client_enter() {}
  virtual void client_leave() {}
};

class SyevBatched : public EigSolver {
 public:
  SyevBatched();
  ~SyevBatched();
  int solve(const std::vector<SyevDesc>& probs, cudaStream_t stream) override {
    run(probs, stream);
    return launches_;
  }
  // Solve all problems on `stream`.  Throws CudaError on failure (including
  // a convergence failure or a barrier timeout reported by the kernels).
  void run(const std::vector<SyevDesc>& probs, cudaStream_t stream);
  // Device bytes of workspace that run() will reserve for these sizes.
  static size_t workspace_bytes(const std::vector<int>& n);
  // Launch statistics of the last run().
  int last_launches() const { return launches_; }
  // Largest block the cluster tridiagonalisation holds (0: cluster path off);
  // larger blocks also take the cooperative panel launches.
  int cluster_nmax() const { return cl_use(); }
  // The cluster kernel's capacity, before the schedule's limit.
  int cluster_capacity() const { return cl_nmax_; }
  // Bound of the grid-barrier waits of the panel launches: 2^poll_log2 polls
  // (default 23, about a second) before a wait gives up with an error.
  void set_wait_limit(int poll_log2) { wait_log2_ = poll_log2; }
  // Host-side fault injection: while on, every panel launch's barriers
  // expect one CTA more than is launched (a lost CTA), so each wait must
  // run out; run() then throws "grid barrier timed out".
  void inject_barrier_shortfall(bool on) { inject_shortfall_ = on; }

 private:
  DeviceArena arena_;
  int* d_err_ = nullptr;
  GridBarrier* d_bar_ = nullptr;
  int launches_ = 0;
  int wait_log2_ = 23;
  bool inject_shortfall_ = false;
  int coop_ctas_ = 0;
  int sms_ = 0;
  int cl_max_[17] = {};               // resident clusters of CL = 1..16 CTAs (0: not usable or not built)
  size_t cl_smem_ = 0;                // shared memory per CTA of the cluster kernel
  int cl_nmax_ = 0;                   // largest block it holds (0: cluster path off)
  int cl_one_ = 1;                    // cluster kernel: 0 two barriers per column, 1 one, 2 one and fused
  // dynamic shared memory of one CTA of the cluster kernel in use
  size_t trdc_bytes(int n, int cl) const;
  // blocks up to this size go to the cluster kernel whole: the capacity, or
  // the schedule's limit when it is lower (schedule.cuh)
  int cl_use() const;
  // side streams on which the cluster launches of different sizes overlap
  static constexpr int NAUX = 16;
  int naux_ = NAUX;  // side streams in use (NRGB_SIDE_STREAMS, for comparisons)
  cudaStream_t aux_[NAUX] = {};
  cudaEvent_t fork_ = nullptr, join_[NAUX] = {};
  // the warp solver for blocks up to 32 runs beside the larger blocks' work
  cudaStream_t small_st_ = nullptr;
  cudaEvent_t small_done_ = nullptr;
};

}  // namespace nrgb
