// Grouped, segmented-K FP64 GEMM on the FP64 tensor cores (DMMA) of sm_100a.
//
//   C_p[m_p x n_p] = beta_p * C_p + sum_{s in segments(p)} alpha_s * op(A_s) op(B_s)
//
// All matrices are column-major.  One launch covers every problem of a
// batch; a CTA computes one BM x BN tile of one problem and runs the K loop
// over all segments of that problem, so several products that accumulate
// into the same output (the rows j of a recalculation table, the
// combinations i of a density-matrix update) need no atomics and no
// ordering between launches.
//
// This is the contraction that replaces the BLAS gemm calls of
// src/recalc.cc:90-91, 268-272 and src/dmnrg.h:382-387.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace nrgb {

struct GemmSeg {
  const double* A;   // op(A) is m x k
  const double* B;   // op(B) is k x n
  int lda, ldb;
  int k;
  int transA, transB;  // 0: as stored (col-major), 1: transposed
  double alpha;
};

struct GemmProb {
  double* C;
  int ldc;
  int m, n;
  double beta;         // 0 -> C is overwritten (not read)
  int seg0, nseg;      // segment range in the segment array
  int tile0;           // first global tile index of this problem
  int tiles_n;         // number of tiles along n
  int ksplit;          // >1: the K loop is split over this many CTAs per output
                       // tile, which accumulate with atomics (C must be zero
                       // on entry and beta is ignored); 0 or 1: no split
  int stile0;          // first global 128x128 tile index (large-tile kernel)
  int stiles_n;        // number of 128x128 tiles along n
};

// Fill tile0/tiles_n/stile0/stiles_n of `p` (m, n, ksplit set) and advance
// the running tile counters of a launch.
void gemm_assign_tiles(GemmProb& p, int& tiles, int& stiles);

// Launch: problems/segments already in device memory.  total_tiles is the
// sum over problems of ceil(m/BM)*ceil(n/BN)*max(1,ksplit).  Returns cudaError_t.
// `tag` names the call site in the launch accounting (KernelStats).
// total_stiles > 0 allows the 128x128-tile kernel, chosen when the launch's
// problems are large enough that the bigger tiles waste little work.
cudaError_t gemm_grouped_launch(const GemmProb* d_probs, int nprob, const GemmSeg* d_segs,
                                int total_tiles, cudaStream_t stream, const char* tag = "gemm_f64",
                                int total_stiles = 0);

// Same launch without the library's launch accounting (no host bookkeeping,
// no events): used by the allocation-free entry point.
cudaError_t gemm_grouped_launch_unaccounted(const GemmProb* d_probs, int nprob, const GemmSeg* d_segs,
                                            int total_tiles, cudaStream_t stream);

// Algorithmic flops of a grouped launch described on the host
// (sum over problems and their segments of 2 m n k); for the launch
// accounting's work counters.
double gemm_flops(const GemmProb* probs, int nprob, const GemmSeg* segs);

// Tile sizes (exported so hosts can compute tile counts).
constexpr int GEMM_BM = 64;
constexpr int GEMM_BN = 64;
constexpr int GEMM_BK = 16;

}  // namespace nrgb
