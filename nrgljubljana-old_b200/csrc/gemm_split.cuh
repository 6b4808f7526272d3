// Split-precision grouped GEMM: FP64 products computed as exact INT8
// tensor-core products (tcgen05.mma kind::i8, INT32 accumulators in tensor
// memory) with FP64 recombination.
//
//   C_p = beta_p * C_p + sum_{s in segments(p)} alpha_s * op(A_s) op(B_s)
//
// Same problem/segment description as the FP64 grouped GEMM (GemmProb,
// GemmSeg; column-major, op = as stored or transposed).  Each row i of op(A)
// is scaled by a power of two 2^eA_i (and each column j of op(B) by 2^eB_j)
// so that its entries lie in (-1, 1), and cut into `slices` signed 7-bit
// digits:  op(A)_il = 2^eA_i sum_{p=1..S} a^(p)_il 2^(-7p) + r_il with
// |r_il| < 2^(eA_i - 7S)  (Ozaki-type splitting, Ozaki, Ogita, Oishi and
// Rump 2012, with integer slices as in the INT8 emulation of DGEMM).  Every
// slice product a^(p) b^(q) is exact in INT32; the products with the same
// p + q share one accumulator; products with p + q > S + 1 are dropped (they
// lie below the slicing error).  The result is recombined in FP64 with a
// compensated (TwoSum) sum of the S scaled accumulators, then scaled by
// 2^(eA_i + eB_j).  The error per entry is bounded by about
// k * 2^(eA_i + eB_j) * 2^(-7S) * (S + 1): with S = 8 that is below the
// rounding error bound of an FP64 product (k 2^-53 |A||B|) for rows and
// columns whose entries are of similar size.
//
// This replaces the BLAS gemm calls of the operator recalculation
// (src/recalc.cc:90-91, 268-272) and of the density matrices
// (src/dmnrg.h:382-387) in the split-precision form of a run.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"
#include "gemm_f64.cuh"

namespace nrgb {

constexpr int SPLIT_MIN_SLICES = 2;
constexpr int SPLIT_MAX_SLICES = 8;
// Largest inner dimension of one segment: the accumulator of p + q = d sums
// d - 1 <= S slice products of magnitude <= 127^2 k, which must stay below
// 2^31.  Longer segments are cut into pieces of this length.
constexpr int SPLIT_MAX_K = 16000;

// Device bytes of workspace that split_gemm_grouped needs for these
// problems (host descriptors, as for the FP64 launch).
size_t split_gemm_workspace(const GemmProb* probs, int nprob, const GemmSeg* segs, int slices);

// Slice every segment's operands into `ws` (reset by the caller; it must
// hold split_gemm_workspace bytes) and launch the tensor-core products.
// `tag` names the call site in the launch accounting.  Throws CudaError.
void split_gemm_grouped(const GemmProb* probs, int nprob, const GemmSeg* segs, int slices, DeviceArena& ws,
                        cudaStream_t st, const char* tag = "gemm_i8");

// Error flag of the split kernels' bounded waits (nonzero: a wait gave up);
// read and cleared by the host after a synchronisation.
int split_gemm_take_error(cudaStream_t st);

}  // namespace nrgb
