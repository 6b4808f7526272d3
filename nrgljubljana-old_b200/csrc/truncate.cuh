// Truncation of one NRG step on the device: ground-state energy, the
// reference's fixeps splitting correction, the global ordering of all
// eigenvalues, the number of retained states per block and the partial sums
// of the thermodynamics.  The host gets back one small record per step
// (ground-state energy, kept counts, per-block Boltzmann sums) instead of
// every eigenvalue.
//
//   src/nrg.cc:1420-1455   find_groundstate / subtract_groundstate_energy
//   src/splitting.cc:5-77  fix_splittings / find_clusters (with the
//                          reference's conventions: the last cluster of the
//                          sorted list is not processed, an existing
//                          mapping is never overwritten, and the mapping
//                          persists for the rest of the run)
//   src/nrg.cc:1919-1998   highest_retained_energy / nrg_truncate_prepare
//   src/nrg.cc:2333-2369   nrg_calculate_TD (partial sums per block)
#pragma once
#include <cuda_runtime.h>

namespace nrgb {

struct TruncBlock {
  double* w;  // this block's eigenvalues (ascending), inside the step's contiguous array
  int n;
  int off;    // offset of w in the step's array
};

struct TruncRules {
  double fixeps;      // splitting correction tolerance (src/param.cc fixeps)
  double keepenergy;  // <= 0: keep a fixed number
  int keep, keepmin;
  double safeguard;
  int safeguardmax;
  int keep_all;       // keep every state of the step (last step with CFS/FDM)
  double betabar;     // Boltzmann factor of the thermodynamics sums
};

// Device-side record of one step, copied to the host in one piece.
struct TruncTail {
  double Egs;         // ground-state energy subtracted from every value
  double Emax;        // highest retained energy
  int map_count;      // entries of the splitting map after this step
  int flags;          // bit 0: ground state not at zero after the shift;
                      // bit 1: a block's values not ascending after the correction
  int pad[2];
  // followed by kept[nblocks] (int, padded to 8 bytes) and
  // sums[3 * nblocks] (double: sum e^-bE, sum bE e^-bE, sum (bE)^2 e^-bE)
};

size_t trunc_tail_bytes(int nblocks);
inline const int* trunc_tail_kept(const void* tail) {
  return reinterpret_cast<const int*>(static_cast<const char*>(tail) + sizeof(TruncTail));
}
const double* trunc_tail_sums(const void* tail, int nblocks);

// Persistent state of one run: the splitting map (sorted keys with their
// replacement values, two buffers for the merge) and the step workspace.
struct TruncState {
  double* map_k[2] = {nullptr, nullptr};
  double* map_v[2] = {nullptr, nullptr};
  int cur = 0;          // buffer holding the current map
  int map_count = 0;    // host copy (from the last tail)
  int map_cap = 0;
  int* d_count = nullptr;  // device map size
};

// Workspace doubles/ints per step of `wtot` values: see truncate.cu.
size_t trunc_work_bytes(int wtot, int nblocks);

// Run the truncation of one step on `st`: values `wall` (wtot doubles, the
// blocks' arrays back to back, each ascending) are shifted by the ground
// state energy and corrected in place; `tail_dev` receives the record.
// d_blocks: nblocks TruncBlock in device memory.  `work` holds
// trunc_work_bytes.  The map buffers must hold map_count + 2 * wtot entries.
cudaError_t truncate_step(const TruncBlock* d_blocks, int nblocks, double* wall, int wtot, const TruncRules& R,
                          TruncState& S, void* work, void* tail_dev, cudaStream_t st);

}  // namespace nrgb
