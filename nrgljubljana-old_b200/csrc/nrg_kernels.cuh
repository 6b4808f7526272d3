// Device kernels of one NRG step besides the eigensolver and the GEMM:
// block-Hamiltonian assembly, gathers, spectral weights and log binning.
#pragma once
#include <vector>
#include <cuda_runtime.h>

namespace nrgb {

// ---- assembly (src/nrg.cc:2456-2478, src/matrix.cc:86-192) ----
// Diagonal segment of block b: H[off + r, off + r] = scale * E[r] + shift, r < len.
struct AsmDiag {
  double* H;       // block matrix (ld = n)
  const double* E; // ancestor eigenvalues (kept prefix), may be null for shift-only
  int n, off, len;
  double scale, shift;
};
// Off-diagonal sub-block: H[offi + r, offj + c] += f * M[r + c*ldm] and the
// symmetric entry H[offj + c, offi + r] (both triangles are filled); M null:
// the identity (f on the diagonal of a square sub-block).
struct AsmOff {
  double* H;
  const double* M;
  int n, offi, offj, rows, cols, ldm;
  double f;
};
cudaError_t assemble_launch(const AsmDiag* d_diag, int ndiag, const AsmOff* d_off, int noff,
                            int max_len, int max_rc, cudaStream_t st);
// Splits off-diagonal terms into layers in which no two terms touch the same
// sub-block or its mirror, so that the terms of one launch add without
// races (symmetries whose couplings do not conserve charge give a sub-block
// a hopping and an anomalous term).  Layers are launched one after another.
std::vector<std::vector<AsmOff>> asm_off_layers(const std::vector<AsmOff>& terms);

// ---- gathers ----
// dst[dst_off[t] + r] = src[t][r * (ld[t] + 1)] for r < len[t]  (diagonals)
struct DiagGather {
  const double* src;
  int ld, len, dst_off;
};
cudaError_t gather_diag_launch(const DiagGather* d_g, int ng, int max_len, double* dst, cudaStream_t st);

// ---- spectral weights + binning ----
struct BinGrid {
  double l0;     // log10 of the lowest grid point
  double bpd;    // bins per decade
  int nbins;
  double discard;  // discard_immediately
};

// DM-NRG pair (src/spec_DMNRG.cc:13-52): for rj < dim1, rm < dimp
//   w = sf * (SA[rj,rm] * op1[rj,rm] + msign * SB[rj,rm] * op2[rj,rm])
//   E = E1[rj] - Ep[rm], kept if Emin <= |E| <= Emax; binned at scale*E.
struct SpecDmnrgPair {
  const double* op1;  // dim1 x dimp (ld1)
  const double* op2;
  const double* SA;   // op2 * rho_p   (ld dim1)
  const double* SB;   // rho_1 * op1   (ld dim1)
  const double* E1;
  const double* Ep;
  int ldo, dim1, dimp;
  double sf;
};
// FDM pair (src/spec_FDM.cc:41-119), absolute energies, all x all states.
struct SpecFdmPair {
  const double* op1;   // allj x alli (ld ldo)
  const double* op2;
  const double* O2R;   // op2[:allj, :reti] * rho_i  (allj x reti, ld allj), may be null
  const double* RO2;   // rho_j * op2[:retj, :alli] (retj x alli, ld retj), may be null
  const double* Ej;    // absolute energies (shifted by the ground state)
  const double* Ei;
  const double* XEj;   // their Boltzmann factors exp(-E/T), one per state
  const double* XEi;
  int ldo, allj, alli, retj, reti;
  double sf;
};
// bins: [pos(nbins) | neg(nbins)] accumulated with atomics.
cudaError_t spec_dmnrg_launch(const SpecDmnrgPair* d_pairs, int npairs, int max_elems, BinGrid g,
                              double scale, double Emin, double Emax, double msign, double* bins,
                              cudaStream_t st);
cudaError_t spec_fdm_launch(const SpecFdmPair* d_pairs, int npairs, int max_elems, BinGrid g,
                            double T, double wnf, double msign, double* bins, cudaStream_t st);

// Merge chain bins into the full spectrum: FDM adds; DM-NRG applies the
// N/N+2 window (src/spectrumrealfreq.cc:96-185) to bins with Emin<e<Emax.
cudaError_t merge_bins_launch(const double* chain, double* full, const double* ebins, BinGrid g,
                              int mode, double Emin,
                              double Ex, double Emax, double nntanh, double factor, int first,
                              int last, cudaStream_t st);

// Column scaling: dst[:, c] = src[:, c] * s[c] for c < cols (rows x cols, ld).
struct ColScale {
  const double* src;
  double* dst;
  const double* s;
  int rows, cols, lds, ldd;
};
cudaError_t col_scale_launch(const ColScale* d_cs, int ncs, int max_rows, int max_cols, cudaStream_t st);

// Broadened spectral function on a mesh (SpectrumRealFreq::continuous with
// the BR_NEW kernel, src/spectrumrealfreq.cc:271-306, src/spectral.h:70-102):
// out[k] = sum_i w[i] K(E_k, e[i]) for E_k = mesh[k] (k < nmesh) and
// E_k = -mesh[k - nmesh], with K the log-Gaussian of width alpha (shifted by
// gamma) blended into a Gaussian of width omega0 below |E| = omega0.
// e[] are the signed bin energies, w[] their weights.  One CTA per point.
cudaError_t broaden_launch(const double* d_e, const double* d_w, int nb, const double* d_mesh, int nmesh,
                           double alpha, double gamma, double omega0, double* d_out, cudaStream_t st);

}  // namespace nrgb
