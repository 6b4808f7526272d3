// Device kernels of one NRG step besides the eigensolver and the GEMM.
#include <map>
#include <tuple>
#include <math.h>

#include "common.cuh"
#include "nrg_kernels.cuh"

namespace nrgb {

namespace {

__global__ void asm_diag_kernel(const AsmDiag* __restrict__ t) {
  const AsmDiag D = t[blockIdx.y];
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < D.len; r += gridDim.x * blockDim.x) {
    const size_t p = (size_t)(D.off + r) * (D.n + 1);
    const double e = D.E ? D.scale * D.E[r] : 0.0;
    D.H[p] += e + D.shift;
  }
}

// One 32x32 tile of an off-diagonal sub-block per CTA (32x8 threads).
__global__ void asm_off_kernel(const AsmOff* __restrict__ t) {
  __shared__ double tile[32][33];
  const AsmOff O = t[blockIdx.y];
  const int tiles_r = (O.rows + 31) / 32;
  const int ntiles = tiles_r * ((O.cols + 31) / 32);
  for (int tt = blockIdx.x; tt < ntiles; tt += gridDim.x) {
    const int r0 = (tt % tiles_r) * 32, c0 = (tt / tiles_r) * 32;
    // load M tile (coalesced in r), scale, write the direct block
    for (int cc = threadIdx.y; cc < 32; cc += blockDim.y) {
      const int r = r0 + threadIdx.x, c = c0 + cc;
      double v = 0.0;
      if (r < O.rows && c < O.cols) {
        v = O.M ? O.f * O.M[r + (size_t)c * O.ldm] : (r == c ? O.f : 0.0);
        O.H[(size_t)(O.offi + r) + (size_t)(O.offj + c) * O.n] += v;
      }
      tile[threadIdx.x][cc] = v;
    }
    __syncthreads();
    // mirror block H[offj + c, offi + r]: coalesced in c
    for (int rr = threadIdx.y; rr < 32; rr += blockDim.y) {
      const int c = c0 + threadIdx.x, r = r0 + rr;
      if (r < O.rows && c < O.cols)
        O.H[(size_t)(O.offj + c) + (size_t)(O.offi + r) * O.n] += tile[rr][threadIdx.x];
    }
    __syncthreads();
  }
}

__global__ void gather_diag_kernel(const DiagGather* __restrict__ g, double* __restrict__ dst) {
  const DiagGather G = g[blockIdx.y];
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < G.len; r += gridDim.x * blockDim.x)
    dst[G.dst_off + r] = G.src[(size_t)r * (G.ld + 1)];
}

// Bins::add / add_std (src/bins.h:102-131) with the positive/negative split
// of ChainSpectrumBinning::add: the (up to two) bins of one peak and the
// weights they receive; bins < 0 take nothing.
__device__ __forceinline__ void bin_targets(const BinGrid& g, double E, double w, int& k0, double& v0, int& k1,
                                            double& v1) {
  k0 = k1 = -1;
  v0 = v1 = 0.0;
  int base = 0;
  if (E < 0.0) {
    E = -E;
    base = g.nbins;
  }
  if (fabs(w) < g.discard * E) return;
  const double pos = (log10(E) - g.l0) * g.bpd;
  const long idx = (long)pos;  // truncation toward zero, as the reference's long(pos)
  if (idx < 0) {
    k0 = base;
    v0 = w;
  } else if (idx >= g.nbins - 1) {
    k0 = base + g.nbins - 1;
    v0 = w;
  } else {
    const double rem = pos - (double)idx;
    k0 = base + (int)idx;
    v0 = (1.0 - rem) * w;
    k1 = k0 + 1;
    v1 = rem * w;
  }
}

// Warp-level reduction of one contribution per lane into shared-memory bins:
// lanes that hit the same bin are found with __match_any_sync, their values
// summed by the group's lowest lane (shuffles over the group), and one atomic
// add per distinct bin remains.  Every lane of the warp calls it.
__device__ __forceinline__ void bin_add_warp(double* sbins, int k, double v) {
  const unsigned peers = __match_any_sync(0xffffffffu, k);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(peers) - 1;
  double sum = 0.0;
  for (unsigned m = peers; m; m &= m - 1) {
    const double x = __shfl_sync(peers, v, __ffs(m) - 1);
    sum += x;
  }
  if (lane == leader && k >= 0 && sum != 0.0) atomicAdd(&sbins[k], sum);
}

// One peak per lane (active lanes only) into the shared-memory bins, with
// the warp-level reduction.  Every lane of the warp calls it.
__device__ __forceinline__ void bin_add(double* sbins, const BinGrid& g, double E, double w, bool active) {
  int k0, k1;
  double v0, v1;
  if (active) {
    bin_targets(g, E, w, k0, v0, k1, v1);
  } else {
    k0 = k1 = -1;
    v0 = v1 = 0.0;
  }
  bin_add_warp(sbins, k0, v0);
  bin_add_warp(sbins, k1, v1);
}

__device__ __forceinline__ void flush_bins(const double* sbins, double* bins, int nb2) {
  __syncthreads();
  for (int i = threadIdx.x; i < nb2; i += blockDim.x) {
    const double v = sbins[i];
    if (v != 0.0) atomicAdd(&bins[i], v);
  }
}

constexpr int SPEC_NT = 256;
constexpr int SPEC_PER_CTA = 8192;

__global__ void __launch_bounds__(SPEC_NT) spec_dmnrg_kernel(const SpecDmnrgPair* __restrict__ pairs,
                                                             BinGrid g, double scale, double Emin,
                                                             double Emax, double msign,
                                                             double* __restrict__ bins) {
  extern __shared__ double sbins[];
  const int nb2 = 2 * g.nbins;
  for (int i = threadIdx.x; i < nb2; i += blockDim.x) sbins[i] = 0.0;
  __syncthreads();
  const SpecDmnrgPair P = pairs[blockIdx.y];
  const long total = (long)P.dim1 * P.dimp;
  const long e0 = (long)blockIdx.x * SPEC_PER_CTA;
  const long e1 = min(total, e0 + SPEC_PER_CTA);
  // the loop runs the same number of rounds in every lane of a warp, so the
  // warp-level binning sees whole warps
  for (long e00 = e0; e00 < e1; e00 += SPEC_NT) {
    const long e = e00 + threadIdx.x;
    bool on = e < e1;
    double dE = 0.0, w = 0.0;
    if (on) {
      const int rj = (int)(e % P.dim1), rm = (int)(e / P.dim1);
      dE = P.E1[rj] - P.Ep[rm];
      const double a = fabs(dE);
      on = !(a < Emin || a > Emax);
      if (on) {
        const size_t io = (size_t)rj + (size_t)rm * P.ldo;
        const size_t is = (size_t)rj + (size_t)rm * P.dim1;
        w = P.sf * (P.SA[is] * P.op1[io] + msign * P.SB[is] * P.op2[io]);
      }
    }
    bin_add(sbins, g, scale * dE, w, on);
  }
  flush_bins(sbins, bins, nb2);
}

__global__ void __launch_bounds__(SPEC_NT) spec_fdm_kernel(const SpecFdmPair* __restrict__ pairs,
                                                           BinGrid g, double T, double wnf,
                                                           double msign, double* __restrict__ bins) {
  extern __shared__ double sbins[];
  const int nb2 = 2 * g.nbins;
  for (int i = threadIdx.x; i < nb2; i += blockDim.x) sbins[i] = 0.0;
  __syncthreads();
  const SpecFdmPair P = pairs[blockIdx.y];
  const long total = (long)P.allj * P.alli;
  const long e0 = (long)blockIdx.x * SPEC_PER_CTA;
  const long e1 = min(total, e0 + SPEC_PER_CTA);
  for (long e00 = e0; e00 < e1; e00 += SPEC_NT) {
    const long e = e00 + threadIdx.x;
    double dE = 0.0, wg = 0.0, wl = 0.0;
    bool ong = false, onl = false;
    if (e < e1) {
      const int j = (int)(e % P.allj), i = (int)(e / P.allj);
      const size_t io = (size_t)j + (size_t)i * P.ldo;
      const double o1 = P.op1[io];
      const double Ej = P.Ej[j], Ei = P.Ei[i];
      dE = Ej - Ei;
      const bool idisc = i >= P.reti, jdisc = j >= P.retj;
      // greater correlation function
      if (idisc) {
        wg = P.sf * o1 * P.op2[io] * wnf * P.XEi[i];  // A3, A2
        ong = true;
      } else if (jdisc) {
        wg = P.sf * o1 * P.O2R[(size_t)j + (size_t)i * P.allj];  // A1
        ong = true;
      }
      // lesser correlation function
      if (idisc && jdisc) {
        wl = P.sf * o1 * P.op2[io] * msign * wnf * P.XEj[j];  // B3
        onl = true;
      } else if (idisc && !jdisc) {
        wl = P.sf * o1 * P.RO2[(size_t)j + (size_t)i * P.retj] * msign;  // B2
        onl = true;
      } else if (!idisc && jdisc) {
        wl = P.sf * o1 * P.op2[io] * msign * wnf * P.XEj[j];  // B1
        onl = true;
      }
    }
    bin_add(sbins, g, dE, wg, ong);
    bin_add(sbins, g, dE, wl, onl);
  }
  flush_bins(sbins, bins, nb2);
}

__device__ double window_fnc(double x, double nntanh) {
  if (nntanh > 0.0) {
    const double f0 = tanh(nntanh * (0.0 - 0.5)), fx = tanh(nntanh * (x - 0.5)),
                 f1 = tanh(nntanh * (1.0 - 0.5));
    return (fx - f0) / (f1 - f0);
  }
  return x;
}

__global__ void merge_bins_kernel(const double* __restrict__ chain, double* __restrict__ full,
                                  const double* __restrict__ ebins, BinGrid g, int mode, double Emin, double Ex, double Emax,
                                  double nntanh, double factor, int first, int last) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 2 * g.nbins) return;
  const double w = chain[i];
  if (mode == 0) {
    full[i] += w;
    return;
  }
  const double e = ebins[i % g.nbins];  // representative energies computed on the host
  if (!(Emin < e && e < Emax && w != 0.0)) return;
  double win;
  if (e <= Ex && last) win = 1.0;
  else if (e >= Ex && first) win = 1.0;
  else if (e <= Emin || e >= Emax) win = 0.0;
  else if (e <= Ex) win = window_fnc((e - Emin) / (Ex - Emin), nntanh);
  else win = 1.0 - window_fnc((e - Ex) / (Emax - Ex), nntanh);
  full[i] += factor * w * win;
}

__global__ void col_scale_kernel(const ColScale* __restrict__ cs) {
  const ColScale C = cs[blockIdx.y];
  const long total = (long)C.rows * C.cols;
  for (long e = (long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
    const int r = (int)(e % C.rows), c = (int)(e / C.rows);
    C.dst[(size_t)r + (size_t)c * C.ldd] = C.src[(size_t)r + (size_t)c * C.lds] * C.s[c];
  }
}

inline int cdiv(long a, long b) { return (int)((a + b - 1) / b); }

}  // namespace

cudaError_t assemble_launch(const AsmDiag* d_diag, int ndiag, const AsmOff* d_off, int noff,
                            int max_len, int max_rc, cudaStream_t st) {
  if (ndiag > 0) {
    dim3 g(max(1, min(64, cdiv(max_len, 256))), ndiag);
    NRGB_LAUNCH("assemble_diag", st, asm_diag_kernel<<<g, 256, 0, st>>>(d_diag));
  }
  if (noff > 0) {
    dim3 g(max(1, min(1024, cdiv(max_rc, 1024))), noff);
    NRGB_LAUNCH("assemble_off", st, asm_off_kernel<<<g, dim3(32, 8), 0, st>>>(d_off));
  }
  return cudaGetLastError();
}

std::vector<std::vector<AsmOff>> asm_off_layers(const std::vector<AsmOff>& terms) {
  std::vector<std::vector<AsmOff>> layers;
  std::map<std::tuple<double*, int, int>, int> seen;  // (H, lower offset, higher offset) -> terms so far
  for (const AsmOff& t : terms) {
    const int k = seen[std::make_tuple(t.H, std::min(t.offi, t.offj), std::max(t.offi, t.offj))]++;
    if ((int)layers.size() <= k) layers.resize(k + 1);
    layers[k].push_back(t);
  }
  return layers;
}

cudaError_t gather_diag_launch(const DiagGather* d_g, int ng, int max_len, double* dst, cudaStream_t st) {
  if (ng <= 0) return cudaSuccess;
  dim3 g(max(1, min(64, cdiv(max_len, 256))), ng);
  NRGB_LAUNCH("gather_diag", st, gather_diag_kernel<<<g, 256, 0, st>>>(d_g, dst));
  return cudaGetLastError();
}

cudaError_t spec_dmnrg_launch(const SpecDmnrgPair* d_pairs, int npairs, int max_elems, BinGrid g,
                              double scale, double Emin, double Emax, double msign, double* bins,
                              cudaStream_t st) {
  if (npairs <= 0 || max_elems <= 0) return cudaSuccess;
  dim3 grid(cdiv(max_elems, SPEC_PER_CTA), npairs);
  const size_t smem = 2 * (size_t)g.nbins * sizeof(double);
  NRGB_LAUNCH("spec_dmnrg", st, spec_dmnrg_kernel<<<grid, SPEC_NT, smem, st>>>(d_pairs, g, scale, Emin, Emax, msign, bins));
  return cudaGetLastError();
}

cudaError_t spec_fdm_launch(const SpecFdmPair* d_pairs, int npairs, int max_elems, BinGrid g,
                            double T, double wnf, double msign, double* bins, cudaStream_t st) {
  if (npairs <= 0 || max_elems <= 0) return cudaSuccess;
  dim3 grid(cdiv(max_elems, SPEC_PER_CTA), npairs);
  const size_t smem = 2 * (size_t)g.nbins * sizeof(double);
  NRGB_LAUNCH("spec_fdm", st, spec_fdm_kernel<<<grid, SPEC_NT, smem, st>>>(d_pairs, g, T, wnf, msign, bins));
  return cudaGetLastError();
}

cudaError_t merge_bins_launch(const double* chain, double* full, const double* ebins, BinGrid g,
                              int mode, double Emin,
                              double Ex, double Emax, double nntanh, double factor, int first,
                              int last, cudaStream_t st) {
  NRGB_LAUNCH("merge_bins", st,
              merge_bins_kernel<<<cdiv(2 * g.nbins, 256), 256, 0, st>>>(chain, full, ebins, g, mode, Emin, Ex,
                                                                        Emax, nntanh, factor, first, last));
  return cudaGetLastError();
}

cudaError_t col_scale_launch(const ColScale* d_cs, int ncs, int max_rows, int max_cols, cudaStream_t st) {
  if (ncs <= 0) return cudaSuccess;
  dim3 g(max(1, min(256, cdiv((long)max_rows * max_cols, 256))), ncs);
  NRGB_LAUNCH("col_scale", st, col_scale_kernel<<<g, 256, 0, st>>>(d_cs));
  return cudaGetLastError();
}

// --------------------------------------------------------------------------
// Broadening of binned spectra on a mesh
// --------------------------------------------------------------------------
namespace {

__device__ __forceinline__ double br_new(double e, double ept, double alpha, double gamma, double omega0) {
  const double sqpi = 1.7724538509055160273;
  double pl = 0.0;
  if (!((e < 0.0 && ept > 0.0) || (e > 0.0 && ept < 0.0) || ept == 0.0)) {
    const double x = log(e / ept) / alpha - gamma;
    pl = exp(-x * x) / (alpha * fabs(e) * sqpi);
  }
  if (fabs(e) > omega0) return pl;
  const double l = log(fabs(e) / omega0) / alpha;
  const double h = exp(-l * l);
  const double gx = (e - ept) / omega0;
  return pl * h + exp(-gx * gx) / (omega0 * sqpi) * (1.0 - h);
}

__global__ void broaden_kernel(const double* __restrict__ e, const double* __restrict__ w, int nb,
                               const double* __restrict__ mesh, int nmesh, double alpha, double gamma,
                               double omega0, double* __restrict__ out) {
  __shared__ double scratch[32];
  const int k = blockIdx.x;
  const double E = k < nmesh ? mesh[k] : -mesh[k - nmesh];
  double s = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) s += w[i] * br_new(E, e[i], alpha, gamma, omega0);
  s = block_sum(s, scratch);
  if (threadIdx.x == 0) out[k] = s;
}

}  // namespace

cudaError_t broaden_launch(const double* d_e, const double* d_w, int nb, const double* d_mesh, int nmesh,
                           double alpha, double gamma, double omega0, double* d_out, cudaStream_t st) {
  if (nmesh <= 0) return cudaSuccess;
  NRGB_LAUNCH("broaden", st,
              broaden_kernel<<<2 * nmesh, 256, 0, st>>>(d_e, d_w, nb, d_mesh, nmesh, alpha, gamma, omega0, d_out));
  return cudaGetLastError();
}

}  // namespace nrgb
