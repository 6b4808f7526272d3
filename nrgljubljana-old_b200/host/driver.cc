// NRG iteration on the GPU: the two sweeps of src/nrg.cc:3429-3469
// (start_calculation) with every O(n^2)/O(n^3) stage on the device and the
// reference's host-side decisions (subspace lists, truncation, thermodynamics,
// output files) kept on the host.
//
//   sweep 1 (src/nrg.cc:3106-3118, 2881-3040): per step N
//     subspaces + ancestors (2415-2430, 2753-2781)      host
//     block Hamiltonians (2456-2478, matrix.cc)          assemble kernels
//     eigen-decomposition (diag.h:54-89)                 SyevBatched
//     ground state, fixeps clusters, truncation          host (Sigma n values)
//     thermodynamics td (2333-2369)                      host
//     <f> recalculation (recalc.cc:12-97)                grouped DMMA GEMM
//     singlet operators + expectation values             grouped DMMA GEMM
//   density matrices (dmnrg.h:327-596)                   grouped DMMA GEMM
//   sweep 2: doublet/triplet operators, spectral weights (spec_DMNRG.cc,
//     spec_FDM.cc) and log binning (bins.h)              GEMM + spectral kernels
//
// Eigenvectors and density matrices stay resident in device memory for the
// whole run (the reference stores them in unitary*/rho* files).
#include "driver.h"

#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <fstream>
#include <iomanip>
#include <map>
#include <memory>
#include <set>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "../csrc/common.cuh"
#include "../csrc/gemm_f64.cuh"
#include "../csrc/gemm_split.cuh"
#include "../csrc/nrg_kernels.cuh"
#include "../csrc/syev.cuh"
#include "../csrc/truncate.cuh"
#include "data.h"
#include "params.h"
#include "symmetry.h"

namespace nrgb {

namespace {

using Clock = std::chrono::steady_clock;
double secs(Clock::time_point a) { return std::chrono::duration<double>(Clock::now() - a).count(); }

struct DevMat {
  double* p = nullptr;
  int rows = 0, cols = 0, ld = 0;
  DevMat view(int r, int c) const { return DevMat{p, r, c, ld}; }
};
using DevBlocks = std::map<Twoinvar, DevMat>;

// Device bytes held by the slabs of one run (current and peak).
struct MemCount {
  size_t cur = 0, peak = 0;
};
// The run executing on this host thread (set for the duration of run()).
thread_local MemCount* tl_mem = nullptr;

// Stream-ordered device memory owned by one generation of data.  Requests
// are carved out of chunks (256-byte aligned) so that thousands of operator
// blocks per step cost a handful of cudaMallocAsync/cudaFreeAsync calls;
// chunks grow geometrically from 1 MiB to 64 MiB (a larger request gets a
// chunk of its own size).
class Slab {
 public:
  explicit Slab(cudaStream_t s) : st_(s), mc_(tl_mem) {}
  ~Slab() { release(); }
  Slab(const Slab&) = delete;
  double* alloc(size_t n) {
    if (n == 0) return nullptr;
    const size_t bytes = (n * sizeof(double) + 255) & ~size_t(255);
    if (chunks_.empty() || off_ + bytes > chunks_.back().second) {
      const size_t sz = std::max(bytes, next_);
      next_ = std::min(next_ * 2, size_t(64) << 20);
      void* p = nullptr;
      NRGB_CUDA(cudaMallocAsync(&p, sz, st_));
      chunks_.push_back({p, sz});
      off_ = 0;
      if (mc_) {
        mc_->cur += sz;
        mc_->peak = std::max(mc_->peak, mc_->cur);
      }
    }
    char* p = static_cast<char*>(chunks_.back().first) + off_;
    off_ += bytes;
    return reinterpret_cast<double*>(p);
  }
  void release() {
    for (auto& c : chunks_) {
      cudaFreeAsync(c.first, st_);
      if (mc_) mc_->cur -= c.second;
    }
    chunks_.clear();
    off_ = 0;
    next_ = size_t(1) << 20;
  }

 private:
  cudaStream_t st_;
  MemCount* mc_;
  std::vector<std::pair<void*, size_t>> chunks_;
  size_t off_ = 0;
  size_t next_ = size_t(1) << 20;
};

struct Block {
  int dim = 0;
  std::vector<int> rmax, off;
  std::vector<Invar> anc;
  double* Z = nullptr;  // dim x dim eigenvectors (device)
  double* w = nullptr;  // dim eigenvalues, GS-subtracted and cluster-fixed (device)
  std::vector<double> value;  // same on the host
  std::vector<double> absE;   // absolute energies (not yet shifted by the GS energy)
  double shift = 0.0;
  int kept = 0;
};

struct Step {
  std::map<Invar, Block> blocks;
  double Egs = 0.0, scale = 0.0;
  double total = 0.0;       // total energy after this step
  double* wall = nullptr;   // the blocks' eigenvalues back to back (device)
  int wtot = 0;
  std::unique_ptr<Slab> slab;
};

// Singlet expectation values of one step, gathered on the device and
// evaluated once the step's eigenvalues are on the host.
struct ExpvDeferred {
  size_t step;
  double T;
  const double* diag = nullptr;  // gathered diagonals (device)
  std::vector<std::pair<std::string, Invar>> order;
  std::vector<int> len;
};

struct Prev {
  const double* w = nullptr;
  int kept = 0;
};

// A grouped GEMM under construction (host side), launched in one go.
struct Grouped {
  std::vector<GemmProb> probs;
  std::vector<GemmSeg> segs;
  int tiles = 0, stiles = 0;
  void out(double* C, int ldc, int m, int n, double beta, const std::vector<GemmSeg>& ss) {
    if (m <= 0 || n <= 0) return;
    GemmProb p{};
    p.C = C;
    p.ldc = ldc;
    p.m = m;
    p.n = n;
    p.beta = beta;
    p.seg0 = (int)segs.size();
    p.nseg = (int)ss.size();
    gemm_assign_tiles(p, tiles, stiles);
    segs.insert(segs.end(), ss.begin(), ss.end());
    probs.push_back(p);
  }
};

GemmSeg seg(const double* A, int lda, int ta, const double* B, int ldb, int tb, int k, double alpha) {
  GemmSeg s{};
  s.A = A;
  s.lda = lda;
  s.transA = ta;
  s.B = B;
  s.ldb = ldb;
  s.transB = tb;
  s.k = k;
  s.alpha = alpha;
  return s;
}

std::string fmt_g(double x, int prec) {
  std::ostringstream o;
  o << std::setprecision(prec) << x;
  return o.str();
}

}  // namespace

struct NrgDriver::Impl {
  cudaStream_t st;
  EigSolver* syev;
  Params P;
  DataFile D;
  std::unique_ptr<Symmetry> sym;
  int Nmax = 0, Ninit = 0;
  std::vector<Step> steps;
  double totalenergy = 0.0, GSenergy = 0.0;
  std::vector<std::vector<double>> td_rows;
  std::vector<std::pair<double, std::map<std::string, double>>> expv_rows;
  // per measured step: energy scale, total energy, all (energy, subspace) pairs
  struct Annotated {
    double scale, total;
    std::vector<std::pair<double, Invar>> levels;
  };
  std::vector<Annotated> annotated;
  // statistics
  double t_diag = 0, t_recalc = 0, t_dm = 0, t_spec = 0;
  double launches = 0, h2d = 0, d2h = 0;
  // wall time per named section, reported on stderr when NRGB_TIMING is set
  // (the counterpart of the reference's Timing report, src/nrg.h:136-190)
  std::map<std::string, double> sections;
  struct Section {
    Impl* d;
    const char* name;
    Clock::time_point t0;
    Section(Impl* d_, const char* n) : d(d_), name(n), t0(Clock::now()) {}
    ~Section() { d->sections[name] += secs(t0); }
  };
  // device scratch for descriptors
  DeviceArena desc;
  size_t desc_off = 0;

  // device truncation: splitting map, step workspace, the per-step record
  TruncState tstate;
  void* twork = nullptr;
  size_t twork_bytes = 0;
  void* tail_dev = nullptr;
  size_t tail_dev_bytes = 0;
  char* tail_pin = nullptr;
  size_t tail_pin_bytes = 0;
  std::vector<ExpvDeferred> expv_def;
  std::unique_ptr<Slab> expv_slab;
  void free_trunc() {
    for (int i = 0; i < 2; ++i) {
      if (tstate.map_k[i]) cudaFreeAsync(tstate.map_k[i], st);
      if (tstate.map_v[i]) cudaFreeAsync(tstate.map_v[i], st);
      tstate.map_k[i] = tstate.map_v[i] = nullptr;
    }
    if (tstate.d_count) cudaFreeAsync(tstate.d_count, st);
    tstate = TruncState();
    if (twork) cudaFreeAsync(twork, st);
    twork = nullptr;
    twork_bytes = 0;
    if (tail_dev) cudaFreeAsync(tail_dev, st);
    tail_dev = nullptr;
    tail_dev_bytes = 0;
  }
  // Map buffers that hold `need` entries (the current map is copied over).
  void ensure_map(int need) {
    if (need <= tstate.map_cap) return;
    int cap = std::max(4096, tstate.map_cap);
    while (cap < need) cap *= 2;
    double *nk[2], *nv[2];
    for (int i = 0; i < 2; ++i) {
      NRGB_CUDA(cudaMallocAsync((void**)&nk[i], sizeof(double) * cap, st));
      NRGB_CUDA(cudaMallocAsync((void**)&nv[i], sizeof(double) * cap, st));
    }
    if (!tstate.d_count) {
      NRGB_CUDA(cudaMallocAsync((void**)&tstate.d_count, sizeof(int), st));
      NRGB_CUDA(cudaMemsetAsync(tstate.d_count, 0, sizeof(int), st));
    }
    const int c = tstate.cur;
    if (tstate.map_count > 0) {
      NRGB_CUDA(cudaMemcpyAsync(nk[c], tstate.map_k[c], sizeof(double) * tstate.map_count, cudaMemcpyDeviceToDevice, st));
      NRGB_CUDA(cudaMemcpyAsync(nv[c], tstate.map_v[c], sizeof(double) * tstate.map_count, cudaMemcpyDeviceToDevice, st));
    }
    for (int i = 0; i < 2; ++i) {
      if (tstate.map_k[i]) cudaFreeAsync(tstate.map_k[i], st);
      if (tstate.map_v[i]) cudaFreeAsync(tstate.map_v[i], st);
      tstate.map_k[i] = nk[i];
      tstate.map_v[i] = nv[i];
    }
    tstate.map_cap = cap;
  }

  MemCount mem;
  double eig_calls = 0;
  std::vector<double> wstage;  // host staging of per-step eigenvalue uploads

  Impl(cudaStream_t s, EigSolver* e) : st(s), syev(e) {}
  ~Impl() {
    free_trunc();
    cudaStreamSynchronize(st);
    if (desc_pin) cudaFreeHost(desc_pin);
    if (tail_pin) cudaFreeHost(tail_pin);
  }
  Impl(const Impl&) = delete;
  Impl& operator=(const Impl&) = delete;

  // ---------------- small helpers ----------------
  // Launch descriptors: the first DESC_PINNED bytes of the descriptor arena
  // have a pinned host mirror, so their uploads are plain DMA (a pageable
  // source goes through the CUDA driver's staging buffer, which the run
  // threads of a server share).  The mirror is rewritten only after
  // desc_reset(), which waits for the stream.
  static constexpr size_t DESC_PINNED = 4 << 20;
  char* desc_pin = nullptr;
  template <class T>
  T* upload(const std::vector<T>& v) {
    if (v.empty()) return nullptr;
    const size_t bytes = v.size() * sizeof(T);
    T* d = static_cast<T*>(desc.alloc(bytes));
    const size_t off = desc.offset_of(d);
    if (desc_pin && off + bytes <= DESC_PINNED) {
      memcpy(desc_pin + off, v.data(), bytes);
      NRGB_CUDA(cudaMemcpyAsync(d, desc_pin + off, bytes, cudaMemcpyHostToDevice, st));
    } else {
      NRGB_CUDA(cudaMemcpyAsync(d, v.data(), bytes, cudaMemcpyHostToDevice, st));
    }
    h2d += bytes;
    return d;
  }
  void desc_reset() {
    // descriptors of the previous launches must not be overwritten while in use
    NRGB_CUDA(cudaStreamSynchronize(st));
    desc.reset();
  }
  DeviceArena split_ws;  // operand slices of the split-precision products
  void run_gemm(const Grouped& g) {
    if (g.probs.empty()) return;
    if (P.gemm_slices > 0) {
      // split precision: INT8 slices on the tensor cores (the launches of
      // one stream run in order, so the workspace is reused call to call)
      split_ws.reserve(split_gemm_workspace(g.probs.data(), (int)g.probs.size(), g.segs.data(), P.gemm_slices));
      split_ws.reset();
      split_gemm_grouped(g.probs.data(), (int)g.probs.size(), g.segs.data(), P.gemm_slices, split_ws, st,
                         "gemm_i8_nrg");
      launches += 3;
      return;
    }
    GemmProb* dp = upload(g.probs);
    GemmSeg* ds = upload(g.segs);
    KernelStats::get().add_work("gemm_f64_nrg", gemm_flops(g.probs.data(), (int)g.probs.size(), g.segs.data()));
    NRGB_CUDA(gemm_grouped_launch(dp, (int)g.probs.size(), ds, g.tiles, st, "gemm_f64_nrg", g.stiles));
    launches += 1;
  }
  DevMat upload_mat(const HostMat& M, Slab& slab) {
    DevMat d;
    d.rows = M.rows;
    d.cols = M.cols;
    d.ld = std::max(1, M.rows);
    d.p = slab.alloc((size_t)M.rows * M.cols);
    if (d.p) {
      NRGB_CUDA(cudaMemcpyAsync(d.p, M.a.data(), M.a.size() * sizeof(double), cudaMemcpyHostToDevice, st));
      h2d += M.a.size() * sizeof(double);
    }
    return d;
  }
  DevBlocks upload_blocks(const HostBlocks& b, Slab& slab) {
    DevBlocks out;
    for (const auto& kv : b) out[kv.first] = upload_mat(kv.second, slab);
    return out;
  }
  std::vector<double> download(const double* p, size_t n) {
    std::vector<double> h(n);
    if (n) {
      NRGB_CUDA(cudaMemcpyAsync(h.data(), p, n * sizeof(double), cudaMemcpyDeviceToHost, st));
      NRGB_CUDA(cudaStreamSynchronize(st));
      d2h += n * sizeof(double);
    }
    return h;
  }
  bool last(int N) const { return N + 1 == Nmax; }
  bool cfs_flags() const { return P.cfs || P.fdm; }

  // ---------------- recalculation of operator matrix elements ----------------
  // Target k1 x kp block for (I1, Ip): sum over table rows of
  //   factor * U1^T * O(IN1,INp) * Up  with U = Z[off : off+r, 0 : k]
  // (src/recalc.cc:164-281).  O empty (null) -> recalc_f form U1^T Up.
  struct Term {
    double factor;
    const Block* B1;
    int i1;
    const Block* Bp;
    int ip;
    DevMat O;
    bool f_form;
  };
  struct Target {
    Twoinvar II;
    int k1, kp;
    std::vector<Term> terms;
  };

  DevBlocks compute_targets(std::vector<Target>& tg, Slab& slab) {
    DevBlocks out;
    // stage 1: temp = O * Zp_sub  (r1 x kp) for every general term
    Grouped g1, g2;
    std::vector<std::vector<double*>> temps(tg.size());
    for (size_t t = 0; t < tg.size(); ++t) {
      for (const Term& x : tg[t].terms) {
        double* T = nullptr;
        if (!x.f_form) {
          const int r1 = x.B1->rmax[x.i1], rp = x.Bp->rmax[x.ip];
          T = slab.alloc((size_t)r1 * tg[t].kp);
          g1.out(T, r1, r1, tg[t].kp, 0.0,
                 {seg(x.O.p, x.O.ld, 0, x.Bp->Z + x.Bp->off[x.ip], x.Bp->dim, 0, rp, 1.0)});
        }
        temps[t].push_back(T);
      }
    }
    for (size_t t = 0; t < tg.size(); ++t) {
      DevMat C;
      C.rows = tg[t].k1;
      C.cols = tg[t].kp;
      C.ld = std::max(1, tg[t].k1);
      C.p = slab.alloc((size_t)C.rows * C.cols);
      out[tg[t].II] = C;
      if (!C.p) continue;
      std::vector<GemmSeg> ss;
      for (size_t j = 0; j < tg[t].terms.size(); ++j) {
        const Term& x = tg[t].terms[j];
        const int r1 = x.B1->rmax[x.i1];
        if (x.f_form)
          ss.push_back(seg(x.B1->Z + x.B1->off[x.i1], x.B1->dim, 1, x.Bp->Z + x.Bp->off[x.ip], x.Bp->dim, 0,
                           r1, x.factor));
        else
          ss.push_back(seg(x.B1->Z + x.B1->off[x.i1], x.B1->dim, 1, temps[t][j], r1, 0, r1, x.factor));
      }
      if (ss.empty()) {
        NRGB_CUDA(cudaMemsetAsync(C.p, 0, (size_t)C.rows * C.cols * sizeof(double), st));
      } else {
        g2.out(C.p, C.ld, C.rows, C.cols, 0.0, ss);
      }
    }
    run_gemm(g1);
    run_gemm(g2);
    return out;
  }

  // <f> blocks of the new last site (recalc_irreduc + recalc_f).
  std::vector<DevBlocks> recalc_f(const Step& S, Slab& slab) {
    std::vector<std::vector<Target>> per(P.channels);
    for (const auto& kv : S.blocks) {
      const Invar& Ip = kv.first;
      const Block& Bp = kv.second;
      for (const RecalcTable& tab : sym->recalc_f(Ip)) {
        auto it = S.blocks.find(tab.Ip);  // tab.Ip holds I1 here
        if (it == S.blocks.end()) continue;
        const Block& B1 = it->second;
        if (B1.kept == 0 || Bp.kept == 0) continue;
        Target t{{tab.Ip, Ip}, B1.kept, Bp.kept, {}};
        for (const RecalcRow& r : tab.rows) {
          const int r1 = B1.rmax[r.i1 - 1], rp = Bp.rmax[r.ip - 1];
          if (!(r1 > 0 && rp > 0)) continue;
          if (r1 != rp) throw std::runtime_error("recalc_f: rmax mismatch");
          t.terms.push_back(Term{r.factor, &B1, r.i1 - 1, &Bp, r.ip - 1, DevMat{}, true});
        }
        per[tab.ch].push_back(std::move(t));
      }
    }
    std::vector<DevBlocks> out(P.channels);
    for (int ch = 0; ch < P.channels; ++ch) out[ch] = compute_targets(per[ch], slab);
    return out;
  }

  // recalc_singlet / recalc_doublet / recalc_triplet through recalc_general.
  DevBlocks recalc_op(char kind, const Step& S, const DevBlocks& cold, bool all_states, Slab& slab) {
    auto nst = [&](const Block& b) { return all_states ? b.dim : b.kept; };
    std::vector<Target> tg;
    const Invar Iop = kind == 's' ? sym->singlet() : kind == 'd' ? sym->doublet() : sym->triplet();
    for (const auto& kv : S.blocks) {
      const Invar& I1 = kv.first;
      const Block& B1 = kv.second;
      std::vector<RecalcTable> tabs;
      if (kind == 's') {
        RecalcTable t{I1, 0, {}};
        for (int i = 1; i <= sym->combs(); ++i) t.rows.push_back({i, i, 1.0});
        tabs.push_back(t);
      } else if (kind == 'd') {
        tabs = sym->recalc_doublet(I1);
      } else {
        tabs = sym->recalc_triplet(I1);
      }
      for (const RecalcTable& tab : tabs) {
        const Invar& Ip = tab.Ip;
        auto it = S.blocks.find(Ip);
        if (it == S.blocks.end()) continue;
        const Block& Bp = it->second;
        if (!sym->connects(I1, Ip, Iop)) continue;
        Target t{{I1, Ip}, nst(B1), nst(Bp), {}};
        if (t.k1 > 0 && t.kp > 0) {
          for (const RecalcRow& r : tab.rows) {
            const Invar IN1 = Symmetry::combine(sym->In()[r.i1 - 1], I1);
            const Invar INp = Symmetry::combine(sym->In()[r.ip - 1], Ip);
            if (!sym->allowed(IN1) || !sym->allowed(INp)) continue;
            const int r1 = B1.rmax[r.i1 - 1], rp = Bp.rmax[r.ip - 1];
            if (r1 == 0 || rp == 0) continue;
            auto ot = cold.find({IN1, INp});
            const bool cnt = ot != cold.end();
            if (!sym->connects(IN1, INp, Iop) && !cnt) continue;
            if (!cnt) throw std::runtime_error("recalc: cold.count(ININ) != 1");
            if (!std::isfinite(r.factor)) throw std::runtime_error("recalc: factor not finite");
            if (ot->second.rows < r1 || ot->second.cols < rp) throw std::runtime_error("recalc: operator too small");
            t.terms.push_back(Term{r.factor, &B1, r.i1 - 1, &Bp, r.ip - 1, ot->second.view(r1, rp), false});
          }
        }
        tg.push_back(std::move(t));
      }
    }
    return compute_targets(tg, slab);
  }

  std::vector<double> td(const Step& S, int N) {
    const double f = P.betabar;
    double Z = 0, E = 0, E2 = 0;
    std::vector<std::pair<Invar, const std::vector<double>*>> bl;
    for (const auto& kv : S.blocks) {
      double sZ = 0, sE = 0, sE2 = 0;
      for (double x : kv.second.value) {
        const double bE = f * x, ex = exp(-bE);
        sE += bE * ex;
        sE2 += bE * bE * ex;
        sZ += ex;
      }
      const int m = sym->mult(kv.first);
      Z += m * sZ;
      E += m * sE;
      E2 += m * sE2;
      bl.push_back({kv.first, &kv.second.value});
    }
    E /= Z;
    E2 /= Z;
    const double C = E2 - E * E, F = -log(Z), Sent = E - F;
    std::vector<double> row = {scale_of(P, N + 1) / P.betabar};
    for (double v : sym->td_values(bl, f, Z)) row.push_back(v);
    for (double v : {E, E2, C, F, Sent}) row.push_back(v);
    return row;
  }

  // docalc0 (src/nrg.cc:3063-3070, called from start_run at 3183-3186):
  // td, annotated energies and singlet expectation values of the initial
  // cluster from `data`, at N = Ninit-1 (temperature SCALE(Ninit)/betabar,
  // STAT::set_N at src/nrg.cc:545-553), over all states of the cluster.
  void calc0() {
    Step S0;
    for (const auto& kv : D.energies) {
      Block b;
      b.dim = (int)kv.second.size();
      b.value = kv.second;
      b.kept = b.dim;
      S0.blocks[kv.first] = std::move(b);
    }
    td_rows.push_back(td(S0, Ninit - 1));
    const double sc0 = scale_of(P, Ninit);
    if (P.dumpannotated) {
      std::vector<std::pair<double, Invar>> l;
      for (const auto& kv : S0.blocks)
        for (double x : kv.second.value) l.push_back({x, kv.first});
      std::sort(l.begin(), l.end());
      annotated.push_back({sc0, totalenergy, std::move(l)});
    }
    std::map<std::string, double> row;
    if (D.ops.count('s')) {
      double Zs = 0;
      for (const auto& kv : S0.blocks)
        for (double x : kv.second.value) Zs += sym->mult(kv.first) * exp(-P.betabar * x);
      for (const auto& op : D.ops.at('s')) {
        double tr = 0;
        for (const auto& kv : S0.blocks) {
          auto it = op.second.find({kv.first, kv.first});
          if (it == op.second.end()) throw std::runtime_error("calc0: singlet operator block missing");
          const HostMat& M = it->second;
          double s = 0;
          for (int r = 0; r < kv.second.dim; ++r) s += exp(-P.betabar * kv.second.value[r]) * M.a[(size_t)r * M.cols + r];
          tr += sym->mult(kv.first) * s;
        }
        row[op.first] = tr / Zs;
      }
    }
    expv_rows.push_back({sc0 / P.betabar, row});
  }

  // nrg_calculate_TD (src/nrg.cc:2333-2369) from the per-block sums of
  // e^-bE, bE e^-bE and (bE)^2 e^-bE computed on the device
  std::vector<double> td_sums(const Step& S, int N, const double* sums) {
    double Z = 0, E = 0, E2 = 0;
    std::vector<std::pair<Invar, double>> zs;
    size_t b = 0;
    for (const auto& kv : S.blocks) {
      const int m = sym->mult(kv.first);
      Z += m * sums[3 * b];
      E += m * sums[3 * b + 1];
      E2 += m * sums[3 * b + 2];
      zs.push_back({kv.first, sums[3 * b]});
      ++b;
    }
    E /= Z;
    E2 /= Z;
    const double C = E2 - E * E, F = -log(Z), Sent = E - F;
    std::vector<double> row = {scale_of(P, N + 1) / P.betabar};
    for (double v : sym->td_values_sums(zs, Z)) row.push_back(v);
    for (double v : {E, E2, C, F, Sent}) row.push_back(v);
    return row;
  }

  // The eigenvalues of every step of sweep 1 to the host, once the sweep
  // is done (one copy per step, one synchronisation): absolute energies,
  // the energy flow and the deferred expectation values.
  void finish_sweep1() {
    std::vector<std::vector<double>> hv(steps.size());
    for (size_t k = 0; k < steps.size(); ++k) {
      hv[k].resize(steps[k].wtot);
      NRGB_CUDA(cudaMemcpyAsync(hv[k].data(), steps[k].wall, steps[k].wtot * sizeof(double), cudaMemcpyDeviceToHost, st));
      d2h += steps[k].wtot * sizeof(double);
    }
    std::vector<std::vector<double>> hd(expv_def.size());
    for (size_t k = 0; k < expv_def.size(); ++k) {
      size_t n = 0;
      for (int l : expv_def[k].len) n += l;
      hd[k].resize(n);
      if (n) {
        NRGB_CUDA(cudaMemcpyAsync(hd[k].data(), expv_def[k].diag, n * sizeof(double), cudaMemcpyDeviceToHost, st));
        d2h += n * sizeof(double);
      }
    }
    NRGB_CUDA(cudaStreamSynchronize(st));
    for (size_t k = 0; k < steps.size(); ++k) {
      Step& S = steps[k];
      size_t o = 0;
      for (auto& kv : S.blocks) {
        Block& b = kv.second;
        b.value.assign(hv[k].begin() + o, hv[k].begin() + o + b.dim);
        o += b.dim;
        b.absE.resize(b.dim);
        for (int r = 0; r < b.dim; ++r) b.absE[r] = S.total + b.value[r] * S.scale;
      }
      if (P.dumpannotated) {
        std::vector<std::pair<double, Invar>> l;
        for (const auto& kv : S.blocks)
          for (double x : kv.second.value) l.push_back({x, kv.first});
        std::sort(l.begin(), l.end());
        annotated.push_back({S.scale, S.total, std::move(l)});
      }
    }
    // expectation values of singlet operators (nrg_measure_singlet, src/nrg.cc:2226-2236)
    for (size_t k = 0; k < expv_def.size(); ++k) {
      const ExpvDeferred& x = expv_def[k];
      const Step& S = steps[x.step];
      std::map<std::string, double> row;
      double Zs = 0;
      for (const auto& kv : S.blocks)
        for (int r = 0; r < kv.second.kept; ++r) Zs += sym->mult(kv.first) * exp(-P.betabar * kv.second.value[r]);
      size_t p = 0;
      for (size_t j = 0; j < x.order.size(); ++j) {
        const Block& b = S.blocks.at(x.order[j].second);
        double sv = 0;
        for (int r = 0; r < x.len[j]; ++r) sv += exp(-P.betabar * b.value[r]) * hd[k][p + r];
        row[x.order[j].first] += sym->mult(x.order[j].second) * sv;
        p += x.len[j];
      }
      for (auto& kv : row) kv.second /= Zs;
      expv_rows.push_back({x.T, row});
    }
    expv_def.clear();
  }

  // ---------------- transformation files ----------------
  // unitary<N>: "NRGBU001", int32 N, int32 nblocks, then per block int32 Q,
  // int32 SS, int32 dim, int32 0, the dim eigenvalues as returned by the
  // eigensolver (before the ground-state shift) and the dim x dim
  // eigenvectors (column-major, eigenvector r in column r); little endian.
  std::string workdir;
  int laststored = -1;
  std::string unitary_fn(int N) const { return workdir + "/unitary" + std::to_string(N); }
  void find_laststored() {
    // init_laststored (src/nrg.cc:3512-3524)
    laststored = -1;
    if (!P.resume) return;
    for (int N = Ninit; N < Nmax; ++N) {
      std::ifstream f(unitary_fn(N), std::ios::binary);
      if (f.good()) laststored = N;
    }
  }
  void store_transformations(int N, const Step& S) {
    std::vector<double> w, z;
    std::ofstream f(unitary_fn(N), std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + unitary_fn(N) + " for writing");
    const int32_t hdr[2] = {N, (int32_t)S.blocks.size()};
    f.write("NRGBU001", 8);
    f.write(reinterpret_cast<const char*>(hdr), sizeof(hdr));
    for (const auto& kv : S.blocks) {
      const Block& b = kv.second;
      w.resize(b.dim);
      z.resize((size_t)b.dim * b.dim);
      NRGB_CUDA(cudaMemcpyAsync(w.data(), b.w, b.dim * sizeof(double), cudaMemcpyDeviceToHost, st));
      NRGB_CUDA(cudaMemcpyAsync(z.data(), b.Z, z.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
      NRGB_CUDA(cudaStreamSynchronize(st));
      d2h += (w.size() + z.size()) * sizeof(double);
      const int32_t bh[4] = {kv.first.first, kv.first.second, b.dim, 0};
      f.write(reinterpret_cast<const char*>(bh), sizeof(bh));
      f.write(reinterpret_cast<const char*>(w.data()), w.size() * sizeof(double));
      f.write(reinterpret_cast<const char*>(z.data()), z.size() * sizeof(double));
    }
    if (!f) throw std::runtime_error("error writing " + unitary_fn(N));
  }
  void load_transformations(int N, Step& S) {
    std::ifstream f(unitary_fn(N), std::ios::binary);
    char magic[8];
    int32_t hdr[2];
    f.read(magic, 8);
    f.read(reinterpret_cast<char*>(hdr), sizeof(hdr));
    if (!f || memcmp(magic, "NRGBU001", 8) != 0 || hdr[0] != N)
      throw std::runtime_error("not a transformation file of step " + std::to_string(N) + ": " + unitary_fn(N));
    if (hdr[1] != (int32_t)S.blocks.size())
      throw std::runtime_error(unitary_fn(N) + ": subspaces differ from this run's");
    std::vector<double> w, z;
    for (auto& kv : S.blocks) {
      Block& b = kv.second;
      int32_t bh[4];
      f.read(reinterpret_cast<char*>(bh), sizeof(bh));
      if (!f || bh[0] != kv.first.first || bh[1] != kv.first.second || bh[2] != b.dim)
        throw std::runtime_error(unitary_fn(N) + ": subspaces differ from this run's");
      w.resize(b.dim);
      z.resize((size_t)b.dim * b.dim);
      f.read(reinterpret_cast<char*>(w.data()), w.size() * sizeof(double));
      f.read(reinterpret_cast<char*>(z.data()), z.size() * sizeof(double));
      if (!f) throw std::runtime_error("error reading " + unitary_fn(N));
      // pageable sources: the copies complete before the calls return
      NRGB_CUDA(cudaMemcpy(b.w, w.data(), w.size() * sizeof(double), cudaMemcpyHostToDevice));
      NRGB_CUDA(cudaMemcpy(b.Z, z.data(), z.size() * sizeof(double), cudaMemcpyHostToDevice));
      h2d += (w.size() + z.size()) * sizeof(double);
    }
  }

  // ---------------- sweep 1 ----------------
  void sweep1(Slab& persist) {
    std::map<Invar, Prev> prev;
    std::map<Invar, std::vector<double>> prev_host;
    for (const auto& kv : D.energies) {
      double* w = persist.alloc(kv.second.size());
      NRGB_CUDA(cudaMemcpyAsync(w, kv.second.data(), kv.second.size() * sizeof(double), cudaMemcpyHostToDevice, st));
      h2d += kv.second.size() * sizeof(double);
      prev[kv.first] = Prev{w, (int)kv.second.size()};
    }
    auto f_slab = std::make_unique<Slab>(st);
    std::vector<DevBlocks> opch;
    for (const auto& b : D.opch) opch.push_back(upload_blocks(b, *f_slab));
    auto s_slab = std::make_unique<Slab>(st);
    std::map<std::string, DevBlocks> singlets;
    if (D.ops.count('s'))
      for (const auto& kv : D.ops.at('s')) singlets[kv.first] = upload_blocks(kv.second, *s_slab);
    totalenergy = D.gs_energy;
    if (P.calc0) calc0();
    Slab hslab(st);
    size_t hcap = 0;
    double* H = nullptr;
    for (int N = Ninit; N < Nmax; ++N) {
      auto ts = Clock::now();
      const double scale1 = scale_of(P, N + 1);
      desc_reset();
      // subspaces of the new step and their ancestors
      std::set<Invar> subs;
      for (const auto& kv : prev)
        if (kv.second.kept > 0)
          for (const Invar& d : sym->In()) {
            const Invar J = Symmetry::combine(Symmetry::inverse(d), kv.first);
            if (sym->allowed(J)) subs.insert(J);
          }
      steps.emplace_back();
      Step& S = steps.back();
      S.scale = scale1;
      S.slab.reset(new Slab(st));
      size_t htot = 0;
      for (const Invar& I : subs) {
        Block b;
        int off = 0;
        for (int i = 0; i < sym->combs(); ++i) {
          const Invar anc = Symmetry::combine(sym->In()[i], I);
          auto it = prev.find(anc);
          const int r = (sym->triangle(I, anc, sym->QN()[i]) && it != prev.end()) ? it->second.kept : 0;
          b.anc.push_back(anc);
          b.rmax.push_back(r);
          b.off.push_back(off);
          off += r;
        }
        b.dim = off;
        if (b.dim == 0) continue;
        htot += (size_t)b.dim * b.dim;
        S.blocks[I] = std::move(b);
      }
      // device buffers: H (transient), Z and w (persistent for DM / sweep 2)
      if (htot > hcap) {
        hslab.release();
        hcap = htot + htot / 4;
        H = hslab.alloc(hcap);
      }
      NRGB_CUDA(cudaMemsetAsync(H, 0, htot * sizeof(double), st));
      std::vector<AsmDiag> ad;
      std::vector<AsmOff> ao;
      std::vector<SyevDesc> sd;
      size_t hoff = 0;
      size_t wtot = 0, woff = 0;
      for (const auto& kv : S.blocks) wtot += kv.second.dim;
      double* wall = S.slab->alloc(wtot);
      int maxlen = 0, maxrc = 0;
      for (auto& kv : S.blocks) {
        const Invar& I = kv.first;
        Block& b = kv.second;
        double* Hb = H + hoff;
        hoff += (size_t)b.dim * b.dim;
        b.Z = S.slab->alloc((size_t)b.dim * b.dim);
        b.w = wall + woff;  // the eigenvalues of a step are contiguous: one copy each way
        woff += b.dim;
        for (int i = 0; i < sym->combs(); ++i) {
          if (!b.rmax[i]) continue;
          double shift = 0.0;
          for (const DiagTerm& dt : sym->diag())
            if (dt.i - 1 == i) shift += D.zeta[dt.ch][N + 1] * (dt.number - 1.0) / scale1;
          ad.push_back(AsmDiag{Hb, prev[b.anc[i]].w, b.dim, b.off[i], b.rmax[i], sqrt(P.Lambda), shift});
          maxlen = std::max(maxlen, b.rmax[i]);
        }
        for (const OffdiagTerm& t : sym->offdiag(I)) {
          const int i0 = t.i - 1, j0 = t.j - 1;
          if (!(b.rmax[i0] > 0 && b.rmax[j0] > 0)) continue;
          // coefficient of the term: hopping xi_N, anomalous hopping kappa_N,
          // or the new site's pairing 2 delta_N+1 (src/sym-SPSU2.cc:107-113)
          const double coef = t.kind == 0 ? D.xi[t.ch][N]
                              : t.kind == 1 ? D.chain_coef(D.kappa, t.ch, N)
                                            : 2.0 * D.chain_coef(D.delta, t.ch, N + 1);
          const double fs = t.factor * coef / scale1;
          if (!std::isfinite(fs)) throw std::runtime_error("offdiag_function: factor is not finite");
          if (fabs(fs) < 1e-8) continue;
          if (t.kind == 2) {
            // identity between two combinations of the same ancestor
            // (diag_offdiag_function, src/matrix.cc:256-276)
            if (b.anc[i0] != b.anc[j0] || b.rmax[i0] != b.rmax[j0])
              throw std::runtime_error("diag_offdiag_function: combinations of different ancestors");
            ao.push_back(AsmOff{Hb, nullptr, b.dim, b.off[i0], b.off[j0], b.rmax[i0], b.rmax[j0], 1, fs});
            maxrc = std::max(maxrc, b.rmax[i0] * b.rmax[j0]);
            continue;
          }
          auto it = opch[t.ch].find({b.anc[i0], b.anc[j0]});
          if (it == opch[t.ch].end()) throw std::runtime_error("offdiag_function: <||f||> subspace does not exist");
          const DevMat& M = it->second;
          if (M.rows != b.rmax[i0] || M.cols != b.rmax[j0]) throw std::runtime_error("offdiag: block size mismatch");
          ao.push_back(AsmOff{Hb, M.p, b.dim, b.off[i0], b.off[j0], b.rmax[i0], b.rmax[j0], M.ld, fs});
          maxrc = std::max(maxrc, b.rmax[i0] * b.rmax[j0]);
        }
        sd.push_back(SyevDesc{b.dim, Hb, b.w, b.Z});
      }
      sections["sweep1 setup"] += secs(ts);
      auto t0 = Clock::now();
      if (P.resume && N <= laststored) {
        // the step's eigen-decompositions from the previous run's file
        // (nrg_do_diag, src/nrg.cc:2891-2895)
        NRGB_CUDA(cudaStreamSynchronize(st));
        load_transformations(N, S);
      } else {
        const auto layers = asm_off_layers(ao);
        NRGB_CUDA(assemble_launch(upload(ad), (int)ad.size(), layers.empty() ? nullptr : upload(layers[0]),
                                  layers.empty() ? 0 : (int)layers[0].size(), maxlen, maxrc, st));
        for (size_t k = 1; k < layers.size(); ++k)
          NRGB_CUDA(assemble_launch(nullptr, 0, upload(layers[k]), (int)layers[k].size(), 0, maxrc, st));
        launches += 1 + (int)std::max<size_t>(1, layers.size());
        launches += syev->solve(sd, st);
        eig_calls += 1;
        if (!P.removefiles) store_transformations(N, S);
      }
      t_diag += secs(t0);
      sections["sweep1 diag"] += secs(t0);
      ts = Clock::now();
      // truncation on the device: ground state, splitting correction,
      // retained states, thermodynamics sums; one small record comes back
      {
        const int nb = (int)S.blocks.size();
        std::vector<TruncBlock> tb;
        int o = 0;
        for (const auto& kv : S.blocks) {
          tb.push_back(TruncBlock{kv.second.w, kv.second.dim, o});
          o += kv.second.dim;
        }
        ensure_map(tstate.map_count + 2 * (int)wtot + 16);
        const size_t wb = trunc_work_bytes((int)wtot, nb);
        if (wb > twork_bytes) {
          if (twork) NRGB_CUDA(cudaFreeAsync(twork, st));
          twork_bytes = wb + wb / 2;
          NRGB_CUDA(cudaMallocAsync(&twork, twork_bytes, st));
        }
        const size_t tbytes = trunc_tail_bytes(nb);
        if (tbytes > tail_dev_bytes) {
          if (tail_dev) NRGB_CUDA(cudaFreeAsync(tail_dev, st));
          tail_dev_bytes = tbytes + tbytes / 2;
          NRGB_CUDA(cudaMallocAsync(&tail_dev, tail_dev_bytes, st));
        }
        if (tbytes > tail_pin_bytes) {
          NRGB_CUDA(cudaStreamSynchronize(st));
          if (tail_pin) NRGB_CUDA(cudaFreeHost(tail_pin));
          tail_pin_bytes = tbytes + tbytes / 2;
          NRGB_CUDA(cudaMallocHost(&tail_pin, tail_pin_bytes));
        }
        TruncRules R{P.fixeps, P.keepenergy, P.keep, P.keepmin, P.safeguard, P.safeguardmax,
                     (cfs_flags() && last(N) && !P.lastalloverride) ? 1 : 0, P.betabar};
        NRGB_CUDA(truncate_step(upload(tb), nb, wall, (int)wtot, R, tstate, twork, tail_dev, st));
        launches += 17;
        NRGB_CUDA(cudaMemcpyAsync(tail_pin, tail_dev, tbytes, cudaMemcpyDeviceToHost, st));
        NRGB_CUDA(cudaStreamSynchronize(st));
        d2h += tbytes;
        const TruncTail& T = *reinterpret_cast<const TruncTail*>(tail_pin);
        if (T.flags & 1) throw std::runtime_error("truncation: ground state not at zero");
        if (T.flags & 2)
          throw std::runtime_error("truncation: eigenvalues of a block not ascending after the splitting correction");
        tstate.map_count = T.map_count;
        const int* kept = trunc_tail_kept(tail_pin);
        const double Egs = T.Egs;
        S.Egs = Egs;
        size_t b = 0;
        for (auto& kv : S.blocks) {
          kv.second.kept = kept[b++];
          kv.second.shift = Egs;
        }
        if (getenv("NRGB_LOG")) {
          // the reference's per-step log line (src/nrg.cc:3010-3013), to stderr
          size_t nk = 0, na = 0;
          for (const auto& kv : S.blocks) {
            nk += kv.second.kept;
            na += kv.second.dim;
          }
          fprintf(stderr, "N=%d Egs=%.17g Kept: %zu out of %zu\n", N, Egs, nk, na);
        }
        totalenergy += Egs * scale1;
        S.total = totalenergy;
        S.wall = wall;
        S.wtot = (int)wtot;
        td_rows.push_back(td_sums(S, N, trunc_tail_sums(tail_pin, nb)));
      }
      sections["sweep1 truncate+td"] += secs(ts);
      // operator recalculation
      t0 = Clock::now();
      auto f_new = std::make_unique<Slab>(st);
      std::vector<DevBlocks> opch_new;
      if (!last(N)) opch_new = recalc_f(S, *f_new);
      auto s_new = std::make_unique<Slab>(st);
      std::map<std::string, DevBlocks> singlets_new;
      for (const auto& kv : singlets) singlets_new[kv.first] = recalc_op('s', S, kv.second, false, *s_new);
      // expectation values of singlet operators (nrg_measure_singlet,
      // src/nrg.cc:2226-2236): the diagonals are gathered now, the sums
      // are taken when the eigenvalues come to the host after the sweep
      {
        ExpvDeferred x;
        x.step = steps.size() - 1;
        x.T = scale1 / P.betabar;
        if (!singlets_new.empty()) {
          std::vector<DiagGather> dg;
          int off = 0, maxl = 0;
          for (const auto& op : singlets_new)
            for (const auto& kv : S.blocks) {
              const DevMat& M = op.second.at({kv.first, kv.first});
              dg.push_back(DiagGather{M.p, M.ld, M.rows, off});
              x.order.push_back({op.first, kv.first});
              x.len.push_back(M.rows);
              off += M.rows;
              maxl = std::max(maxl, M.rows);
            }
          double* buf = expv_slab->alloc(off + 1);
          NRGB_CUDA(gather_diag_launch(upload(dg), (int)dg.size(), maxl, buf, st));
          launches += 1;
          x.diag = buf;
        }
        expv_def.push_back(std::move(x));
      }
      t_recalc += secs(t0);
      sections["sweep1 recalc"] += secs(t0);
      // the new <f> and singlets replace the old ones; truncated values become prev
      opch = std::move(opch_new);
      f_slab = std::move(f_new);
      singlets = std::move(singlets_new);
      s_slab = std::move(s_new);
      prev.clear();
      for (const auto& kv : S.blocks) prev[kv.first] = Prev{kv.second.w, kv.second.kept};
    }
    finish_sweep1();
    GSenergy = totalenergy;
  }

  // ---------------- density matrices ----------------
  std::map<int, DevBlocks> rho, rhofdm;
  std::vector<double> ZnD, wn, wnfactor;
  std::vector<std::unique_ptr<Slab>> rho_slabs;

  DevMat diag_matrix(const std::vector<double>& d, Slab& slab) {
    DevMat M;
    M.rows = M.cols = (int)d.size();
    M.ld = std::max(1, M.rows);
    M.p = slab.alloc(d.size() * d.size());
    if (!M.p) return M;
    NRGB_CUDA(cudaMemsetAsync(M.p, 0, d.size() * d.size() * sizeof(double), st));
    double* v = slab.alloc(d.size());
    NRGB_CUDA(cudaMemcpyAsync(v, d.data(), d.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    h2d += d.size() * sizeof(double);
    std::vector<AsmDiag> a = {AsmDiag{M.p, v, M.rows, 0, M.rows, 1.0, 0.0}};
    NRGB_CUDA(assemble_launch(upload(a), 1, nullptr, 0, M.rows, 0, st));
    launches += 1;
    return M;
  }

  double trace_of(const DevBlocks& r) {
    std::vector<DiagGather> dg;
    int off = 0, maxl = 0;
    std::vector<int> mult;
    for (const auto& kv : r) {
      if (!kv.second.p) continue;
      dg.push_back(DiagGather{kv.second.p, kv.second.ld, kv.second.rows, off});
      mult.push_back(sym->mult(kv.first.first));
      off += kv.second.rows;
      maxl = std::max(maxl, kv.second.rows);
    }
    if (!off) return 0.0;
    Slab tmp(st);
    double* buf = tmp.alloc(off);
    NRGB_CUDA(gather_diag_launch(upload(dg), (int)dg.size(), maxl, buf, st));
    launches += 1;
    const std::vector<double> v = download(buf, off);
    double tr = 0;
    size_t p = 0;
    for (size_t k = 0; k < dg.size(); ++k) {
      double s = 0;
      for (int i = 0; i < dg[k].len; ++i) s += v[p + i];
      tr += mult[k] * s;
      p += dg[k].len;
    }
    return tr;
  }

  // rho_{N-1}[I] = sum_i coef_i Zsub (rhoKK + rhoDD) Zsub^T  (cdmI, src/dmnrg.h:327-388)
  DevBlocks backward_step(int N, const DevBlocks& rhoN, const std::map<Invar, std::vector<double>>* dd,
                          Slab& slab) {
    const Step& SN = steps[N - Ninit];
    const Step& Sp = steps[N - 1 - Ninit];
    DevBlocks out;
    Grouped g1, g2;
    Slab tmp(st);
    std::vector<ColScale> cs;
    int maxr = 0, maxc = 0;
    for (const auto& kv : Sp.blocks) {
      const Invar& I = kv.first;
      const int dim = kv.second.kept;
      DevMat C;
      C.rows = C.cols = dim;
      C.ld = std::max(1, dim);
      C.p = slab.alloc((size_t)dim * dim);
      out[{I, I}] = C;
      if (!dim) continue;
      std::vector<GemmSeg> ss;
      for (int i = 0; i < sym->combs(); ++i) {
        const Invar child = Symmetry::combine(Symmetry::inverse(sym->In()[i]), I);
        auto bi = SN.blocks.find(child);
        if (bi == SN.blocks.end()) continue;
        const Block& Bc = bi->second;
        const int rm = Bc.rmax[i];
        if (rm == 0) continue;
        if (rm != dim) throw std::runtime_error("cdmI: range mismatch");
        const double coef = double(sym->mult(child)) / double(sym->mult(I));
        const double* Zs = Bc.Z + Bc.off[i];  // dim x nomega sub-block, ld Bc.dim
        auto ri = rhoN.find({child, child});
        if (ri != rhoN.end() && ri->second.rows > 0) {
          const int nom = ri->second.rows;
          double* T = tmp.alloc((size_t)dim * nom);
          g1.out(T, dim, dim, nom, 0.0, {seg(Zs, Bc.dim, 0, ri->second.p, ri->second.ld, 0, nom, 1.0)});
          ss.push_back(seg(T, dim, 0, Zs, Bc.dim, 1, nom, coef));
        }
        if (dd) {
          auto di = dd->find(child);
          if (di != dd->end()) {
            const int lo = Bc.kept, hi = Bc.dim;
            if (hi > lo) {
              double* T = tmp.alloc((size_t)dim * (hi - lo));
              double* s = tmp.alloc(hi - lo);
              NRGB_CUDA(cudaMemcpyAsync(s, di->second.data() + lo, (hi - lo) * sizeof(double), cudaMemcpyHostToDevice, st));
              h2d += (hi - lo) * sizeof(double);
              cs.push_back(ColScale{Zs + (size_t)lo * Bc.dim, T, s, dim, hi - lo, Bc.dim, dim});
              maxr = std::max(maxr, dim);
              maxc = std::max(maxc, hi - lo);
              ss.push_back(seg(T, dim, 0, Zs + (size_t)lo * Bc.dim, Bc.dim, 1, hi - lo, coef));
            }
          }
        }
      }
      if (ss.empty())
        NRGB_CUDA(cudaMemsetAsync(C.p, 0, (size_t)dim * dim * sizeof(double), st));
      else
        g2.out(C.p, C.ld, dim, dim, 0.0, ss);
    }
    if (!cs.empty()) {
      NRGB_CUDA(col_scale_launch(upload(cs), (int)cs.size(), maxr, maxc, st));
      launches += 1;
    }
    run_gemm(g1);
    run_gemm(g2);
    NRGB_CUDA(cudaStreamSynchronize(st));
    return out;
  }

  void calc_densitymatrix() {
    const Step& L = steps.back();
    const double scale = scale_of(P, Nmax);
    double ZZ = 0;
    for (const auto& kv : L.blocks)
      for (int r = 0; r < kv.second.kept; ++r) ZZ += sym->mult(kv.first) * exp(-kv.second.value[r] * scale / P.T);
    rho_slabs.emplace_back(new Slab(st));
    DevBlocks r0;
    for (const auto& kv : L.blocks) {
      std::vector<double> d(kv.second.kept);
      for (int r = 0; r < kv.second.kept; ++r) d[r] = exp(-kv.second.value[r] * scale / P.T) / ZZ;
      r0[{kv.first, kv.first}] = diag_matrix(d, *rho_slabs.back());
    }
    rho[Nmax - 1] = r0;
    if (fabs(trace_of(r0) - 1.0) > 1e-8) throw std::runtime_error("init_rho: trace != 1");
    for (int N = Nmax - 1; N > Ninit; --N) {
      desc_reset();
      rho_slabs.emplace_back(new Slab(st));
      rho[N - 1] = backward_step(N, rho[N], nullptr, *rho_slabs.back());
      const double tr = trace_of(rho[N - 1]);
      if (fabs(tr - 1.0) > 1e-10) throw std::runtime_error("check_trace_rho() failed: " + std::to_string(tr));
    }
  }

  void calc_ZnD() {
    ZnD.assign(Nmax, 0.0);
    for (int N = Ninit; N < Nmax; ++N) {
      long double Z = 0;
      for (const auto& kv : steps[N - Ninit].blocks) {
        const int lo = last(N) ? 0 : kv.second.kept;
        for (int i = lo; i < kv.second.dim; ++i) {
          const long double Eabs = kv.second.absE[i] - GSenergy;
          Z += sym->mult(kv.first) * expl(-Eabs / P.T);
        }
      }
      ZnD[N] = (double)Z;
    }
    double Zt = 0;
    const int combs = sym->combs();
    for (int N = Ninit; N < Nmax; ++N) Zt += pow(double(combs), Nmax - N - 1) * ZnD[N];
    wn.assign(Nmax, 0.0);
    wnfactor.assign(Nmax, 0.0);
    double sw = 0;
    for (int N = Ninit; N < Nmax; ++N) {
      wn[N] = pow(double(combs), Nmax - N - 1) * ZnD[N] / Zt;
      sw += wn[N];
      const double w = wn[N] / ZnD[N];
      wnfactor[N] = std::isnan(w) ? 0.0 : w;
    }
    if (fabs(sw - 1.0) > 1e-12) throw std::runtime_error("sum of w_n != 1");
  }

  std::map<Invar, std::vector<double>> rho_fdm_diag(int N) {
    std::map<Invar, std::vector<double>> out;
    for (const auto& kv : steps[N - Ninit].blocks) {
      std::vector<double> d(kv.second.dim, 0.0);
      const int lo = last(N) ? 0 : kv.second.kept;
      for (int i = lo; i < kv.second.dim; ++i) {
        const long double Eabs = kv.second.absE[i] - GSenergy;
        long double v = expl(-Eabs / P.T) * ((long double)wn[N] / ZnD[N]);
        d[i] = std::isfinite((double)v) ? (double)v : 0.0;
      }
      out[kv.first] = d;
    }
    return out;
  }

  void calc_fulldensitymatrix() {
    rho_slabs.emplace_back(new Slab(st));
    DevBlocks r0;
    for (const auto& kv : rho_fdm_diag(Nmax - 1)) r0[{kv.first, kv.first}] = diag_matrix(kv.second, *rho_slabs.back());
    rhofdm[Nmax - 1] = r0;
    for (int N = Nmax - 1; N > Ninit; --N) {
      desc_reset();
      rho_slabs.emplace_back(new Slab(st));
      std::map<Invar, std::vector<double>> dd;
      if (!last(N)) dd = rho_fdm_diag(N);
      rhofdm[N - 1] = backward_step(N, rhofdm[N], last(N) ? nullptr : &dd, *rho_slabs.back());
      double expected = 0;
      for (int n = Nmax - 1; n >= N; --n) expected += wn[n];
      const double tr = trace_of(rhofdm[N - 1]);
      if (fabs((tr - expected) / expected) > 1e-10) throw std::runtime_error("FDM trace check failed");
    }
  }

  // ---------------- spectra ----------------
  struct Spec {
    std::string name, prefix, type;  // type DMNRG or FDM
    char kind;                       // 'd' doublet (fermionic) or 't' triplet (bosonic)
    std::string op1, op2;
    int spin = 0;                    // +1 / -1: spin-resolved (symmetries with a field), 0: all pairs
    double* full = nullptr;          // device [pos | neg]
    double* chain = nullptr;
  };
  std::vector<Spec> spectra;
  BinGrid grid{};
  std::vector<double> bin_e;
  double* bin_e_dev = nullptr;

  void setup_bins() {
    const double emax = P.emax > 0 ? P.emax : scale_of(P, 0) * pow(10.0, 2.0);
    const double emin = P.emin > 0 ? P.emin : scale_of(P, Nmax) / pow(10.0, 2.0);
    const double l0 = floor(log10(emin)), l1 = ceil(log10(emax));
    grid.l0 = l0;
    grid.bpd = P.bins;
    grid.nbins = (int)((l1 - l0) * P.bins + 1.0);
    grid.discard = P.discard_immediately;
    bin_e.resize(grid.nbins);
    for (int i = 0; i < grid.nbins; ++i) bin_e[i] = pow(10.0, l0 + (double)i / P.bins);
  }

  void sweep2(Slab& persist) {
    setup_bins();
    auto add_spectra = [&](const std::string& list, char kind, const std::string& prefix) {
      std::istringstream is(list);
      std::string pair;
      while (is >> pair) {
        const auto dash = pair.find('-');
        if (dash == std::string::npos) continue;
        const std::string a = pair.substr(0, dash), b = pair.substr(dash + 1);
        if (!D.ops.count(kind) || !D.ops.at(kind).count(a) || !D.ops.at(kind).count(b)) continue;
        // spin-resolved spectra for the symmetries with a field: names get
        // "-u" / "-d" (SDNAME, src/nrg.cc:1498-1505)
        std::vector<int> spins = {0};
        if (kind == 'd' && sym->isfield()) spins = {-1, 1};
        for (int spin : spins)
          for (const char* type : {"DMNRG", "FDM"}) {
            if (std::string(type) == "DMNRG" && !P.dmnrg) continue;
            if (std::string(type) == "FDM" && !P.fdm) continue;
            Spec s{pair + (spin == 1 ? "-u" : spin == -1 ? "-d" : ""), prefix, type, kind, a, b};
            s.spin = spin;
            s.full = persist.alloc(2 * grid.nbins);
            s.chain = persist.alloc(2 * grid.nbins);
            NRGB_CUDA(cudaMemsetAsync(s.full, 0, 2 * grid.nbins * sizeof(double), st));
            spectra.push_back(s);
          }
      }
    };
    bin_e_dev = persist.alloc(grid.nbins);
    NRGB_CUDA(cudaMemcpyAsync(bin_e_dev, bin_e.data(), grid.nbins * sizeof(double), cudaMemcpyHostToDevice, st));
    add_spectra(P.specd, 'd', "spec");
    add_spectra(P.spect, 't', "spin");
    std::set<std::pair<char, std::string>> needed;
    for (const Spec& s : spectra) {
      needed.insert({s.kind, s.op1});
      needed.insert({s.kind, s.op2});
    }
    auto slab = std::make_unique<Slab>(st);
    std::map<std::pair<char, std::string>, DevBlocks> ops;
    for (const auto& k : needed) ops[k] = upload_blocks(D.ops.at(k.first).at(k.second), *slab);
    const bool recalc_all = cfs_flags();
    double te = D.gs_energy;
    Slab eslab(st);
    for (int N = Ninit; N < Nmax; ++N) {
      desc_reset();
      Step& S = steps[N - Ninit];
      const double scale = S.scale;
      // the truncation of sweep 1 is reused: the reference recomputes it from
      // the stored values with the same rules, which gives the same counts
      te += S.Egs * scale;
      auto t0 = Clock::now();
      auto nslab = std::make_unique<Slab>(st);
      std::map<std::pair<char, std::string>, DevBlocks> nops;
      for (auto& kv : ops) nops[kv.first] = recalc_op(kv.first.first, S, kv.second, recalc_all, *nslab);
      NRGB_CUDA(cudaStreamSynchronize(st));
      t_recalc += secs(t0);
      sections["sweep2 recalc"] += secs(t0);
      t0 = Clock::now();
      // absolute energies shifted by the absolute ground state (FDM), and
      // their Boltzmann factors exp(-E/T) once per state, not per matrix
      // element of the spectral sums
      std::map<Invar, double*> absdev, boltzdev;
      if (P.fdm) {
        wstage.clear();
        for (const auto& kv : S.blocks)
          for (int r = 0; r < kv.second.dim; ++r) wstage.push_back(kv.second.absE[r] - GSenergy);
        const size_t ns = wstage.size();
        for (size_t r = 0; r < ns; ++r) wstage.push_back(exp(-wstage[r] / P.T));
        double* d = nslab->alloc(wstage.size());
        NRGB_CUDA(cudaMemcpyAsync(d, wstage.data(), wstage.size() * sizeof(double), cudaMemcpyHostToDevice, st));
        h2d += wstage.size() * sizeof(double);
        for (const auto& kv : S.blocks) {
          absdev[kv.first] = d;
          boltzdev[kv.first] = d + ns;
          d += kv.second.dim;
        }
      }
      for (Spec& sp : spectra) {
        NRGB_CUDA(cudaMemsetAsync(sp.chain, 0, 2 * grid.nbins * sizeof(double), st));
        const DevBlocks& o1 = nops.at({sp.kind, sp.op1});
        const DevBlocks& o2 = nops.at({sp.kind, sp.op2});
        const double msign = sp.kind == 'd' ? 1.0 : -1.0;  // -sign: fermionic +1, bosonic -1
        Grouped g;
        Slab tmp(st);
        if (sp.type == "DMNRG") {
          const DevBlocks& R = rho.at(N);
          std::vector<SpecDmnrgPair> pr;
          int maxe = 0;
          for (const auto& bi : S.blocks)
            for (const auto& bj : S.blocks) {
              const Twoinvar II{bj.first, bi.first};
              auto a1 = o1.find(II), a2 = o2.find(II);
              if (a1 == o1.end() || a2 == o2.end()) continue;
              if (sp.spin != 0 && !sym->check_spin(bj.first, bi.first, sp.spin)) continue;
              const double sf = sp.kind == 'd' ? sym->specdens_factor(bi.first, bj.first)
                                               : sym->dynsusc_factor(bi.first, bj.first);
              auto rp = R.find({bi.first, bi.first}), r1 = R.find({bj.first, bj.first});
              const int dimp = rp == R.end() ? 0 : rp->second.rows;
              const int dim1 = r1 == R.end() ? 0 : r1->second.rows;
              if (!dimp || !dim1) continue;
              double* SA = tmp.alloc((size_t)dim1 * dimp);
              double* SB = tmp.alloc((size_t)dim1 * dimp);
              g.out(SA, dim1, dim1, dimp, 0.0, {seg(a2->second.p, a2->second.ld, 0, rp->second.p, rp->second.ld, 0, dimp, 1.0)});
              g.out(SB, dim1, dim1, dimp, 0.0, {seg(r1->second.p, r1->second.ld, 0, a1->second.p, a1->second.ld, 0, dim1, 1.0)});
              if (a1->second.ld != a2->second.ld) throw std::runtime_error("spectrum: operator layouts differ");
              pr.push_back(SpecDmnrgPair{a1->second.p, a2->second.p, SA, SB, bj.second.w, bi.second.w,
                                         a1->second.ld, dim1, dimp, sf});
              maxe = std::max(maxe, dim1 * dimp);
            }
          run_gemm(g);
          const double fac = (P.channels == 1 && !P.NN1) ? P.Lambda : sqrt(P.Lambda);
          NRGB_CUDA(spec_dmnrg_launch(upload(pr), (int)pr.size(), maxe, grid, scale, P.goodE,
                                      P.goodE * fac * fac, msign, sp.chain, st));
          launches += 1;
          const bool merge = P.NN1 || P.NN2avg || (P.NN2even ? (N % 2 == 0) : (N % 2 == 1));
          if (merge) {
            NRGB_CUDA(merge_bins_launch(sp.chain, sp.full, bin_e_dev, grid, 1, scale * P.goodE, scale * P.goodE * fac,
                                        scale * P.goodE * fac * fac, P.NNtanh, P.NN2avg ? 0.5 : 1.0,
                                        N == Ninit, last(N), st));
            launches += 1;
          }
        } else {
          const DevBlocks& R = rhofdm.at(N);
          std::vector<SpecFdmPair> pr;
          int maxe = 0;
          for (const auto& bi : S.blocks)
            for (const auto& bj : S.blocks) {
              const Twoinvar II{bj.first, bi.first};
              auto a1 = o1.find(II), a2 = o2.find(II);
              if (a1 == o1.end() || a2 == o2.end()) continue;
              if (sp.spin != 0 && !sym->check_spin(bj.first, bi.first, sp.spin)) continue;
              const double sf = sp.kind == 'd' ? sym->specdens_factor(bi.first, bj.first)
                                               : sym->dynsusc_factor(bi.first, bj.first);
              auto ri = R.find({bi.first, bi.first}), rj = R.find({bj.first, bj.first});
              const int reti = last(N) ? 0 : (ri == R.end() ? 0 : ri->second.rows);
              const int retj = last(N) ? 0 : (rj == R.end() ? 0 : rj->second.rows);
              const int alli = a1->second.cols, allj = a1->second.rows;
              if (!alli || !allj) continue;
              double* O2R = nullptr;
              double* RO2 = nullptr;
              if (allj > 0 && reti > 0) {
                O2R = tmp.alloc((size_t)allj * reti);
                g.out(O2R, allj, allj, reti, 0.0, {seg(a2->second.p, a2->second.ld, 0, ri->second.p, ri->second.ld, 0, reti, 1.0)});
              }
              if (retj > 0 && alli > 0) {
                RO2 = tmp.alloc((size_t)retj * alli);
                g.out(RO2, retj, retj, alli, 0.0, {seg(rj->second.p, rj->second.ld, 0, a2->second.p, a2->second.ld, 0, retj, 1.0)});
              }
              pr.push_back(SpecFdmPair{a1->second.p, a2->second.p, O2R, RO2, absdev.at(bj.first),
                                       absdev.at(bi.first), boltzdev.at(bj.first), boltzdev.at(bi.first),
                                       a1->second.ld, allj, alli, retj, reti, sf});
              maxe = std::max(maxe, allj * alli);
            }
          run_gemm(g);
          NRGB_CUDA(spec_fdm_launch(upload(pr), (int)pr.size(), maxe, grid, P.T, wnfactor[N], msign, sp.chain, st));
          NRGB_CUDA(merge_bins_launch(sp.chain, sp.full, bin_e_dev, grid, 0, 0, 0, 0, 0, 1.0, 0, 0, st));
          launches += 2;
        }
        NRGB_CUDA(cudaStreamSynchronize(st));
      }
      t_spec += secs(t0);
      sections["sweep2 spec"] += secs(t0);
      // operators for the next step: the kept states only (nrg_trim_matrices)
      for (auto& kv : nops)
        for (auto& m : kv.second) {
          const Block& b1 = S.blocks.at(m.first.first);
          const Block& bp = S.blocks.at(m.first.second);
          m.second = m.second.view(std::min(m.second.rows, b1.kept), std::min(m.second.cols, bp.kept));
        }
      ops = std::move(nops);
      slab = std::move(nslab);
    }
    if (fabs(te - GSenergy) > 1e-12 * std::max(1.0, fabs(te))) throw std::runtime_error("GSenergy != totalenergy");
  }

  // ---------------- outputs ----------------
  void write_td(const std::string& dir) {
    std::ofstream F(dir + "/td");
    std::vector<std::string> names = {"T"};
    for (const auto& n : sym->td_names()) names.push_back(n);
    for (const char* n : {"<E>", "<E^2>", "C", "F", "S"}) names.push_back(n);
    F << '#';
    for (const auto& n : names) F << std::setw(P.width_td) << n << ' ';
    F << '\n';
    for (const auto& row : td_rows) {
      F << ' ';
      for (double v : row) F << std::setw(P.width_td) << fmt_g(v, P.prec_td) << ' ';
      F << '\n';
    }
  }
  void write_custom(const std::string& dir) {
    if (expv_rows.empty() || expv_rows[0].second.empty()) return;
    std::ofstream F(dir + "/custom");
    std::vector<std::string> names;
    for (const auto& kv : expv_rows[0].second) names.push_back(kv.first);
    auto fo = [&](const std::string& s) { F << std::setw(P.width_custom) << s << ' '; };
    F << '#';
    fo("1");
    for (size_t c = 1; c <= names.size(); ++c) fo(std::to_string(1 + c));
    F << "\n#";
    fo("T");
    for (const auto& n : names) fo(n);
    F << '\n';
    for (const auto& r : expv_rows) {
      F << ' ';
      fo(fmt_g(r.first, P.prec_custom));
      for (const auto& n : names) fo(fmt_g(r.second.at(n), P.prec_custom));
      F << '\n';
    }
  }
  void write_annotated(const std::string& dir) {
    if (!P.dumpannotated) return;
    std::ofstream F(dir + "/annotated.dat");
    F << std::setprecision(P.dumpprecision);
    // my_fcmp(x, y, eps) == 0 (src/numerics.h:37-53)
    auto fcmp = [&](double x, double y) {
      const double eps = P.grouptol;
      if (x == 0.0 && y == 0.0) return true;
      if (fabs(x) < eps && fabs(y) < eps) return true;
      return fabs(x - y) / (fabs(x) + fabs(y)) < eps;
    };
    for (const Annotated& a : annotated) {
      const auto& l = a.levels;
      size_t len = std::min(l.size(), (size_t)P.dumpannotated);
      for (size_t i = len; i + 1 < l.size() && i > 0; ++i) {
        if (fcmp(l[i].first, l[i - 1].first)) ++len; else break;
      }
      // scaled_energy (src/nrg.cc:2052-2056)
      auto en = [&](double e) { return e * (P.dumpscaled ? 1.0 : a.scale) + (P.dumpabs ? a.total : 0.0); };
      if (P.dumpgroups) {
        for (size_t i = 0; i < len;) {
          F << en(l[i].first);
          std::vector<std::string> qn;
          int deg = 0;
          const size_t i0 = i;
          while (i < len && fcmp(l[i].first, l[i0].first)) {
            qn.push_back(sym->label(l[i].second));
            deg += sym->mult(l[i].second);
            ++i;
          }
          std::sort(qn.begin(), qn.end());
          for (const auto& q : qn) F << " (" << q << ")";
          F << " [" << deg << "]\n";
        }
      } else {
        for (const auto& x : l) F << en(x.first) << " " << sym->label(x.second) << "\n";
      }
      F << "\n";
    }
  }
  void write_spectra(const std::string& dir) {
    for (const Spec& sp : spectra) {
      std::vector<double> h = download(sp.full, 2 * grid.nbins);
      auto trim = [&](int base, std::vector<double>& e, std::vector<double>& w) {
        for (int i = 0; i + 1 < grid.nbins; ++i) {
          const double ew = bin_e[i + 1] - bin_e[i];
          if (!(fabs(h[base + i]) < P.discard_trim * ew)) {
            e.push_back(bin_e[i]);
            w.push_back(h[base + i]);
          }
        }
        e.push_back(bin_e[grid.nbins - 1]);
        w.push_back(h[base + grid.nbins - 1]);
      };
      std::vector<double> ep, wp, en, wn_;
      trim(0, ep, wp);
      trim(grid.nbins, en, wn_);
      const std::string fn = dir + "/" + sp.prefix + "_" + sp.type + "_dens_" + sp.name;
      if (P.savebins) {
        std::ofstream B(fn + ".bin", std::ios::binary);
        for (size_t i = 0; i < ep.size(); ++i) {
          B.write((const char*)&ep[i], 8);
          B.write((const char*)&wp[i], 8);
        }
        for (size_t i = 0; i < en.size(); ++i) {
          const double e = -en[i];
          B.write((const char*)&e, 8);
          B.write((const char*)&wn_[i], 8);
        }
      }
      if (P.broaden) write_broadened(fn + ".dat", ep, wp, en, wn_);
    }
  }
  // SpectrumRealFreq::continuous with BR_NEW (src/spectrumrealfreq.cc:271-306,
  // src/spectral.h:70-102): log-Gaussian kernel, Gaussian below omega0,
  // evaluated on the device (broaden_kernel) for the mesh
  // E = broaden_max / broaden_ratio^k down to broaden_min (both signs).
  void write_broadened(const std::string& fn, const std::vector<double>& ep, const std::vector<double>& wp,
                       const std::vector<double>& en, const std::vector<double>& wn_) {
    const double alpha = P.alpha, gamma = alpha / 4.0;
    const double omega0 = P.omega0 < 0.0 ? P.omega0_ratio * P.T : P.omega0;
    const double bmin = P.broaden_min <= 0.0 ? P.broaden_min_ratio * scale_of(P, Nmax) : P.broaden_min;
    std::vector<double> mesh;
    for (double E = P.broaden_max; E > bmin; E /= P.broaden_ratio) mesh.push_back(E);
    std::vector<double> e(ep), w(wp);
    for (size_t i = 0; i < en.size(); ++i) {
      e.push_back(-en[i]);
      w.push_back(wn_[i]);
    }
    const int nmesh = (int)mesh.size(), nb = (int)e.size();
    std::vector<double> vals(2 * (size_t)nmesh, 0.0);
    if (nmesh > 0 && nb > 0) {
      Slab tmp(st);
      double* d_e = tmp.alloc(nb);
      double* d_w = tmp.alloc(nb);
      double* d_m = tmp.alloc(nmesh);
      double* d_o = tmp.alloc(2 * (size_t)nmesh);
      NRGB_CUDA(cudaMemcpyAsync(d_e, e.data(), nb * sizeof(double), cudaMemcpyHostToDevice, st));
      NRGB_CUDA(cudaMemcpyAsync(d_w, w.data(), nb * sizeof(double), cudaMemcpyHostToDevice, st));
      NRGB_CUDA(cudaMemcpyAsync(d_m, mesh.data(), nmesh * sizeof(double), cudaMemcpyHostToDevice, st));
      h2d += (2.0 * nb + nmesh) * sizeof(double);
      NRGB_CUDA(broaden_launch(d_e, d_w, nb, d_m, nmesh, alpha, gamma, omega0, d_o, st));
      launches += 1;
      vals = download(d_o, 2 * (size_t)nmesh);
    }
    std::vector<std::pair<double, double>> pos, neg;
    for (int k = 0; k < nmesh; ++k) {
      pos.push_back({mesh[k], vals[k]});
      neg.push_back({-mesh[k], vals[nmesh + k]});
    }
    std::sort(pos.begin(), pos.end());
    std::sort(neg.begin(), neg.end());
    std::ofstream F(fn);
    F << std::setprecision(P.prec_xy);
    for (const auto& x : neg) F << x.first << " " << x.second << "\n";
    for (const auto& x : pos) F << x.first << " " << x.second << "\n";
  }

  // Device data of a run: freed at its end, and on the way out of a failed run
  // so that a server can hand the memory to the next run.
  void release_run_data() {
    spectra.clear();
    rho.clear();
    rhofdm.clear();
    rho_slabs.clear();
    steps.clear();
  }

  void run(const std::string& wd, const std::string& od, double* stats, RunExtra* extra) {
    release_run_data();
    mem = MemCount();
    eig_calls = 0;
    struct MemScope {
      explicit MemScope(MemCount* m) { tl_mem = m; }
      ~MemScope() { tl_mem = nullptr; }
    } mem_scope(&mem);
    try {
      run_body(wd, od, stats);
    } catch (...) {
      release_run_data();
      cudaStreamSynchronize(st);
      throw;
    }
    if (extra) {
      extra->peak_bytes = (double)mem.peak;
      extra->eig_calls = eig_calls;
    }
  }

  void run_body(const std::string& wd, const std::string& od, double* stats) {
    const auto t0 = Clock::now();
    t_diag = t_recalc = t_dm = t_spec = 0;
    launches = h2d = d2h = 0;
    free_trunc();
    expv_def.clear();
    expv_slab.reset(new Slab(st));
    td_rows.clear();
    expv_rows.clear();
    annotated.clear();
    sections.clear();
    std::unique_ptr<Section> sec(new Section(this, "read input"));
    desc.reserve(64 << 20);
    desc.reset();
    if (!desc_pin) NRGB_CUDA(cudaMallocHost(&desc_pin, DESC_PINNED));
    P = Params();
    P.read(wd + "/param");
    D = DataFile();
    D.read(wd + "/data");
    P.channels = D.channels;
    if (D.symtype == "QS") {
      sym.reset(new SymmetryQS(D.channels));
    } else if (D.symtype == "QSZ") {
      if (D.channels < 1 || D.channels > 3) throw std::runtime_error("symmetry type QSZ: 1 to 3 channels are built");
      if (!P.spect.empty() || !P.specs.empty())
        throw std::runtime_error("symmetry type QSZ: only the spectral functions of doublet operators are built");
      sym.reset(new SymmetryQSZ(D.channels));
    } else if (D.symtype == "SPSU2") {
      if (D.channels < 1 || D.channels > 3) throw std::runtime_error("symmetry type SPSU2: 1 to 3 channels are built");
      sym.reset(new SymmetrySPSU2(D.channels));
    } else {
      throw std::runtime_error("symmetry type " + D.symtype + " is not built (QS, QSZ, SPSU2)");
    }
    if (P.Nmax == 0) P.Nmax = D.Nmax;
    if ((int)D.xi[0].size() - 1 != P.Nmax) throw std::runtime_error("length of coefficient table != Nmax");
    Nmax = P.Nmax;
    Ninit = P.Ninit;
    workdir = wd;
    find_laststored();
    if (Nmax <= Ninit) throw std::runtime_error("zero-bandwidth runs (Nmax == Ninit) are not supported");
    if (P.dm && P.T <= 0) throw std::runtime_error("density-matrix runs need T > 0");
    Slab persist(st);
    sec.reset();
    {
      struct Client {
        EigSolver* e;
        explicit Client(EigSolver* e_) : e(e_) { e->client_enter(); }
        ~Client() { e->client_leave(); }
      } client(syev);
      Section x(this, "sweep1 (all)");
      sweep1(persist);
    }
    if (P.dm) {
      auto t1 = Clock::now();
      if (P.dmnrg) {
        Section x(this, "DM");
        calc_densitymatrix();
      }
      if (P.fdm) {
        Section x(this, "FDM");
        calc_ZnD();
        calc_fulldensitymatrix();
      }
      t_dm += secs(t1);
      Section x(this, "sweep2 (all)");
      sweep2(persist);
    }
    if (P.gemm_slices > 0 && split_gemm_take_error(st))
      throw CudaError("split-precision products: a barrier wait timed out");
    sec.reset(new Section(this, "write output"));
    write_td(od);
    write_custom(od);
    write_annotated(od);
    write_spectra(od);
    NRGB_CUDA(cudaStreamSynchronize(st));
    sec.reset(new Section(this, "release"));
    release_run_data();
    NRGB_CUDA(cudaStreamSynchronize(st));
    sec.reset();
    if (getenv("NRGB_TIMING")) {
      const double all = secs(t0);
      double sum = 0;
      fprintf(stderr, "Timing report\n=============\n%20s: %.4f s\n", "All", all);
      for (const auto& kv : sections) {
        fprintf(stderr, "%20s: %.4f s\n", kv.first.c_str(), kv.second);
        if (kv.first.find("(all)") == std::string::npos) sum += kv.second;
      }
      fprintf(stderr, "%20s: %.4f s\n", "Other", all - sum);
    }
    if (stats) {
      stats[0] = secs(t0);
      stats[1] = t_diag;
      stats[2] = t_recalc;
      stats[3] = t_dm;
      stats[4] = t_spec;
      stats[5] = launches;
      stats[6] = h2d;
      stats[7] = d2h;
    }
  }
};

NrgDriver::NrgDriver(cudaStream_t stream, EigSolver* eig) : impl_(new Impl(stream, eig)) {}
NrgDriver::~NrgDriver() { delete impl_; }
void NrgDriver::run(const char* workdir, const char* outdir, double* stats, RunExtra* extra) {
  impl_->run(workdir, outdir, stats, extra);
}

}  // namespace nrgb
