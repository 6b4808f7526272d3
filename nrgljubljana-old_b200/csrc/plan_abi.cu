// Step-level C ABI: the reference keeps its own iteration driver
// (nrg_iterate, src/nrg.cc:3043-3051) and its Symmetry plug-ins
// (src/symmetry.cc:64-221, sym-<SYM>.cc, nrg-recalc-<SYM>.cc), expands their
// tables on the host into flat task lists, and the device executes one NRG
// step per call.  Run state (energies, eigenvectors, operator blocks) stays
// in device memory under integer handles between calls.
//
//   nrgb_step    assembly of every block (nrg_prepare_task_for_diag,
//                src/nrg.cc:2456-2478; offdiag_build / diag_function,
//                src/matrix.cc:86-192), eigen-decomposition of all blocks
//                (dsyev per block, src/diag.h:54-89), truncation (ground
//                state, splitting correction, retained states,
//                src/nrg.cc:1420-1455, 1919-1998, src/splitting.cc) and the
//                Boltzmann sums of the thermodynamics (src/nrg.cc:2333-2369)
//   nrgb_recalc  the recalculation of irreducible matrix elements
//                (recalc_f and recalc_general, src/recalc.cc:12-97,
//                164-281) as grouped FP64 tensor-core products
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/nrgb.h"
#include "ctx.h"
#include "gemm_f64.cuh"
#include "nrg_kernels.cuh"
#include "truncate.cuh"

namespace nrgb {

namespace {

PlanMatrix& mat(nrgb_ctx* ctx, int h) {
  if (h < 0 || h >= (int)ctx->plan.mats.size() || !ctx->plan.mats[h].p)
    throw CudaError("step plan: invalid matrix handle " + std::to_string(h));
  return ctx->plan.mats[h];
}

int new_mat(nrgb_ctx* ctx, int rows, int cols) {
  PlanState& S = ctx->plan;
  PlanMatrix m;
  m.rows = rows;
  m.cols = cols;
  const size_t bytes = std::max<size_t>(8, (size_t)rows * cols * sizeof(double));
  NRGB_CUDA(cudaMallocAsync((void**)&m.p, bytes, ctx->stream));
  int h;
  if (!S.free_slots.empty()) {
    h = S.free_slots.back();
    S.free_slots.pop_back();
    S.mats[h] = m;
  } else {
    h = (int)S.mats.size();
    S.mats.push_back(m);
  }
  return h;
}

void free_mat(nrgb_ctx* ctx, int h) {
  PlanMatrix& m = mat(ctx, h);
  NRGB_CUDA(cudaFreeAsync(m.p, ctx->stream));
  m = PlanMatrix{};
  ctx->plan.free_slots.push_back(h);
}

template <class T>
T* stage(nrgb_ctx* ctx, const std::vector<T>& v) {
  if (v.empty()) return nullptr;
  T* d = ctx->scratch.alloc_n<T>(v.size());
  NRGB_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream));
  return d;
}

void free_trunc(nrgb_ctx* ctx) {
  PlanState& S = ctx->plan;
  cudaStream_t st = ctx->stream;
  for (int i = 0; i < 2; ++i) {
    if (S.trunc.map_k[i]) cudaFreeAsync(S.trunc.map_k[i], st);
    if (S.trunc.map_v[i]) cudaFreeAsync(S.trunc.map_v[i], st);
  }
  if (S.trunc.d_count) cudaFreeAsync(S.trunc.d_count, st);
  S.trunc = TruncState();
}

void ensure_map(nrgb_ctx* ctx, int need) {
  TruncState& T = ctx->plan.trunc;
  cudaStream_t st = ctx->stream;
  if (need <= T.map_cap) return;
  int cap = std::max(4096, T.map_cap);
  while (cap < need) cap *= 2;
  double *nk[2], *nv[2];
  for (int i = 0; i < 2; ++i) {
    NRGB_CUDA(cudaMallocAsync((void**)&nk[i], sizeof(double) * cap, st));
    NRGB_CUDA(cudaMallocAsync((void**)&nv[i], sizeof(double) * cap, st));
  }
  if (!T.d_count) {
    NRGB_CUDA(cudaMallocAsync((void**)&T.d_count, sizeof(int), st));
    NRGB_CUDA(cudaMemsetAsync(T.d_count, 0, sizeof(int), st));
  }
  const int c = T.cur;
  if (T.map_count > 0) {
    NRGB_CUDA(cudaMemcpyAsync(nk[c], T.map_k[c], sizeof(double) * T.map_count, cudaMemcpyDeviceToDevice, st));
    NRGB_CUDA(cudaMemcpyAsync(nv[c], T.map_v[c], sizeof(double) * T.map_count, cudaMemcpyDeviceToDevice, st));
  }
  for (int i = 0; i < 2; ++i) {
    if (T.map_k[i]) cudaFreeAsync(T.map_k[i], st);
    if (T.map_v[i]) cudaFreeAsync(T.map_v[i], st);
    T.map_k[i] = nk[i];
    T.map_v[i] = nv[i];
  }
  T.map_cap = cap;
}

}  // namespace

void plan_release(nrgb_ctx* ctx) {
  PlanState& S = ctx->plan;
  for (auto& m : S.mats)
    if (m.p) cudaFreeAsync(m.p, ctx->stream);
  S.mats.clear();
  S.free_slots.clear();
  free_trunc(ctx);
  if (S.twork) cudaFreeAsync(S.twork, ctx->stream);
  if (S.tail_dev) cudaFreeAsync(S.tail_dev, ctx->stream);
  S.twork = S.tail_dev = nullptr;
  S.twork_bytes = S.tail_bytes = 0;
  cudaStreamSynchronize(ctx->stream);
  if (S.tail_pin) cudaFreeHost(S.tail_pin);
  S.tail_pin = nullptr;
  S.tail_pin_bytes = 0;
}

}  // namespace nrgb

using nrgb::guarded;

extern "C" {

int nrgb_mat_upload(nrgb_ctx* ctx, int rows, int cols, const double* host, int* handle) {
  if (rows < 0 || cols < 0 || !handle || (rows * (size_t)cols > 0 && !host)) return 1;
  return guarded(ctx, [&] {
    const int h = nrgb::new_mat(ctx, rows, cols);
    if ((size_t)rows * cols)
      NRGB_CUDA(cudaMemcpyAsync(ctx->plan.mats[h].p, host, (size_t)rows * cols * sizeof(double),
                                cudaMemcpyHostToDevice, ctx->stream));
    NRGB_CUDA(cudaStreamSynchronize(ctx->stream));
    *handle = h;
  });
}

int nrgb_mat_download(nrgb_ctx* ctx, int handle, double* host) {
  return guarded(ctx, [&] {
    const nrgb::PlanMatrix& m = nrgb::mat(ctx, handle);
    if ((size_t)m.rows * m.cols) {
      if (!host) throw nrgb::CudaError("nrgb_mat_download: null destination");
      NRGB_CUDA(cudaMemcpyAsync(host, m.p, (size_t)m.rows * m.cols * sizeof(double), cudaMemcpyDeviceToHost,
                                ctx->stream));
    }
    NRGB_CUDA(cudaStreamSynchronize(ctx->stream));
  });
}

int nrgb_mat_shape(nrgb_ctx* ctx, int handle, int* rows, int* cols) {
  return guarded(ctx, [&] {
    const nrgb::PlanMatrix& m = nrgb::mat(ctx, handle);
    if (rows) *rows = m.rows;
    if (cols) *cols = m.cols;
  });
}

int nrgb_mat_free(nrgb_ctx* ctx, int handle) {
  return guarded(ctx, [&] { nrgb::free_mat(ctx, handle); });
}

int nrgb_run_begin(nrgb_ctx* ctx) {
  return guarded(ctx, [&] { nrgb::plan_release(ctx); });
}

int nrgb_step(nrgb_ctx* ctx, const nrgb_step_plan* plan, int* z_handles, int* w_handles, int* kept,
              double* egs, double* zsums) {
  if (!plan || plan->nblocks <= 0 || !plan->dim || !z_handles || !w_handles || !kept || !egs) return 1;
  return guarded(ctx, [&] {
    using namespace nrgb;
    cudaStream_t st = ctx->stream;
    const int nb = plan->nblocks;
    std::vector<size_t> hoff(nb + 1, 0), woff(nb + 1, 0);
    for (int b = 0; b < nb; ++b) {
      if (plan->dim[b] <= 0) throw CudaError("nrgb_step: every block needs a positive dimension");
      hoff[b + 1] = hoff[b] + (size_t)plan->dim[b] * plan->dim[b];
      woff[b + 1] = woff[b] + plan->dim[b];
    }
    const size_t htot = hoff[nb], wtot = woff[nb];
    // scratch: H of every block, the step's eigenvalues back to back, descriptors
    const size_t desc = (size_t)(plan->ndiag + 1) * sizeof(AsmDiag) + (size_t)(plan->noff + 1) * sizeof(AsmOff) +
                        (size_t)nb * (sizeof(TruncBlock) + 64) + 4096;
    ctx->scratch.reserve(htot * sizeof(double) + wtot * sizeof(double) + desc + 8192);
    ctx->scratch.reset();
    double* H = ctx->scratch.alloc_n<double>(htot);
    double* wall = ctx->scratch.alloc_n<double>(wtot);
    NRGB_CUDA(cudaMemsetAsync(H, 0, htot * sizeof(double), st));
    std::vector<AsmDiag> ad;
    std::vector<AsmOff> ao;
    int maxlen = 0, maxrc = 0;
    for (int t = 0; t < plan->ndiag; ++t) {
      const nrgb_diag_term& d = plan->diag[t];
      if (d.blk < 0 || d.blk >= nb || d.off < 0 || d.len < 0 || d.off + d.len > plan->dim[d.blk])
        throw CudaError("nrgb_step: diagonal term out of its block");
      const double* E = nullptr;
      if (d.src >= 0) {
        const PlanMatrix& m = mat(ctx, d.src);
        if ((size_t)m.rows * m.cols < (size_t)d.len) throw CudaError("nrgb_step: energy vector too short");
        E = m.p;
      }
      ad.push_back(AsmDiag{H + hoff[d.blk], E, plan->dim[d.blk], d.off, d.len, d.scale, d.shift});
      maxlen = std::max(maxlen, d.len);
    }
    for (int t = 0; t < plan->noff; ++t) {
      const nrgb_offdiag_term& o = plan->off[t];
      if (o.blk < 0 || o.blk >= nb) throw CudaError("nrgb_step: off-diagonal term: block out of range");
      const int n = plan->dim[o.blk];
      if (o.offi < 0 || o.offj < 0 || o.rows < 0 || o.cols < 0 || o.offi + o.rows > n || o.offj + o.cols > n)
        throw CudaError("nrgb_step: off-diagonal term out of its block");
      if (o.offi < o.offj + o.cols && o.offj < o.offi + o.rows && o.rows > 0 && o.cols > 0)
        throw CudaError("nrgb_step: off-diagonal term overlaps the diagonal");
      if (!std::isfinite(o.factor)) throw CudaError("nrgb_step: off-diagonal factor not finite");
      const double* M = nullptr;  // src < 0: the identity (diag_offdiag_function, src/matrix.cc:256-276)
      int ldm = 1;
      if (o.src >= 0) {
        const PlanMatrix& m = mat(ctx, o.src);
        if (m.rows != o.rows || m.cols != o.cols) throw CudaError("nrgb_step: off-diagonal source size mismatch");
        M = m.p;
        ldm = std::max(1, m.rows);
      } else if (o.rows != o.cols) {
        throw CudaError("nrgb_step: identity term needs a square sub-block");
      }
      ao.push_back(AsmOff{H + hoff[o.blk], M, n, o.offi, o.offj, o.rows, o.cols, ldm, o.factor});
      maxrc = std::max(maxrc, o.rows * o.cols);
    }
    const auto layers = asm_off_layers(ao);
    NRGB_CUDA(assemble_launch(stage(ctx, ad), (int)ad.size(), layers.empty() ? nullptr : stage(ctx, layers[0]),
                              layers.empty() ? 0 : (int)layers[0].size(), maxlen, maxrc, st));
    for (size_t k = 1; k < layers.size(); ++k)
      NRGB_CUDA(assemble_launch(nullptr, 0, stage(ctx, layers[k]), (int)layers[k].size(), 0, maxrc, st));
    // eigen-decomposition of every block
    std::vector<SyevDesc> sd;
    std::vector<int> zh(nb);
    for (int b = 0; b < nb; ++b) {
      zh[b] = new_mat(ctx, plan->dim[b], plan->dim[b]);
      sd.push_back(SyevDesc{plan->dim[b], H + hoff[b], wall + woff[b], ctx->plan.mats[zh[b]].p});
    }
    solver_of(ctx)->solve(sd, st);
    // truncation on the device
    PlanState& S = ctx->plan;
    std::vector<TruncBlock> tb;
    for (int b = 0; b < nb; ++b) tb.push_back(TruncBlock{wall + woff[b], plan->dim[b], (int)woff[b]});
    ensure_map(ctx, S.trunc.map_count + 2 * (int)wtot + 16);
    const size_t wb = trunc_work_bytes((int)wtot, nb);
    if (wb > S.twork_bytes) {
      if (S.twork) NRGB_CUDA(cudaFreeAsync(S.twork, st));
      S.twork_bytes = wb + wb / 2;
      NRGB_CUDA(cudaMallocAsync(&S.twork, S.twork_bytes, st));
    }
    const size_t tbytes = trunc_tail_bytes(nb);
    if (tbytes > S.tail_bytes) {
      if (S.tail_dev) NRGB_CUDA(cudaFreeAsync(S.tail_dev, st));
      S.tail_bytes = tbytes + tbytes / 2;
      NRGB_CUDA(cudaMallocAsync(&S.tail_dev, S.tail_bytes, st));
    }
    if (tbytes > S.tail_pin_bytes) {
      NRGB_CUDA(cudaStreamSynchronize(st));
      if (S.tail_pin) NRGB_CUDA(cudaFreeHost(S.tail_pin));
      S.tail_pin_bytes = tbytes + tbytes / 2;
      NRGB_CUDA(cudaMallocHost(&S.tail_pin, S.tail_pin_bytes));
    }
    TruncRules R{plan->fixeps, plan->keepenergy, plan->keep, plan->keepmin, plan->safeguard, plan->safeguardmax,
                 plan->keep_all, plan->betabar};
    NRGB_CUDA(truncate_step(stage(ctx, tb), nb, wall, (int)wtot, R, S.trunc, S.twork, S.tail_dev, st));
    // the corrected eigenvalues of each block under their own handles
    std::vector<int> wh(nb);
    for (int b = 0; b < nb; ++b) {
      wh[b] = new_mat(ctx, plan->dim[b], 1);
      NRGB_CUDA(cudaMemcpyAsync(S.mats[wh[b]].p, wall + woff[b], plan->dim[b] * sizeof(double),
                                cudaMemcpyDeviceToDevice, st));
    }
    NRGB_CUDA(cudaMemcpyAsync(S.tail_pin, S.tail_dev, tbytes, cudaMemcpyDeviceToHost, st));
    NRGB_CUDA(cudaStreamSynchronize(st));
    const TruncTail& T = *reinterpret_cast<const TruncTail*>(S.tail_pin);
    if (T.flags & 1) throw CudaError("nrgb_step: ground state not at zero");
    if (T.flags & 2) throw CudaError("nrgb_step: eigenvalues of a block not ascending after the splitting correction");
    S.trunc.map_count = T.map_count;
    const int* kp = trunc_tail_kept(S.tail_pin);
    const double* sums = trunc_tail_sums(S.tail_pin, nb);
    for (int b = 0; b < nb; ++b) {
      z_handles[b] = zh[b];
      w_handles[b] = wh[b];
      kept[b] = kp[b];
      if (zsums)
        for (int k = 0; k < 3; ++k) zsums[3 * b + k] = sums[3 * b + k];
    }
    *egs = T.Egs;
  });
}

int nrgb_recalc(nrgb_ctx* ctx, int nout, const nrgb_recalc_out* outs, int nterms, const nrgb_recalc_term* terms,
                int* out_handles) {
  if (nout < 0 || nterms < 0 || (nout > 0 && (!outs || !out_handles)) || (nterms > 0 && !terms)) return 1;
  return guarded(ctx, [&] {
    using namespace nrgb;
    cudaStream_t st = ctx->stream;
    // the sub-block Z[off : off+r, 0 : k] of a block's eigenvectors (column-major,
    // ld = block dimension) is U^T of the reference's split_in_blocks
    std::vector<GemmProb> p1, p2;
    std::vector<GemmSeg> s1, s2;
    int t1 = 0, st1 = 0, t2 = 0, st2 = 0;
    size_t tbytes = 0;
    for (int o = 0; o < nout; ++o)
      for (int t = outs[o].term0; t < outs[o].term0 + outs[o].nterms; ++t) {
        if (t < 0 || t >= nterms) throw CudaError("nrgb_recalc: term range out of bounds");
        if (terms[t].op >= 0) tbytes += ((size_t)terms[t].r1 * outs[o].kp * sizeof(double) + 255) & ~size_t(255);
      }
    ctx->scratch.reserve(tbytes + (size_t)(2 * nterms + 2 * nout + 8) * (sizeof(GemmProb) + sizeof(GemmSeg)) + 8192);
    ctx->scratch.reset();
    for (int o = 0; o < nout; ++o) {
      const nrgb_recalc_out& Y = outs[o];
      if (Y.k1 < 0 || Y.kp < 0) throw CudaError("nrgb_recalc: negative output size");
      const int h = new_mat(ctx, Y.k1, Y.kp);
      out_handles[o] = h;
      double* C = ctx->plan.mats[h].p;
      if (Y.k1 == 0 || Y.kp == 0) continue;
      std::vector<GemmSeg> segs;
      for (int t = Y.term0; t < Y.term0 + Y.nterms; ++t) {
        const nrgb_recalc_term& x = terms[t];
        const PlanMatrix& Z1 = mat(ctx, x.z1);
        const PlanMatrix& Zp = mat(ctx, x.zp);
        if (x.r1 <= 0 || x.rp <= 0) continue;
        if (x.off1 < 0 || x.off1 + x.r1 > Z1.rows || Y.k1 > Z1.cols || x.offp < 0 || x.offp + x.rp > Zp.rows ||
            Y.kp > Zp.cols)
          throw CudaError("nrgb_recalc: sub-block outside its eigenvector matrix");
        if (x.op < 0) {
          // recalc_f form: factor * U1 Up^T = Z1sub^T Zpsub (r1 == rp)
          if (x.r1 != x.rp) throw CudaError("nrgb_recalc: identity term needs r1 == rp");
          segs.push_back(GemmSeg{Z1.p + x.off1, Zp.p + x.offp, Z1.rows, Zp.rows, x.r1, 1, 0, x.factor});
        } else {
          const PlanMatrix& O = mat(ctx, x.op);
          if (O.rows < x.r1 || O.cols < x.rp) throw CudaError("nrgb_recalc: operator block too small");
          // temp = O[0:r1, 0:rp] * Zp[offp : offp+rp, 0 : kp]   (r1 x kp)
          double* Tm = static_cast<double*>(ctx->scratch.alloc((size_t)x.r1 * Y.kp * sizeof(double)));
          GemmProb a{};
          a.C = Tm;
          a.ldc = x.r1;
          a.m = x.r1;
          a.n = Y.kp;
          a.beta = 0.0;
          a.seg0 = (int)s1.size();
          a.nseg = 1;
          gemm_assign_tiles(a, t1, st1);
          p1.push_back(a);
          s1.push_back(GemmSeg{O.p, Zp.p + x.offp, std::max(1, O.rows), Zp.rows, x.rp, 0, 0, 1.0});
          segs.push_back(GemmSeg{Z1.p + x.off1, Tm, Z1.rows, x.r1, x.r1, 1, 0, x.factor});
        }
      }
      if (segs.empty()) {
        NRGB_CUDA(cudaMemsetAsync(C, 0, (size_t)Y.k1 * Y.kp * sizeof(double), st));
        continue;
      }
      GemmProb b{};
      b.C = C;
      b.ldc = Y.k1;
      b.m = Y.k1;
      b.n = Y.kp;
      b.beta = 0.0;
      b.seg0 = (int)s2.size();
      b.nseg = (int)segs.size();
      gemm_assign_tiles(b, t2, st2);
      p2.push_back(b);
      s2.insert(s2.end(), segs.begin(), segs.end());
    }
    auto launch = [&](std::vector<GemmProb>& P, std::vector<GemmSeg>& Sg, int tiles, int stiles) {
      if (P.empty()) return;
      GemmProb* dP = stage(ctx, P);
      GemmSeg* dS = stage(ctx, Sg);
      KernelStats::get().add_work("gemm_f64_recalc", gemm_flops(P.data(), (int)P.size(), Sg.data()));
      NRGB_CUDA(gemm_grouped_launch(dP, (int)P.size(), dS, tiles, st, "gemm_f64_recalc", stiles));
    };
    launch(p1, s1, t1, st1);
    launch(p2, s2, t2, st2);
    NRGB_CUDA(cudaStreamSynchronize(st));
  });
}

int nrgb_dm_backward(nrgb_ctx* ctx, int nout, const nrgb_dm_out* outs, int nterms, const nrgb_dm_term* terms,
                     int* out_handles) {
  if (nout < 0 || nterms < 0 || (nout > 0 && (!outs || !out_handles)) || (nterms > 0 && !terms)) return 1;
  return guarded(ctx, [&] {
    using namespace nrgb;
    cudaStream_t st = ctx->stream;
    // output (r1 x rp) = sum factor * Z1sub * rho * Zpsub^T with Zsub = Z[off : off+r, 0 : k]:
    // first T = rho * Zpsub^T (k1 x rp), then factor * Z1sub * T
    std::vector<GemmProb> p1, p2;
    std::vector<GemmSeg> s1, s2;
    int t1 = 0, st1 = 0, t2 = 0, st2 = 0;
    size_t tbytes = 0;
    for (int o = 0; o < nout; ++o)
      for (int t = outs[o].term0; t < outs[o].term0 + outs[o].nterms; ++t) {
        if (t < 0 || t >= nterms) throw CudaError("nrgb_dm_backward: term range out of bounds");
        if (terms[t].k1 > 0) tbytes += ((size_t)terms[t].k1 * std::max(0, outs[o].rp) * sizeof(double) + 255) & ~size_t(255);
      }
    ctx->scratch.reserve(tbytes + (size_t)(2 * nterms + 2 * nout + 8) * (sizeof(GemmProb) + sizeof(GemmSeg)) + 8192);
    ctx->scratch.reset();
    for (int o = 0; o < nout; ++o) {
      const nrgb_dm_out& Y = outs[o];
      if (Y.r1 < 0 || Y.rp < 0) throw CudaError("nrgb_dm_backward: negative output size");
      const int h = new_mat(ctx, Y.r1, Y.rp);
      out_handles[o] = h;
      double* C = ctx->plan.mats[h].p;
      if (Y.r1 == 0 || Y.rp == 0) continue;
      std::vector<GemmSeg> segs;
      for (int t = Y.term0; t < Y.term0 + Y.nterms; ++t) {
        const nrgb_dm_term& x = terms[t];
        if (x.k1 <= 0 || x.kp <= 0) continue;
        const PlanMatrix& Z1 = mat(ctx, x.z1);
        const PlanMatrix& Zp = mat(ctx, x.zp);
        const PlanMatrix& R = mat(ctx, x.rho);
        if (x.off1 < 0 || x.off1 + Y.r1 > Z1.rows || x.k1 > Z1.cols || x.offp < 0 || x.offp + Y.rp > Zp.rows ||
            x.kp > Zp.cols)
          throw CudaError("nrgb_dm_backward: sub-block outside its eigenvector matrix");
        if (R.rows < x.k1 || R.cols < x.kp) throw CudaError("nrgb_dm_backward: density matrix too small");
        double* Tm = static_cast<double*>(ctx->scratch.alloc((size_t)x.k1 * Y.rp * sizeof(double)));
        GemmProb a{};
        a.C = Tm;
        a.ldc = x.k1;
        a.m = x.k1;
        a.n = Y.rp;
        a.beta = 0.0;
        a.seg0 = (int)s1.size();
        a.nseg = 1;
        gemm_assign_tiles(a, t1, st1);
        p1.push_back(a);
        // op(B)[p, j] = Zp[offp + j, p]: the sub-block read transposed
        s1.push_back(GemmSeg{R.p, Zp.p + x.offp, std::max(1, R.rows), Zp.rows, x.kp, 0, 1, 1.0});
        segs.push_back(GemmSeg{Z1.p + x.off1, Tm, Z1.rows, x.k1, x.k1, 0, 0, x.factor});
      }
      if (segs.empty()) {
        NRGB_CUDA(cudaMemsetAsync(C, 0, (size_t)Y.r1 * Y.rp * sizeof(double), st));
        continue;
      }
      GemmProb b{};
      b.C = C;
      b.ldc = Y.r1;
      b.m = Y.r1;
      b.n = Y.rp;
      b.beta = 0.0;
      b.seg0 = (int)s2.size();
      b.nseg = (int)segs.size();
      gemm_assign_tiles(b, t2, st2);
      p2.push_back(b);
      s2.insert(s2.end(), segs.begin(), segs.end());
    }
    auto launch = [&](std::vector<GemmProb>& P, std::vector<GemmSeg>& Sg, int tiles, int stiles) {
      if (P.empty()) return;
      GemmProb* dP = stage(ctx, P);
      GemmSeg* dS = stage(ctx, Sg);
      KernelStats::get().add_work("gemm_f64_dm", gemm_flops(P.data(), (int)P.size(), Sg.data()));
      NRGB_CUDA(gemm_grouped_launch(dP, (int)P.size(), dS, tiles, st, "gemm_f64_dm", stiles));
    };
    launch(p1, s1, t1, st1);
    launch(p2, s2, t2, st2);
    NRGB_CUDA(cudaStreamSynchronize(st));
  });
}

int nrgb_spectrum_fdm(nrgb_ctx* ctx, int npairs, const nrgb_fdm_pair* pairs, double T, double wn, int fermionic,
                      double bins_per_decade, double emin, double emax, double discard, int nbins, double* bins) {
  if (npairs < 0 || (npairs > 0 && !pairs) || !bins || !(T > 0.0) || !(bins_per_decade > 0.0) || !(emin > 0.0) ||
      !(emax > emin) || !(discard >= 0.0))
    return 1;
  return guarded(ctx, [&] {
    using namespace nrgb;
    cudaStream_t st = ctx->stream;
    // the logarithmic grid of src/bins.h:22-131, as the whole-run driver builds it
    BinGrid grid{};
    const double l0 = floor(log10(emin)), l1 = ceil(log10(emax));
    grid.l0 = l0;
    grid.bpd = bins_per_decade;
    grid.nbins = (int)((l1 - l0) * bins_per_decade + 1.0);
    grid.discard = discard;
    if (grid.nbins != nbins) throw CudaError("nrgb_spectrum_fdm: nbins does not match the grid");
    // per pair: the two products with the density matrices and the
    // Boltzmann factors of both blocks' states
    size_t bytes = 2 * (size_t)nbins * sizeof(double) + (size_t)npairs * sizeof(SpecFdmPair) + 8192;
    std::vector<double> hx;  // every pair's two energy lists, back to back, then exp(-E/T) in place
    std::vector<size_t> xo(2 * (size_t)npairs);
    for (int k = 0; k < npairs; ++k) {
      const nrgb_fdm_pair& q = pairs[k];
      const PlanMatrix& A = mat(ctx, q.op1);
      const PlanMatrix& B = mat(ctx, q.op2);
      if (A.rows != B.rows || A.cols != B.cols) throw CudaError("nrgb_spectrum_fdm: operator blocks differ in shape");
      if (q.reti < 0 || q.retj < 0 || q.reti > A.cols || q.retj > A.rows)
        throw CudaError("nrgb_spectrum_fdm: kept states outside the block");
      bytes += (((size_t)A.rows * q.reti + (size_t)q.retj * A.cols) * sizeof(double) + 512);
      for (int side = 0; side < 2; ++side) {
        const PlanMatrix& E = mat(ctx, side ? q.e_j : q.e_i);
        const int want = side ? A.rows : A.cols;
        if ((long)E.rows * E.cols != want) throw CudaError("nrgb_spectrum_fdm: energy list length differs from the block");
        xo[2 * k + side] = hx.size();
        hx.resize(hx.size() + want);
      }
    }
    for (int k = 0; k < npairs; ++k)
      for (int side = 0; side < 2; ++side) {
        const PlanMatrix& E = mat(ctx, side ? pairs[k].e_j : pairs[k].e_i);
        const size_t want = (size_t)E.rows * E.cols;
        if (want)
          NRGB_CUDA(cudaMemcpyAsync(hx.data() + xo[2 * k + side], E.p, want * sizeof(double), cudaMemcpyDeviceToHost,
                                    st));
      }
    NRGB_CUDA(cudaStreamSynchronize(st));
    for (double& x : hx) x = exp(-x / T);
    bytes += hx.size() * sizeof(double) + (size_t)(4 * npairs + 16) * 512;  // allocations and their alignment
    ctx->scratch.reserve(bytes + (size_t)(2 * npairs + 8) * (sizeof(GemmProb) + sizeof(GemmSeg)));
    ctx->scratch.reset();
    double* dx = static_cast<double*>(ctx->scratch.alloc(std::max<size_t>(1, hx.size()) * sizeof(double)));
    if (!hx.empty()) NRGB_CUDA(cudaMemcpyAsync(dx, hx.data(), hx.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    std::vector<GemmProb> gp;
    std::vector<GemmSeg> gs;
    int tiles = 0, stiles = 0;
    auto product = [&](double* C, int m, int n, const double* a, int lda, const double* b, int ldb, int k) {
      GemmProb g{};
      g.C = C;
      g.ldc = m;
      g.m = m;
      g.n = n;
      g.beta = 0.0;
      g.seg0 = (int)gs.size();
      g.nseg = 1;
      gemm_assign_tiles(g, tiles, stiles);
      gp.push_back(g);
      gs.push_back(GemmSeg{a, b, lda, ldb, k, 0, 0, 1.0});
    };
    std::vector<SpecFdmPair> sp;
    int maxe = 0;
    for (int k = 0; k < npairs; ++k) {
      const nrgb_fdm_pair& q = pairs[k];
      const PlanMatrix& A = mat(ctx, q.op1);
      const PlanMatrix& B = mat(ctx, q.op2);
      const int allj = A.rows, alli = A.cols;
      if (!allj || !alli) continue;
      double* O2R = nullptr;
      double* RO2 = nullptr;
      if (q.reti > 0) {  // op2[:allj, :reti] * rho_i
        const PlanMatrix& R = mat(ctx, q.rho_i);
        if (R.rows < q.reti || R.cols < q.reti) throw CudaError("nrgb_spectrum_fdm: rho_i too small");
        O2R = static_cast<double*>(ctx->scratch.alloc((size_t)allj * q.reti * sizeof(double)));
        product(O2R, allj, q.reti, B.p, B.rows, R.p, R.rows, q.reti);
      }
      if (q.retj > 0) {  // rho_j * op2[:retj, :alli]
        const PlanMatrix& R = mat(ctx, q.rho_j);
        if (R.rows < q.retj || R.cols < q.retj) throw CudaError("nrgb_spectrum_fdm: rho_j too small");
        RO2 = static_cast<double*>(ctx->scratch.alloc((size_t)q.retj * alli * sizeof(double)));
        product(RO2, q.retj, alli, R.p, R.rows, B.p, B.rows, q.retj);
      }
      sp.push_back(SpecFdmPair{A.p, B.p, O2R, RO2, mat(ctx, q.e_j).p, mat(ctx, q.e_i).p, dx + xo[2 * k + 1],
                               dx + xo[2 * k], A.rows, allj, alli, q.retj, q.reti, q.factor});
      maxe = std::max(maxe, allj * alli);
    }
    if (!gp.empty()) {
      GemmProb* dP = stage(ctx, gp);
      GemmSeg* dS = stage(ctx, gs);
      NRGB_CUDA(gemm_grouped_launch(dP, (int)gp.size(), dS, tiles, st, "gemm_f64_spec", stiles));
    }
    double* dbins = static_cast<double*>(ctx->scratch.alloc(2 * (size_t)nbins * sizeof(double)));
    NRGB_CUDA(cudaMemsetAsync(dbins, 0, 2 * (size_t)nbins * sizeof(double), st));
    if (!sp.empty())
      NRGB_CUDA(spec_fdm_launch(stage(ctx, sp), (int)sp.size(), maxe, grid, T, wn, fermionic ? 1.0 : -1.0, dbins, st));
    std::vector<double> hb(2 * (size_t)nbins);
    NRGB_CUDA(cudaMemcpyAsync(hb.data(), dbins, hb.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    NRGB_CUDA(cudaStreamSynchronize(st));
    for (size_t i = 0; i < hb.size(); ++i) bins[i] += hb[i];
  });
}

int nrgb_spectrum_dmnrg(nrgb_ctx* ctx, int npairs, const nrgb_dmnrg_pair* pairs, double scale, double ewin_min,
                        double ewin_max, int fermionic, double bins_per_decade, double emin, double emax,
                        double discard, int nbins, double* bins) {
  if (npairs < 0 || (npairs > 0 && !pairs) || !bins || !(scale > 0.0) || !(ewin_max >= ewin_min) ||
      !(bins_per_decade > 0.0) || !(emin > 0.0) || !(emax > emin) || !(discard >= 0.0))
    return 1;
  return guarded(ctx, [&] {
    using namespace nrgb;
    cudaStream_t st = ctx->stream;
    BinGrid grid{};
    const double l0 = floor(log10(emin)), l1 = ceil(log10(emax));
    grid.l0 = l0;
    grid.bpd = bins_per_decade;
    grid.nbins = (int)((l1 - l0) * bins_per_decade + 1.0);
    grid.discard = discard;
    if (grid.nbins != nbins) throw CudaError("nrgb_spectrum_dmnrg: nbins does not match the grid");
    size_t bytes = 2 * (size_t)nbins * sizeof(double) + (size_t)(4 * npairs + 16) * 512 +
                   (size_t)(2 * npairs + 8) * (sizeof(GemmProb) + sizeof(GemmSeg) + sizeof(SpecDmnrgPair));
    for (int k = 0; k < npairs; ++k) {
      const int d1 = mat(ctx, pairs[k].rho_1).rows, dp = mat(ctx, pairs[k].rho_p).rows;
      bytes += 2 * (size_t)d1 * dp * sizeof(double);
    }
    ctx->scratch.reserve(bytes);
    ctx->scratch.reset();
    std::vector<GemmProb> gp;
    std::vector<GemmSeg> gs;
    int tiles = 0, stiles = 0;
    auto product = [&](double* C, int m, int n, const double* a, int lda, const double* b, int ldb, int k) {
      GemmProb g{};
      g.C = C;
      g.ldc = m;
      g.m = m;
      g.n = n;
      g.beta = 0.0;
      g.seg0 = (int)gs.size();
      g.nseg = 1;
      gemm_assign_tiles(g, tiles, stiles);
      gp.push_back(g);
      gs.push_back(GemmSeg{a, b, lda, ldb, k, 0, 0, 1.0});
    };
    std::vector<SpecDmnrgPair> sp;
    int maxe = 0;
    for (int k = 0; k < npairs; ++k) {
      const nrgb_dmnrg_pair& q = pairs[k];
      const PlanMatrix& A = mat(ctx, q.op1);
      const PlanMatrix& B = mat(ctx, q.op2);
      const PlanMatrix& R1 = mat(ctx, q.rho_1);
      const PlanMatrix& Rp = mat(ctx, q.rho_p);
      const int d1 = R1.rows, dp = Rp.rows;
      if (R1.cols != d1 || Rp.cols != dp) throw CudaError("nrgb_spectrum_dmnrg: density matrices must be square");
      if (A.rows != B.rows || A.cols != B.cols || A.rows < d1 || A.cols < dp)
        throw CudaError("nrgb_spectrum_dmnrg: operator blocks smaller than the kept states or of different shapes");
      const PlanMatrix& E1 = mat(ctx, q.e_1);
      const PlanMatrix& Ep = mat(ctx, q.e_p);
      if ((long)E1.rows * E1.cols < d1 || (long)Ep.rows * Ep.cols < dp)
        throw CudaError("nrgb_spectrum_dmnrg: energy list shorter than the kept states");
      if (!d1 || !dp) continue;
      // SA = op2[:d1, :dp] * rho_p,  SB = rho_1 * op1[:d1, :dp]  (src/spec_DMNRG.cc:13-52)
      double* SA = static_cast<double*>(ctx->scratch.alloc((size_t)d1 * dp * sizeof(double)));
      double* SB = static_cast<double*>(ctx->scratch.alloc((size_t)d1 * dp * sizeof(double)));
      product(SA, d1, dp, B.p, B.rows, Rp.p, Rp.rows, dp);
      product(SB, d1, dp, R1.p, R1.rows, A.p, A.rows, d1);
      sp.push_back(SpecDmnrgPair{A.p, B.p, SA, SB, E1.p, Ep.p, A.rows, d1, dp, q.factor});
      maxe = std::max(maxe, d1 * dp);
    }
    if (!gp.empty()) {
      GemmProb* dP = stage(ctx, gp);
      GemmSeg* dS = stage(ctx, gs);
      NRGB_CUDA(gemm_grouped_launch(dP, (int)gp.size(), dS, tiles, st, "gemm_f64_spec", stiles));
    }
    double* dbins = static_cast<double*>(ctx->scratch.alloc(2 * (size_t)nbins * sizeof(double)));
    NRGB_CUDA(cudaMemsetAsync(dbins, 0, 2 * (size_t)nbins * sizeof(double), st));
    if (!sp.empty())
      NRGB_CUDA(spec_dmnrg_launch(stage(ctx, sp), (int)sp.size(), maxe, grid, scale, ewin_min, ewin_max,
                                  fermionic ? 1.0 : -1.0, dbins, st));
    std::vector<double> hb(2 * (size_t)nbins);
    NRGB_CUDA(cudaMemcpyAsync(hb.data(), dbins, hb.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    NRGB_CUDA(cudaStreamSynchronize(st));
    for (size_t i = 0; i < hb.size(); ++i) bins[i] += hb[i];
  });
}

}  // extern "C"
