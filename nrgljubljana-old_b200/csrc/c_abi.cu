// C ABI of libnrgb.so (declarations and the reference seams they replace are
// in include/nrgb.h).
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "../../include/nrgb.h"
#include "common.cuh"
#include "gemm_f64.cuh"
#include "autotune.cuh"
#include "gemm_split.cuh"
#include "schedule.cuh"
#include "syev.cuh"
#include "../host/driver.h"

#include "ctx.h"

using nrgb::guarded;
using nrgb::solver_of;

extern "C" {

const char* nrgb_version(void) { return "nrgb 0.1 (sm_100a, FP64 DMMA)"; }

int nrgb_create(int device, nrgb_ctx** out) {
  if (!out) return 1;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return 3;
  if (device < 0 || device >= count) return 4;
  auto* c = new nrgb_ctx;
  c->device = device;
  int rc = guarded(c, [&] {
    NRGB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->syev.reset(new nrgb::SyevBatched());
  });
  if (rc) {
    delete c;
    return rc;
  }
  *out = c;
  return 0;
}

int nrgb_destroy(nrgb_ctx* ctx) {
  if (!ctx) return 0;
  cudaSetDevice(ctx->device);
  ctx->driver.reset();
  nrgb::plan_release(ctx);
  ctx->syev.reset();
  ctx->scratch.release();
  ctx->io.release();
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return 0;
}

const char* nrgb_last_error(const nrgb_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int nrgb_syev_batched_dev(nrgb_ctx* ctx, int nblocks, const int* n, double* const* a_dev,
                          double* const* w_dev, double* const* z_dev, void* stream) {
  return guarded(ctx, [&] {
    std::vector<nrgb::SyevDesc> d(nblocks);
    for (int b = 0; b < nblocks; ++b) {
      if (n[b] > 0 && a_dev[b] == z_dev[b]) throw nrgb::CudaError("z_dev must not alias a_dev");
      d[b] = nrgb::SyevDesc{n[b], a_dev[b], w_dev[b], z_dev[b]};
    }
    ctx->syev->run(d, (cudaStream_t)stream);
  });
}

int nrgb_syev_batched(nrgb_ctx* ctx, int nblocks, const int* n, double* const* a, double* const* w) {
  return guarded(ctx, [&] {
    size_t tot = 0;
    for (int b = 0; b < nblocks; ++b) tot += 2 * (size_t)n[b] * n[b] + n[b] + 96;
    ctx->scratch.reserve(tot * sizeof(double) + 256 * (size_t)nblocks * 4 + (1 << 16));
    ctx->scratch.reset();
    std::vector<nrgb::SyevDesc> d(nblocks);
    cudaStream_t st = ctx->stream;
    for (int b = 0; b < nblocks; ++b) {
      const size_t nn = (size_t)n[b] * n[b];
      double* A = ctx->scratch.alloc_n<double>(nn);
      double* Z = ctx->scratch.alloc_n<double>(nn);
      double* W = ctx->scratch.alloc_n<double>(n[b] + 1);
      if (nn) NRGB_CUDA(cudaMemcpyAsync(A, a[b], nn * sizeof(double), cudaMemcpyHostToDevice, st));
      d[b] = nrgb::SyevDesc{n[b], A, W, Z};
    }
    solver_of(ctx)->solve(d, st);
    for (int b = 0; b < nblocks; ++b) {
      const size_t nn = (size_t)n[b] * n[b];
      if (!nn) continue;
      NRGB_CUDA(cudaMemcpyAsync(a[b], d[b].Z, nn * sizeof(double), cudaMemcpyDeviceToHost, st));
      NRGB_CUDA(cudaMemcpyAsync(w[b], d[b].w, n[b] * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    NRGB_CUDA(cudaStreamSynchronize(st));
  });
}

int nrgb_gemm_grouped_split_dev(nrgb_ctx* ctx, int slices, int nout, const nrgb_gemm_out* outs, int nterms,
                                const nrgb_gemm_term* terms, void* stream) {
  if (slices < nrgb::SPLIT_MIN_SLICES || slices > nrgb::SPLIT_MAX_SLICES) return 1;
  return guarded(ctx, [&] {
    std::vector<nrgb::GemmProb> P;
    std::vector<nrgb::GemmSeg> S(nterms);
    for (int t = 0; t < nterms; ++t) {
      const nrgb_gemm_term& x = terms[t];
      S[t] = nrgb::GemmSeg{x.a, x.b, x.lda, x.ldb, x.k, x.trans_a, x.trans_b, x.alpha};
    }
    for (int o = 0; o < nout; ++o) {
      const nrgb_gemm_out& y = outs[o];
      if (y.m <= 0 || y.n <= 0) continue;
      if (y.term0 < 0 || y.term0 + y.nterms > nterms) throw nrgb::CudaError("gemm: term range out of bounds");
      nrgb::GemmProb p{};
      p.C = y.c;
      p.ldc = y.ldc;
      p.m = y.m;
      p.n = y.n;
      p.beta = y.beta;
      p.seg0 = y.term0;
      p.nseg = y.nterms;
      P.push_back(p);
    }
    if (P.empty()) return;
    cudaStream_t st = (cudaStream_t)stream;
    ctx->scratch.reserve(nrgb::split_gemm_workspace(P.data(), (int)P.size(), S.data(), slices));
    ctx->scratch.reset();
    nrgb::split_gemm_grouped(P.data(), (int)P.size(), S.data(), slices, ctx->scratch, st);
    if (nrgb::split_gemm_take_error(st)) throw nrgb::CudaError("split gemm: a barrier wait timed out");
  });
}

int nrgb_gemm_grouped_dev(nrgb_ctx* ctx, int nout, const nrgb_gemm_out* outs, int nterms,
                          const nrgb_gemm_term* terms, void* stream) {
  return guarded(ctx, [&] {
    std::vector<nrgb::GemmProb> P;
    std::vector<nrgb::GemmSeg> S(nterms);
    for (int t = 0; t < nterms; ++t) {
      const nrgb_gemm_term& x = terms[t];
      S[t] = nrgb::GemmSeg{x.a, x.b, x.lda, x.ldb, x.k, x.trans_a, x.trans_b, x.alpha};
    }
    int tiles = 0, stiles = 0;
    for (int o = 0; o < nout; ++o) {
      const nrgb_gemm_out& y = outs[o];
      if (y.m <= 0 || y.n <= 0) continue;
      if (y.term0 < 0 || y.term0 + y.nterms > nterms) throw nrgb::CudaError("gemm: term range out of bounds");
      nrgb::GemmProb p{};
      p.C = y.c;
      p.ldc = y.ldc;
      p.m = y.m;
      p.n = y.n;
      p.beta = y.beta;
      p.seg0 = y.term0;
      p.nseg = y.nterms;
      nrgb::gemm_assign_tiles(p, tiles, stiles);
      P.push_back(p);
    }
    if (P.empty()) return;
    cudaStream_t st = (cudaStream_t)stream;
    const size_t bytes = P.size() * sizeof(nrgb::GemmProb) + S.size() * sizeof(nrgb::GemmSeg) + 1024;
    ctx->scratch.reserve(bytes);
    ctx->scratch.reset();
    auto* dP = ctx->scratch.alloc_n<nrgb::GemmProb>(P.size());
    auto* dS = ctx->scratch.alloc_n<nrgb::GemmSeg>(S.size());
    NRGB_CUDA(cudaMemcpyAsync(dP, P.data(), P.size() * sizeof(nrgb::GemmProb), cudaMemcpyHostToDevice, st));
    NRGB_CUDA(cudaMemcpyAsync(dS, S.data(), S.size() * sizeof(nrgb::GemmSeg), cudaMemcpyHostToDevice, st));
    nrgb::KernelStats::get().add_work("gemm_f64", nrgb::gemm_flops(P.data(), (int)P.size(), S.data()));
    NRGB_CUDA(nrgb::gemm_grouped_launch(dP, (int)P.size(), dS, tiles, st, "gemm_f64", stiles));
    NRGB_CUDA(cudaStreamSynchronize(st));
  });
}

namespace {
// out[o] = Z_bra^T * op[o] * Z_ket for all o, two grouped GEMM launches.
void recalc_pairs(nrgb_ctx* ctx, int nops, const int* n, const int* bra, const int* ket, double* const* Z,
                  const double* const* op, double* const* out, nrgb::DeviceArena& scr, cudaStream_t st) {
  std::vector<nrgb::GemmProb> p1, p2;
  std::vector<nrgb::GemmSeg> s1, s2;
  int t1 = 0, t2 = 0, u1 = 0, u2 = 0;
  auto add = [](std::vector<nrgb::GemmProb>& P, std::vector<nrgb::GemmSeg>& S, int& tiles, int& stiles,
                double* C, int m, int nn, const nrgb::GemmSeg& g) {
    nrgb::GemmProb q{};
    q.C = C;
    q.ldc = m;
    q.m = m;
    q.n = nn;
    q.beta = 0.0;
    q.seg0 = (int)S.size();
    q.nseg = 1;
    nrgb::gemm_assign_tiles(q, tiles, stiles);
    P.push_back(q);
    S.push_back(g);
  };
  for (int o = 0; o < nops; ++o) {
    const int nb = n[bra[o]], nk = n[ket[o]];
    if (nb <= 0 || nk <= 0) continue;
    double* T = scr.alloc_n<double>((size_t)nb * nk);
    add(p1, s1, t1, u1, T, nb, nk, nrgb::GemmSeg{op[o], Z[ket[o]], nb, nk, nk, 0, 0, 1.0});
    add(p2, s2, t2, u2, out[o], nb, nk, nrgb::GemmSeg{Z[bra[o]], T, nb, nb, nb, 1, 0, 1.0});
  }
  if (p1.empty()) return;
  auto* d1 = scr.alloc_n<nrgb::GemmProb>(p1.size());
  auto* e1 = scr.alloc_n<nrgb::GemmSeg>(s1.size());
  auto* d2 = scr.alloc_n<nrgb::GemmProb>(p2.size());
  auto* e2 = scr.alloc_n<nrgb::GemmSeg>(s2.size());
  NRGB_CUDA(cudaMemcpyAsync(d1, p1.data(), p1.size() * sizeof(p1[0]), cudaMemcpyHostToDevice, st));
  NRGB_CUDA(cudaMemcpyAsync(e1, s1.data(), s1.size() * sizeof(s1[0]), cudaMemcpyHostToDevice, st));
  NRGB_CUDA(cudaMemcpyAsync(d2, p2.data(), p2.size() * sizeof(p2[0]), cudaMemcpyHostToDevice, st));
  NRGB_CUDA(cudaMemcpyAsync(e2, s2.data(), s2.size() * sizeof(s2[0]), cudaMemcpyHostToDevice, st));
  nrgb::KernelStats::get().add_work("gemm_f64_recalc", nrgb::gemm_flops(p1.data(), (int)p1.size(), s1.data()) +
                                                           nrgb::gemm_flops(p2.data(), (int)p2.size(), s2.data()));
  NRGB_CUDA(nrgb::gemm_grouped_launch(d1, (int)p1.size(), e1, t1, st, "gemm_f64_recalc", u1));
  NRGB_CUDA(nrgb::gemm_grouped_launch(d2, (int)p2.size(), e2, t2, st, "gemm_f64_recalc", u2));
}

size_t recalc_scratch(int nops, const int* n, const int* bra, const int* ket) {
  size_t b = 0;
  for (int o = 0; o < nops; ++o) b += ((size_t)n[bra[o]] * n[ket[o]] + 64) * sizeof(double);
  return b + (size_t)nops * 4 * 128 + (1 << 16);
}
}  // namespace

int nrgb_eig_recalc_step_dev(nrgb_ctx* ctx, int nblocks, const int* n, double* const* a_dev,
                             double* const* w_dev, double* const* z_dev, int nops, const int* bra,
                             const int* ket, const double* const* op_dev, double* const* out_dev,
                             void* stream) {
  return guarded(ctx, [&] {
    cudaStream_t st = (cudaStream_t)stream;
    for (int o = 0; o < nops; ++o)
      if (bra[o] < 0 || bra[o] >= nblocks || ket[o] < 0 || ket[o] >= nblocks)
        throw nrgb::CudaError("eig_recalc: operator block index out of range");
    std::vector<nrgb::SyevDesc> d(nblocks);
    for (int b = 0; b < nblocks; ++b) d[b] = nrgb::SyevDesc{n[b], a_dev[b], w_dev[b], z_dev[b]};
    solver_of(ctx)->solve(d, st);
    ctx->scratch.reserve(recalc_scratch(nops, n, bra, ket));
    ctx->scratch.reset();
    recalc_pairs(ctx, nops, n, bra, ket, z_dev, op_dev, out_dev, ctx->scratch, st);
    NRGB_CUDA(cudaStreamSynchronize(st));
  });
}

int nrgb_eig_recalc_step(nrgb_ctx* ctx, int nblocks, const int* n, const double* const* h,
                         double* const* w, double* const* z, int nops, const int* bra, const int* ket,
                         const double* const* op, double* const* out) {
  return guarded(ctx, [&] {
    cudaStream_t st = ctx->stream;
    for (int o = 0; o < nops; ++o)
      if (bra[o] < 0 || bra[o] >= nblocks || ket[o] < 0 || ket[o] >= nblocks)
        throw nrgb::CudaError("eig_recalc: operator block index out of range");
    size_t tot = recalc_scratch(nops, n, bra, ket);
    for (int b = 0; b < nblocks; ++b) tot += (2 * (size_t)n[b] * n[b] + n[b] + 96) * sizeof(double);
    for (int o = 0; o < nops; ++o) tot += (2 * (size_t)n[bra[o]] * n[ket[o]] + 64) * sizeof(double);
    ctx->io.reserve(tot);
    ctx->io.reset();
    std::vector<double*> A(nblocks), W(nblocks), Z(nblocks), O(nops), R(nops);
    std::vector<nrgb::SyevDesc> d(nblocks);
    for (int b = 0; b < nblocks; ++b) {
      const size_t nn = (size_t)n[b] * n[b];
      A[b] = ctx->io.alloc_n<double>(nn);
      Z[b] = ctx->io.alloc_n<double>(nn);
      W[b] = ctx->io.alloc_n<double>(n[b] + 1);
      if (nn) NRGB_CUDA(cudaMemcpyAsync(A[b], h[b], nn * sizeof(double), cudaMemcpyHostToDevice, st));
      d[b] = nrgb::SyevDesc{n[b], A[b], W[b], Z[b]};
    }
    for (int o = 0; o < nops; ++o) {
      const size_t nn = (size_t)n[bra[o]] * n[ket[o]];
      O[o] = ctx->io.alloc_n<double>(nn);
      R[o] = ctx->io.alloc_n<double>(nn);
      if (nn) NRGB_CUDA(cudaMemcpyAsync(O[o], op[o], nn * sizeof(double), cudaMemcpyHostToDevice, st));
    }
    solver_of(ctx)->solve(d, st);
    ctx->scratch.reserve(recalc_scratch(nops, n, bra, ket));
    ctx->scratch.reset();
    recalc_pairs(ctx, nops, n, bra, ket, Z.data(), (const double* const*)O.data(), R.data(), ctx->scratch, st);
    for (int b = 0; b < nblocks; ++b) {
      if (!n[b]) continue;
      NRGB_CUDA(cudaMemcpyAsync(w[b], W[b], n[b] * sizeof(double), cudaMemcpyDeviceToHost, st));
      if (z && z[b])
        NRGB_CUDA(cudaMemcpyAsync(z[b], Z[b], (size_t)n[b] * n[b] * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    for (int o = 0; o < nops; ++o) {
      const size_t nn = (size_t)n[bra[o]] * n[ket[o]];
      if (nn) NRGB_CUDA(cudaMemcpyAsync(out[o], R[o], nn * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    NRGB_CUDA(cudaStreamSynchronize(st));
  });
}

int nrgb_profile(nrgb_ctx* ctx, int enable) {
  return guarded(ctx, [&] { nrgb::KernelStats::get().enable(enable != 0); });
}

int nrgb_profile_only(nrgb_ctx* ctx, const char* name) {
  if (!name) return 1;
  return guarded(ctx, [&] { nrgb::KernelStats::get().enable(true, name); });
}

int nrgb_kernel_stats(nrgb_ctx* ctx, const char* name, long* launches, double* ms) {
  return guarded(ctx, [&] { nrgb::KernelStats::get().query(name ? name : "*", launches, ms); });
}

int nrgb_kernel_work(nrgb_ctx* ctx, const char* name, double* units) {
  return guarded(ctx, [&] {
    const double w = nrgb::KernelStats::get().work(name ? name : "*");
    if (units) *units = w;
  });
}

int nrgb_run(nrgb_ctx* ctx, const char* workdir, const char* outdir, double* stats) {
  return guarded(ctx, [&] {
    if (!ctx->driver) ctx->driver.reset(new nrgb::NrgDriver(ctx->stream, solver_of(ctx)));
    ctx->driver->run(workdir, outdir, stats);
  });
}

int nrgb_autotune(nrgb_ctx* ctx, char* report, int report_len) {
  return guarded(ctx, [&] {
    const std::string r = nrgb::autotune(*ctx->syev, ctx->syev->cluster_capacity(), ctx->stream);
    if (report && report_len > 0) {
      const size_t n = std::min((size_t)report_len - 1, r.size());
      memcpy(report, r.data(), n);
      report[n] = 0;
    }
  });
}

int nrgb_set_schedule(nrgb_ctx* ctx, int cluster_limit, int gemm_large_from) {
  if (cluster_limit < 0 || gemm_large_from < 0) return 1;
  return guarded(ctx, [&] {
    nrgb::Schedule& s = nrgb::schedule_of(ctx->device);
    s.cluster_limit.store(cluster_limit);
    s.gemm_large_from.store(gemm_large_from);
  });
}

int nrgb_get_schedule(nrgb_ctx* ctx, int* cluster_limit, int* gemm_large_from, int* cluster_capacity) {
  return guarded(ctx, [&] {
    const nrgb::Schedule& s = nrgb::schedule_of(ctx->device);
    if (cluster_limit) *cluster_limit = s.cluster_limit.load();
    if (gemm_large_from) *gemm_large_from = s.gemm_large_from.load();
    if (cluster_capacity) *cluster_capacity = ctx->syev->cluster_capacity();
  });
}

int nrgb_set_wait_limit(nrgb_ctx* ctx, int poll_log2) {
  if (poll_log2 < 4 || poll_log2 > 30) return 1;
  return guarded(ctx, [&] { ctx->syev->set_wait_limit(poll_log2); });
}

int nrgb_inject_barrier_shortfall(nrgb_ctx* ctx, int on) {
  return guarded(ctx, [&] { ctx->syev->inject_barrier_shortfall(on != 0); });
}

int nrgb_set_eig_mode(nrgb_ctx* ctx, int mode) {
  if (mode != 0 && mode != 1) return 1;
  return guarded(ctx, [&] {
    ctx->eig_mode = mode;
    ctx->driver.reset();  // rebuilt with the chosen solver by the next nrgb_run
  });
}

}  // extern "C"
