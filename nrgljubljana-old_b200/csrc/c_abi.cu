// C ABI of libnrgb.so (declarations and the reference seams they replace are
// in include/nrgb.h).
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "../../include/nrgb.h"
#include "common.cuh"
#include "gemm_f64.cuh"
#include "syev.cuh"
#include "../host/driver.h"

struct nrgb_ctx {
  int device = 0;
  std::string err;
  cudaStream_t stream = nullptr;
  std::unique_ptr<nrgb::SyevBatched> syev;
  nrgb::DeviceArena scratch;
  std::unique_ptr<nrgb::NrgDriver> driver;
};

namespace {

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

}  // namespace

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
  ctx->syev.reset();
  ctx->scratch.release();
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
    ctx->syev->run(d, st);
    for (int b = 0; b < nblocks; ++b) {
      const size_t nn = (size_t)n[b] * n[b];
      if (!nn) continue;
      NRGB_CUDA(cudaMemcpyAsync(a[b], d[b].Z, nn * sizeof(double), cudaMemcpyDeviceToHost, st));
      NRGB_CUDA(cudaMemcpyAsync(w[b], d[b].w, n[b] * sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    NRGB_CUDA(cudaStreamSynchronize(st));
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
    int tiles = 0;
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
      p.tile0 = tiles;
      p.tiles_n = (y.n + nrgb::GEMM_BN - 1) / nrgb::GEMM_BN;
      tiles += ((y.m + nrgb::GEMM_BM - 1) / nrgb::GEMM_BM) * p.tiles_n;
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
    NRGB_CUDA(nrgb::gemm_grouped_launch(dP, (int)P.size(), dS, tiles, st));
    NRGB_CUDA(cudaStreamSynchronize(st));
  });
}

int nrgb_run(nrgb_ctx* ctx, const char* workdir, const char* outdir, double* stats) {
  return guarded(ctx, [&] {
    if (!ctx->driver) ctx->driver.reset(new nrgb::NrgDriver(ctx->stream, ctx->syev.get()));
    ctx->driver->run(workdir, outdir, stats);
  });
}

}  // extern "C"
