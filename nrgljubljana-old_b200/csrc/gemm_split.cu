// Split-precision grouped GEMM on the 5th-generation tensor cores of
// sm_100a (tcgen05.mma kind::i8 with INT32 accumulators in tensor memory,
// operands staged in shared memory by bulk asynchronous copies); see
// gemm_split.cuh for the arithmetic.
//
// Operand packing.  A slicing pass writes every operand as ready-made
// shared-memory images: op(A) in tiles of 128 rows x 64 K-bytes, op(B)^T in
// tiles of 64 rows x 64 K-bytes, each in the canonical K-major layout
// without swizzle (core matrices of 8 rows x 16 bytes; consecutive core
// matrices along K 128 bytes apart, along the rows 512 bytes apart).  The S
// slices of one (row tile, K chunk) follow each other, so one stage of the
// GEMM is two contiguous bulk copies: S x 8 KB of A and S x 4 KB of B.
//
// GEMM kernel.  One CTA (4 warps) per 128 x 64 output tile of a problem.
// Warp 1 lane 0 issues the bulk copies into a two-stage ring
// (cp.async.bulk with mbarrier transaction counts); warp 0 lane 0 issues
// the tcgen05.mma instructions: for every chunk, the slice pairs (p, q) with
// p + q <= S + 1, two K = 32 instructions each, into the accumulator of
// p + q (S accumulators of 64 INT32 columns: up to 512 tensor-memory
// columns), and commits to the stage's "empty" barrier.  After a segment's
// last chunk a commit to the "done" barrier releases the epilogue: each warp
// reads its 32 rows (tensor-memory lanes) with tcgen05.ld, recombines the
// accumulators in FP64 and adds alpha times the result into C.  Every wait
// on a barrier is bounded; a wait that gives up sets an error flag, ends
// the CTA's work (waiting, bounded, for its copies in flight), frees the
// tensor memory and returns.
#include "gemm_split.cuh"

#include <math.h>
#include <string.h>

#include <algorithm>

namespace nrgb {

namespace {

constexpr int SBM = 128;              // output rows per CTA (tensor-memory lanes)
constexpr int SBN = 64;               // output columns per CTA
constexpr int SBK = 64;               // K bytes per stage
constexpr int A_TILE = SBM * SBK;     // 8 KB
constexpr int B_TILE = SBN * SBK;     // 4 KB
constexpr int SPLIT_NT = 128;
constexpr long long WAIT_LIMIT = 1ll << 24;

__device__ int g_split_err = 0;

struct SliceJob {
  const double* X;   // X(r, l) = X[r * rs + l * ls], r < rows, l < K
  long long rs, ls;
  int rows, K;
  int tile_rows;     // 128 (A) or 64 (B)
  int kch;           // K chunks of 64
  int tile0;         // first row tile of this job in the launch
  signed char* out;  // packed slices: [row tile][K chunk][slice] images
  int* exps;         // tile rows of exponents (rows past `rows`: 0)
};

struct SplitSeg {
  const signed char* A;  // packed op(A)
  const signed char* B;  // packed op(B)^T
  const int* eA;         // row exponents of op(A)
  const int* eB;         // column exponents of op(B)
  int kch;
  double alpha;
};

struct SplitProb {
  double* C;
  int ldc, m, n;
  double beta;
  int seg0, nseg;
  int tile0, tiles_n, tiles_m;
};

// ------------------------------------------------------------------ slicing
__device__ __forceinline__ int find_job(const SliceJob* jobs, int njobs, int t) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].tile0 <= t) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Row exponents: E_r with max_l |X(r, l)| < 2^E_r (0 for a zero row).
__global__ void __launch_bounds__(SPLIT_NT) split_exp_kernel(const SliceJob* __restrict__ jobs, int njobs) {
  const SliceJob J = jobs[find_job(jobs, njobs, blockIdx.x)];
  const int t = blockIdx.x - J.tile0;
  const int r0 = t * J.tile_rows;
  if (J.rs == 1) {
    // consecutive rows are adjacent: one thread per row, coalesced over rows
    for (int rr = threadIdx.x; rr < J.tile_rows; rr += blockDim.x) {
      const int r = r0 + rr;
      double mx = 0.0;
      if (r < J.rows)
        for (int l = 0; l < J.K; ++l) mx = fmax(mx, fabs(J.X[(long long)r + l * J.ls]));
      int e = 0;
      if (mx > 0.0) frexp(mx, &e);
      J.exps[r0 + rr] = e;
    }
  } else {
    // the K entries of a row are adjacent: one warp per row
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int rr = warp; rr < J.tile_rows; rr += blockDim.x >> 5) {
      const int r = r0 + rr;
      double mx = 0.0;
      if (r < J.rows)
        for (int l = lane; l < J.K; l += 32) mx = fmax(mx, fabs(J.X[(long long)r * J.rs + (long long)l * J.ls]));
      for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      int e = 0;
      if (mx > 0.0) frexp(mx, &e);
      if (lane == 0) J.exps[r0 + rr] = e;
    }
  }
}

// Digits: one item = 16 consecutive K entries of one row, written as 16
// bytes into each of the S slice images of its (row tile, K chunk).
__global__ void __launch_bounds__(SPLIT_NT) split_digits_kernel(const SliceJob* __restrict__ jobs, int njobs,
                                                                 int slices) {
  // blockIdx.x enumerates (row tile, K chunk) pairs: tile0 counts row tiles
  // times K chunks here
  const SliceJob J = jobs[find_job(jobs, njobs, blockIdx.x)];
  const int local = blockIdx.x - J.tile0;
  const int t = local / J.kch, kc = local % J.kch;
  const int R = J.tile_rows;
  const int items = R * (SBK / 16);
  const size_t tile_bytes = (size_t)R * SBK;
  signed char* base = J.out + ((size_t)t * J.kch + kc) * slices * tile_bytes;
  for (int it = threadIdx.x; it < items; it += blockDim.x) {
    int rr, g;
    if (J.rs == 1) {  // rows fastest: coalesced reads across the warp
      rr = it % R;
      g = it / R;
    } else {          // K groups fastest: each thread reads 128 contiguous bytes
      rr = it / (SBK / 16);
      g = it % (SBK / 16);
    }
    const int r = t * R + rr;
    const int l0 = kc * SBK + g * 16;
    double x[16];
    const int e = J.exps[r];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int l = l0 + u;
      double v = 0.0;
      if (r < J.rows && l < J.K) v = J.X[(long long)r * J.rs + (long long)l * J.ls];
      x[u] = ldexp(v, -e);  // |x| < 1, exact
    }
    const size_t off = (size_t)(rr >> 3) * 512 + (size_t)g * 128 + (size_t)(rr & 7) * 16;
    for (int p = 0; p < slices; ++p) {
      unsigned w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const double tt = x[u] * 128.0;  // exact
        const double d = trunc(tt);      // |d| <= 127
        x[u] = tt - d;                   // exact remainder, |x| < 1
        const unsigned byte = (unsigned)((int)d) & 0xffu;
        w[u >> 2] |= byte << (8 * (u & 3));
      }
      *reinterpret_cast<uint4*>(base + (size_t)p * tile_bytes + off) = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

// ------------------------------------------------------------ PTX wrappers
__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n"
      ".reg .pred P;\n"
      "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n"
      "selp.b32 %0, 1, 0, P;\n"
      "}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait for the phase with parity `parity` to complete.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity, volatile int* abort_flag) {
  for (long long it = 0; it < WAIT_LIMIT; ++it) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*abort_flag) return false;
  }
  return false;
}

__device__ __forceinline__ void bulk_g2s(unsigned dst, const void* src, unsigned bytes, unsigned bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(dst),
      "l"(src), "r"(bytes), "r"(bar)
      : "memory");
}

// Shared-memory matrix descriptor: canonical K-major layout, no swizzle.
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr, unsigned lbo, unsigned sbo) {
  unsigned long long d = 0;
  d |= (unsigned long long)((addr & 0x3FFFFu) >> 4);
  d |= (unsigned long long)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (unsigned long long)((sbo >> 4) & 0x3FFFu) << 32;
  d |= 1ull << 46;  // descriptor version of tcgen05
  return d;         // base offset 0, relative LBO mode, no swizzle
}

// Instruction descriptor: kind::i8, D = S32, A and B signed 8-bit, both
// K-major, M = 128, N = 64.
constexpr unsigned IDESC_I8 = (2u << 4)            // D format S32
                              | (1u << 7)          // A signed
                              | (1u << 10)         // B signed
                              | ((SBN >> 3) << 17)  // N / 8
                              | ((SBM >> 4) << 24); // M / 16

__device__ __forceinline__ void mma_i8(unsigned dtmem, unsigned long long adesc, unsigned long long bdesc,
                                       unsigned accumulate) {
  asm volatile(
      "{\n"
      ".reg .pred p;\n"
      "setp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n"
      "}\n" ::"r"(dtmem),
      "l"(adesc), "l"(bdesc), "r"(IDESC_I8), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(unsigned bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar)
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(unsigned taddr, int (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
        "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr)
      : "memory");
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
}

__device__ __forceinline__ int find_prob(const SplitProb* probs, int nprob, int b) {
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (probs[mid].tile0 <= b) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// ------------------------------------------------------------------ GEMM
__global__ void __launch_bounds__(SPLIT_NT, 1) split_gemm_kernel(const SplitProb* __restrict__ probs, int nprob,
                                                                  const SplitSeg* __restrict__ segs, int slices,
                                                                  unsigned tmem_cols) {
  extern __shared__ __align__(1024) unsigned char dsm[];
  // 1024-aligned stage buffers: [stage][A: S x 8 KB | B: S x 4 KB]
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<size_t>(dsm) + 1023) & ~size_t(1023));
  const unsigned stage_bytes = (unsigned)slices * (A_TILE + B_TILE);
  __shared__ __align__(8) unsigned long long bars[5];  // full[2], empty[2], done
  __shared__ unsigned tmem_base_s;
  __shared__ int abort_s;
  __shared__ int issued_s;  // chunks whose copies have been issued (ring position)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  const SplitProb P = probs[find_prob(probs, nprob, blockIdx.x)];
  const int local = blockIdx.x - P.tile0;
  const int mt = local / P.tiles_n, nt = local % P.tiles_n;

  if (tid == 0) {
    for (int i = 0; i < 5; ++i) mbar_init(smem_u32(&bars[i]), 1);
    abort_s = 0;
    issued_s = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const unsigned tmem = tmem_base_s;
  const unsigned full0 = smem_u32(&bars[0]), empty0 = smem_u32(&bars[2]), done = smem_u32(&bars[4]);
  volatile int* abort_flag = &abort_s;

  int g0 = 0;  // chunks issued so far in this CTA (ring position and phases)
  for (int si = 0; si < P.nseg; ++si) {
    const SplitSeg S = segs[P.seg0 + si];
    const int nk = S.kch;
    if (warp == 1 && lane == 0) {
      // producer: bulk copies of each chunk's S A images and S B images
      const signed char* a0 = S.A + (size_t)mt * nk * slices * A_TILE;
      const signed char* b0 = S.B + (size_t)nt * nk * slices * B_TILE;
      for (int c = 0; c < nk && !*abort_flag; ++c) {
        const int g = g0 + c, st = g & 1;
        if (g >= 2 && !mbar_wait(empty0 + 8 * st, ((g >> 1) - 1) & 1, abort_flag)) {
          atomicExch(&g_split_err, 1);
          *abort_flag = 1;
          break;
        }
        const unsigned dst = smem_u32(sm + (size_t)st * stage_bytes);
        mbar_expect_tx(full0 + 8 * st, stage_bytes);
        bulk_g2s(dst, a0 + (size_t)c * slices * A_TILE, (unsigned)slices * A_TILE, full0 + 8 * st);
        bulk_g2s(dst + (unsigned)slices * A_TILE, b0 + (size_t)c * slices * B_TILE, (unsigned)slices * B_TILE,
                 full0 + 8 * st);
        issued_s = g + 1;
      }
    } else if (warp == 0 && lane == 0) {
      // MMA issuer
      unsigned started = 0;  // accumulators written in this segment
      for (int c = 0; c < nk && !*abort_flag; ++c) {
        const int g = g0 + c, st = g & 1;
        if (!mbar_wait(full0 + 8 * st, (g >> 1) & 1, abort_flag)) {
          atomicExch(&g_split_err, 1);
          *abort_flag = 1;
          break;
        }
        tc_fence_after();
        const unsigned sa = smem_u32(sm + (size_t)st * stage_bytes);
        const unsigned sb = sa + (unsigned)slices * A_TILE;
        for (int p = 1; p <= slices; ++p)
          for (int q = 1; p + q <= slices + 1; ++q) {
            const int d = p + q - 2;  // accumulator index 0 .. S-1
            const unsigned dt = tmem + (unsigned)(d * SBN);
#pragma unroll
            for (int ks = 0; ks < SBK / 32; ++ks) {
              const unsigned long long ad = smem_desc(sa + (p - 1) * A_TILE + ks * 256, 128, 512);
              const unsigned long long bd = smem_desc(sb + (q - 1) * B_TILE + ks * 256, 128, 512);
              mma_i8(dt, ad, bd, (started >> d) & 1u);
              started |= 1u << d;
            }
          }
        mma_commit(empty0 + 8 * st);  // the stage is free once these MMAs have read it
      }
      mma_commit(done);  // every MMA of the segment has completed
    }
    __syncwarp();
    // epilogue: wait for the segment's MMAs, then recombine in FP64
    bool ok = mbar_wait(done, si & 1, abort_flag);
    __syncwarp();
    if (!ok) {
      if (tid == 0) atomicExch(&g_split_err, 1);
      *abort_flag = 1;
    }
    tc_fence_after();
    if (!*abort_flag) {
      const int row = mt * SBM + warp * 32 + lane;
      const int ea = (row < P.m) ? S.eA[row] : 0;
      for (int cg = 0; cg < SBN / 16; ++cg) {
        double sum[16], cmp[16];
#pragma unroll
        for (int u = 0; u < 16; ++u) sum[u] = cmp[u] = 0.0;
        for (int d = slices - 1; d >= 0; --d) {  // smallest scale first
          int v[16];
          tmem_ld16(tmem + ((unsigned)(warp * 32) << 16) + (unsigned)(d * SBN + cg * 16), v);
          const double sc = ldexp(1.0, -7 * (d + 2));
#pragma unroll
          for (int u = 0; u < 16; ++u) {
            const double t = (double)v[u] * sc;  // exact
            const double s2 = sum[u] + t;        // TwoSum
            const double bp = s2 - sum[u];
            cmp[u] += (sum[u] - (s2 - bp)) + (t - bp);
            sum[u] = s2;
          }
        }
        if (row < P.m) {
#pragma unroll
          for (int u = 0; u < 16; ++u) {
            const int col = nt * SBN + cg * 16 + u;
            if (col >= P.n) continue;
            const double val = S.alpha * ldexp(sum[u] + cmp[u], ea + S.eB[col]);
            double* cp = P.C + (size_t)col * P.ldc + row;
            double base = 0.0;
            if (si > 0) base = *cp;
            else if (P.beta != 0.0) base = P.beta * *cp;
            *cp = base + val;
          }
        }
      }
    }
    g0 += nk;
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (*abort_flag) {
      // a wait gave up: before the shared memory and the tensor memory are
      // released, let this CTA's copies in flight land and its MMAs finish
      // (both bounded; the MMA thread committed `done` after its last MMA)
      if (tid == 32) {
        const int issued = issued_s;
        for (int st = 0; st < 2; ++st) {
          int last = issued - 1;
          if (last >= 0 && (last & 1) != st) last -= 1;
          if (last < 0) continue;
          for (long long it = 0; it < WAIT_LIMIT && !mbar_try_wait(full0 + 8 * st, (last >> 1) & 1); ++it) {
          }
        }
      }
      if (tid == 0)
        for (long long it = 0; it < WAIT_LIMIT && !mbar_try_wait(done, si & 1); ++it) {
        }
      break;
    }
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(tmem_cols) : "memory");
  }
}

size_t ceil_div(size_t a, size_t b) { return (a + b - 1) / b; }

struct SegShape {
  int m, n, k;
};

}  // namespace

size_t split_gemm_workspace(const GemmProb* probs, int nprob, const GemmSeg* segs, int slices) {
  size_t b = 1 << 16;
  for (int p = 0; p < nprob; ++p)
    for (int s = 0; s < probs[p].nseg; ++s) {
      const GemmSeg& g = segs[probs[p].seg0 + s];
      for (int k0 = 0; k0 < g.k; k0 += SPLIT_MAX_K) {
        const size_t kk = std::min(SPLIT_MAX_K, g.k - k0);
        const size_t kch = ceil_div(kk, SBK);
        const size_t tm = ceil_div(probs[p].m, SBM), tn = ceil_div(probs[p].n, SBN);
        b += (size_t)slices * kch * (tm * A_TILE + tn * B_TILE) + 512;
        b += (tm * SBM + tn * SBN) * sizeof(int) + 512;
      }
      b += 2 * sizeof(SliceJob) + sizeof(SplitSeg) + 64;
    }
  b += (size_t)nprob * (sizeof(SplitProb) + 64);
  return b;
}

void split_gemm_grouped(const GemmProb* probs, int nprob, const GemmSeg* segs, int slices, DeviceArena& ws,
                        cudaStream_t st, const char* tag) {
  if (slices < SPLIT_MIN_SLICES || slices > SPLIT_MAX_SLICES)
    throw CudaError("split gemm: slices must be in [2, 8]");
  std::vector<SliceJob> jobs;
  std::vector<SplitSeg> ss;
  std::vector<SplitProb> ps;
  int exp_tiles = 0, dig_blocks = 0, tiles = 0;
  double flops = 0;
  std::vector<std::pair<int, int>> jobs_dig;  // digit-block prefix per job
  for (int p = 0; p < nprob; ++p) {
    const GemmProb& G = probs[p];
    if (G.m <= 0 || G.n <= 0) continue;
    SplitProb sp{};
    sp.C = G.C;
    sp.ldc = G.ldc;
    sp.m = G.m;
    sp.n = G.n;
    sp.beta = G.beta;
    sp.seg0 = (int)ss.size();
    sp.tiles_m = (int)ceil_div(G.m, SBM);
    sp.tiles_n = (int)ceil_div(G.n, SBN);
    for (int s = 0; s < G.nseg; ++s) {
      const GemmSeg& g = segs[G.seg0 + s];
      flops += 2.0 * G.m * G.n * g.k;
      for (int k0 = 0; k0 < g.k; k0 += SPLIT_MAX_K) {
        const int kk = std::min(SPLIT_MAX_K, g.k - k0);
        const int kch = (int)ceil_div(kk, SBK);
        // op(A)(i, l) = A[i + l lda] (as stored) or A[l + i lda] (transposed)
        SliceJob ja{};
        ja.rows = G.m;
        ja.K = kk;
        ja.rs = g.transA ? g.lda : 1;
        ja.ls = g.transA ? 1 : g.lda;
        ja.X = g.A + (size_t)k0 * ja.ls;
        ja.tile_rows = SBM;
        ja.kch = kch;
        ja.out = ws.alloc_n<signed char>((size_t)slices * kch * sp.tiles_m * A_TILE);
        ja.exps = ws.alloc_n<int>((size_t)sp.tiles_m * SBM);
        // op(B)^T(j, l) = op(B)(l, j) = B[l + j ldb] (as stored) or B[j + l ldb]
        SliceJob jb{};
        jb.rows = G.n;
        jb.K = kk;
        jb.rs = g.transB ? 1 : g.ldb;
        jb.ls = g.transB ? g.ldb : 1;
        jb.X = g.B + (size_t)k0 * jb.ls;
        jb.tile_rows = SBN;
        jb.kch = kch;
        jb.out = ws.alloc_n<signed char>((size_t)slices * kch * sp.tiles_n * B_TILE);
        jb.exps = ws.alloc_n<int>((size_t)sp.tiles_n * SBN);
        SplitSeg q{};
        q.A = ja.out;
        q.B = jb.out;
        q.eA = ja.exps;
        q.eB = jb.exps;
        q.kch = kch;
        q.alpha = g.alpha;
        ss.push_back(q);
        for (SliceJob* j : {&ja, &jb}) {
          const int t = (int)ceil_div(j->rows, j->tile_rows);
          jobs.push_back(*j);
          jobs_dig.push_back({exp_tiles, dig_blocks});
          exp_tiles += t;
          dig_blocks += t * j->kch;
        }
      }
    }
    sp.nseg = (int)ss.size() - sp.seg0;
    if (sp.nseg == 0) {
      // no inner dimension: C = beta C
      if (G.beta == 0.0) {
        for (int c = 0; c < G.n; ++c)
          NRGB_CUDA(cudaMemsetAsync(G.C + (size_t)c * G.ldc, 0, (size_t)G.m * sizeof(double), st));
        continue;
      }
      throw CudaError("split gemm: a problem without segments and beta != 0");
    }
    sp.tile0 = tiles;
    tiles += sp.tiles_m * sp.tiles_n;
    ps.push_back(sp);
  }
  if (ps.empty()) return;
  // the two slicing launches index the jobs by their own prefix counts
  std::vector<SliceJob> je = jobs, jd = jobs;
  for (size_t i = 0; i < jobs.size(); ++i) {
    je[i].tile0 = jobs_dig[i].first;
    jd[i].tile0 = jobs_dig[i].second;
  }
  SliceJob* d_je = ws.alloc_n<SliceJob>(je.size());
  SliceJob* d_jd = ws.alloc_n<SliceJob>(jd.size());
  SplitSeg* d_ss = ws.alloc_n<SplitSeg>(ss.size());
  SplitProb* d_ps = ws.alloc_n<SplitProb>(ps.size());
  NRGB_CUDA(cudaMemcpyAsync(d_je, je.data(), je.size() * sizeof(SliceJob), cudaMemcpyHostToDevice, st));
  NRGB_CUDA(cudaMemcpyAsync(d_jd, jd.data(), jd.size() * sizeof(SliceJob), cudaMemcpyHostToDevice, st));
  NRGB_CUDA(cudaMemcpyAsync(d_ss, ss.data(), ss.size() * sizeof(SplitSeg), cudaMemcpyHostToDevice, st));
  NRGB_CUDA(cudaMemcpyAsync(d_ps, ps.data(), ps.size() * sizeof(SplitProb), cudaMemcpyHostToDevice, st));
  const int nj = (int)jobs.size();
  NRGB_LAUNCH("split_slice", st, split_exp_kernel<<<exp_tiles, SPLIT_NT, 0, st>>>(d_je, nj));
  NRGB_CUDA(cudaGetLastError());
  NRGB_LAUNCH("split_slice", st, split_digits_kernel<<<dig_blocks, SPLIT_NT, 0, st>>>(d_jd, nj, slices));
  NRGB_CUDA(cudaGetLastError());
  const size_t smem = 2 * (size_t)slices * (A_TILE + B_TILE) + 1024;
  static std::once_flag attr_once;
  static cudaError_t attr_err = cudaSuccess;
  std::call_once(attr_once, [&] {
    attr_err = cudaFuncSetAttribute(split_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)(2 * (size_t)SPLIT_MAX_SLICES * (A_TILE + B_TILE) + 1024));
  });
  NRGB_CUDA(attr_err);
  unsigned cols = 32;
  while (cols < (unsigned)(slices * SBN)) cols <<= 1;
  KernelStats::get().add_work(tag, flops);
  NRGB_LAUNCH(tag, st, split_gemm_kernel<<<tiles, SPLIT_NT, smem, st>>>(d_ps, (int)ps.size(), d_ss, slices, cols));
  NRGB_CUDA(cudaGetLastError());
}

int split_gemm_take_error(cudaStream_t st) {
  int h = 0, z = 0;
  NRGB_CUDA(cudaMemcpyFromSymbolAsync(&h, g_split_err, sizeof(int), 0, cudaMemcpyDeviceToHost, st));
  NRGB_CUDA(cudaStreamSynchronize(st));
  if (h) NRGB_CUDA(cudaMemcpyToSymbolAsync(g_split_err, &z, sizeof(int), 0, cudaMemcpyHostToDevice, st));
  return h;
}

}  // namespace nrgb
