// Grouped, segmented-K FP64 GEMM on the DMMA tensor-core path (sm_100a).
// See gemm_f64.cuh for the contract.
//
// Tile: 64x64 per CTA, 4 warps of 32x32, K staged 16 at a time through
// shared memory laid out so that the DMMA fragment loads are bank-conflict
// free: by default a cp.async ring of three K steps of 16
// (gemm_grouped_pipe_kernel<3, 16>), else
// register-staged double buffering (gemm_grouped_kernel; also the kernel of
// the allocation-free entry point) or 128x128 tiles where the schedule picks
// them.  mma.sync.m8n8k4.f64 (the m16n8k4/k8/k16 f64 shapes run at the same
// rate on B200): A fragment A[g][t], B fragment B[t][g], accumulator
// C[g][2t..2t+1] with g = lane/4, t = lane%4.
#include <atomic>
#include "common.cuh"
#include "gemm_f64.cuh"
#include "schedule.cuh"

namespace nrgb {

namespace {

constexpr int BM = GEMM_BM, BN = GEMM_BN, BK = GEMM_BK;
constexpr int PAD = 4;          // row stride 68 doubles: t*68+g hits 16 distinct bank pairs
constexpr int LDS = BM + PAD;   // BM == BN
constexpr int NT = 128;

__device__ __forceinline__ void dmma(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

struct TileLoader {
  // 8 A values and 8 B values per thread per K-tile.
  double ra[8], rb[8];

  __device__ __forceinline__ void load(const GemmSeg& s, int k0, int row0, int col0, int m, int n,
                                       int tid) {
    const double alpha = s.alpha;
    if (!s.transA) {  // A[i + p*lda], contiguous in i
      const int i = tid & 63, pb = tid >> 6;
      const int gi = row0 + i;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int p = pb + 2 * r, gp = k0 + p;
        ra[r] = (gi < m && gp < s.k) ? alpha * __ldg(s.A + (size_t)gp * s.lda + gi) : 0.0;
      }
    } else {  // op(A)[i,p] = A[p + i*lda], contiguous in p
      const int p = tid & 15, ib = tid >> 4;
      const int gp = k0 + p;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int gi = row0 + ib + 8 * r;
        ra[r] = (gi < m && gp < s.k) ? alpha * __ldg(s.A + (size_t)gi * s.lda + gp) : 0.0;
      }
    }
    if (!s.transB) {  // op(B)[p,j] = B[p + j*ldb], contiguous in p
      const int p = tid & 15, jb = tid >> 4;
      const int gp = k0 + p;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int gj = col0 + jb + 8 * r;
        rb[r] = (gj < n && gp < s.k) ? __ldg(s.B + (size_t)gj * s.ldb + gp) : 0.0;
      }
    } else {  // op(B)[p,j] = B[j + p*ldb], contiguous in j
      const int j = tid & 63, pb = tid >> 6;
      const int gj = col0 + j;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int p = pb + 2 * r, gp = k0 + p;
        rb[r] = (gj < n && gp < s.k) ? __ldg(s.B + (size_t)gp * s.ldb + gj) : 0.0;
      }
    }
  }

  __device__ __forceinline__ void store(const GemmSeg& s, double (*As)[LDS], double (*Bs)[LDS],
                                        int tid) {
    if (!s.transA) {
      const int i = tid & 63, pb = tid >> 6;
#pragma unroll
      for (int r = 0; r < 8; ++r) As[pb + 2 * r][i] = ra[r];
    } else {
      const int p = tid & 15, ib = tid >> 4;
#pragma unroll
      for (int r = 0; r < 8; ++r) As[p][ib + 8 * r] = ra[r];
    }
    if (!s.transB) {
      const int p = tid & 15, jb = tid >> 4;
#pragma unroll
      for (int r = 0; r < 8; ++r) Bs[p][jb + 8 * r] = rb[r];
    } else {
      const int j = tid & 63, pb = tid >> 6;
#pragma unroll
      for (int r = 0; r < 8; ++r) Bs[pb + 2 * r][j] = rb[r];
    }
  }
};

__global__ void __launch_bounds__(NT) gemm_grouped_kernel(const GemmProb* __restrict__ probs,
                                                          int nprob,
                                                          const GemmSeg* __restrict__ segs) {
  __shared__ __align__(16) double As[2][BK][LDS];
  __shared__ __align__(16) double Bs[2][BK][LDS];

  // Locate the problem owning this tile (probs sorted by tile0).
  const int tile = blockIdx.x;
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (probs[mid].tile0 <= tile) lo = mid; else hi = mid - 1;
  }
  const GemmProb P = probs[lo];
  const int ks = P.ksplit > 1 ? P.ksplit : 1;
  const int t = (tile - P.tile0) / ks;
  const int kc = (tile - P.tile0) % ks;
  const int row0 = (t / P.tiles_n) * BM;
  const int col0 = (t % P.tiles_n) * BN;
  const int m = P.m, n = P.n;
  if (row0 >= m || col0 >= n) return;  // shapes may be set on the device below the planned bound

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tq = lane & 3;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  // Flattened (segment, k-tile) iteration over this CTA's share of the K tiles.
  const int send = P.seg0 + P.nseg;
  int ktot = 0;
  for (int q = P.seg0; q < send; ++q) ktot += segs[q].k > 0 ? (segs[q].k + BK - 1) / BK : 0;
  const int per = (ktot + ks - 1) / ks;
  const int kt0 = kc * per;
  int remaining = min(ktot, kt0 + per) - kt0;
  int s = P.seg0, k0 = 0;
  {
    int kt = 0;
    while (s < send) {
      const int nt = segs[s].k > 0 ? (segs[s].k + BK - 1) / BK : 0;
      if (kt + nt > kt0) break;
      kt += nt;
      ++s;
    }
    k0 = (kt0 - kt) * BK;
  }
  if (remaining > 0 && s < send) {
    TileLoader L;
    GemmSeg cur = segs[s];
    L.load(cur, k0, row0, col0, m, n, tid);
    L.store(cur, As[0], Bs[0], tid);
    __syncthreads();
    int buf = 0;
    while (true) {
      --remaining;
      // advance to next (segment, k0)
      GemmSeg nxt = cur;
      int nk0 = k0 + BK;
      int ns = s;
      bool more = remaining > 0;
      if (more && nk0 >= cur.k) {
        ns = s + 1;
        while (ns < send && segs[ns].k <= 0) ++ns;
        if (ns < send) {
          nxt = segs[ns];
          nk0 = 0;
        } else {
          more = false;
        }
      }
      if (more) L.load(nxt, nk0, row0, col0, m, n, tid);

#pragma unroll
      for (int kk = 0; kk < BK; kk += 4) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[buf][kk + tq][wm + i * 8 + g];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Bs[buf][kk + tq][wn + j * 8 + g];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
      }
      if (!more) break;
      L.store(nxt, As[buf ^ 1], Bs[buf ^ 1], tid);
      __syncthreads();
      buf ^= 1;
      cur = nxt;
      s = ns;
      k0 = nk0;
    }
  }

  // Epilogue: C = acc + beta*C.
  const double beta = P.beta;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = row0 + wm + i * 8 + g;
    if (r >= m) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c = col0 + wn + j * 8 + 2 * tq + h;
        if (c < n) {
          double* dst = P.C + (size_t)c * P.ldc + r;
          const double v = acc[i][j][h];
          if (ks > 1) atomicAdd(dst, v);
          else *dst = (beta == 0.0) ? v : v + beta * (*dst);
        }
      }
    }
  }
}


// ---------------------------------------------------------------------------
// Large-tile variant: 128x128 per CTA, 8 warps of 64x32, K staged 16 at a
// time through a 3-stage cp.async pipeline (8-byte copies with zero fill at
// the edges, so no register staging); the segment's alpha scales the A
// fragments after the shared-memory load.
// ---------------------------------------------------------------------------
constexpr int LBM = 128, LBN = 128, LSTAGES = 3, LNT = 256;
constexpr int LLDS = LBM + 4;  // 132: t*132+g -> distinct bank pairs

__device__ __forceinline__ void cp_async8(double* smem, const double* gmem, bool pred) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = pred ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N)); }

__global__ void __launch_bounds__(LNT) gemm_grouped_large_kernel(const GemmProb* __restrict__ probs,
                                                                 int nprob,
                                                                 const GemmSeg* __restrict__ segs) {
  extern __shared__ __align__(16) double lsm[];
  double* As = lsm;                               // [LSTAGES][BK][LLDS]
  double* Bs = lsm + LSTAGES * BK * LLDS;         // [LSTAGES][BK][LLDS]
  __shared__ double salpha[LSTAGES];
  const int tile = blockIdx.x;
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (probs[mid].stile0 <= tile) lo = mid; else hi = mid - 1;
  }
  const GemmProb P = probs[lo];
  const int ks = P.ksplit > 1 ? P.ksplit : 1;
  const int t = (tile - P.stile0) / ks;
  const int kc = (tile - P.stile0) % ks;
  const int row0 = (t / P.stiles_n) * LBM;
  const int col0 = (t % P.stiles_n) * LBN;
  const int m = P.m, n = P.n;
  if (row0 >= m || col0 >= n) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tq = lane & 3;
  const int wm = (warp & 1) * 64, wn = (warp >> 1) * 32;

  double acc[8][4][2];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  const int send = P.seg0 + P.nseg;
  int ktot = 0;
  for (int q = P.seg0; q < send; ++q) ktot += segs[q].k > 0 ? (segs[q].k + BK - 1) / BK : 0;
  const int per = (ktot + ks - 1) / ks;
  const int kt0 = kc * per;
  const int nk = max(0, min(ktot, kt0 + per) - kt0);
  // load cursor
  int ls = P.seg0, lk0 = 0;
  {
    int kt = 0;
    while (ls < send) {
      const int nt = segs[ls].k > 0 ? (segs[ls].k + BK - 1) / BK : 0;
      if (kt + nt > kt0) break;
      kt += nt;
      ++ls;
    }
    lk0 = (kt0 - kt) * BK;
  }
  auto issue = [&](int stage) {
    const GemmSeg S = segs[ls];
    double* as = As + stage * BK * LLDS;
    double* bs = Bs + stage * BK * LLDS;
    if (!S.transA) {
      const int i = tid & 127, pb = tid >> 7;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int p = pb + 2 * r, gi = row0 + i, gp = lk0 + p;
        const bool ok = gi < m && gp < S.k;
        cp_async8(&as[p * LLDS + i], ok ? S.A + (size_t)gp * S.lda + gi : S.A, ok);
      }
    } else {
      const int p = tid & 15, ib = tid >> 4;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int i = ib + 16 * r, gi = row0 + i, gp = lk0 + p;
        const bool ok = gi < m && gp < S.k;
        cp_async8(&as[p * LLDS + i], ok ? S.A + (size_t)gi * S.lda + gp : S.A, ok);
      }
    }
    if (!S.transB) {
      const int p = tid & 15, jb = tid >> 4;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int j = jb + 16 * r, gj = col0 + j, gp = lk0 + p;
        const bool ok = gj < n && gp < S.k;
        cp_async8(&bs[p * LLDS + j], ok ? S.B + (size_t)gj * S.ldb + gp : S.B, ok);
      }
    } else {
      const int j = tid & 127, pb = tid >> 7;
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int p = pb + 2 * r, gj = col0 + j, gp = lk0 + p;
        const bool ok = gj < n && gp < S.k;
        cp_async8(&bs[p * LLDS + j], ok ? S.B + (size_t)gp * S.ldb + gj : S.B, ok);
      }
    }
    if (tid == 0) salpha[stage] = S.alpha;
    // advance the cursor
    lk0 += BK;
    if (lk0 >= S.k) {
      ++ls;
      while (ls < send && segs[ls].k <= 0) ++ls;
      lk0 = 0;
    }
  };
  // prologue
#pragma unroll
  for (int st = 0; st < LSTAGES - 1; ++st) {
    if (st < nk) issue(st);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<LSTAGES - 2>();
    __syncthreads();
    const int nxt = kt + LSTAGES - 1;
    if (nxt < nk) issue(nxt % LSTAGES);
    cp_async_commit();
    const int stg = kt % LSTAGES;
    const double* as = As + stg * BK * LLDS;
    const double* bs = Bs + stg * BK * LLDS;
    const double alpha = salpha[stg];
#pragma unroll
    for (int kk = 0; kk < BK; kk += 4) {
      double a[8], b[4];
#pragma unroll
      for (int i = 0; i < 8; ++i) a[i] = alpha * as[(kk + tq) * LLDS + wm + i * 8 + g];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = bs[(kk + tq) * LLDS + wn + j * 8 + g];
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
  }
  cp_async_wait<0>();
  const double beta = P.beta;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = row0 + wm + i * 8 + g;
    if (r >= m) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c = col0 + wn + j * 8 + 2 * tq + h;
        if (c < n) {
          double* dst = P.C + (size_t)c * P.ldc + r;
          const double v = acc[i][j][h];
          if (ks > 1) atomicAdd(dst, v);
          else *dst = (beta == 0.0) ? v : v + beta * (*dst);
        }
      }
    }
  }
}

constexpr size_t LSMEM = 2 * (size_t)LSTAGES * BK * LLDS * sizeof(double);

// ---------------------------------------------------------------------------
// Pipelined variant: the same 64x64 tile and 4 warps of 32x32, with the
// operands copied by cp.async into an S-stage ring of K steps of KB (no
// register staging, S-1 K tiles in flight).  Each operand tile keeps the direction in
// which it is contiguous in global memory:
//   mn-contiguous (A as stored, B transposed): [KB][64 + 4]
//   k-contiguous  (A transposed, B as stored): [64][KB], the 16-byte pairs of
//     row r at pair index (p/2) ^ (2r mod 8)
// and both are read bank-conflict free by the fragment loads (within a
// half-warp, lanes g, t hit double offsets 4t + g, resp. 2((k/2 + t/2) ^ 2g)
// + t%2, mod 16, all distinct).  A segment whose base address
// and leading dimension are 16-byte aligned is copied in element pairs
// (16-byte cp.async; the half of a pair outside the matrix is zero-filled),
// any other segment element by element.
// ---------------------------------------------------------------------------
constexpr int PLD_MN = BM + 4;        // 68

// doubles per operand tile of K step KB: KB * 68 >= 64 * KB
template <int KB>
__host__ __device__ constexpr int ptile() { return KB * PLD_MN; }

// offset of element (row r, K index p) in a k-contiguous tile of K step KB
template <int KB>
__device__ __forceinline__ int pipe_kofs(int r, int p) {
  return r * KB + (((p >> 1) ^ ((2 * r) & 7)) << 1) + (p & 1);
}

__device__ __forceinline__ void cp_async16(double* smem, const double* gmem, int bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes));
}

// Copy one 64 x KB operand tile: rows mn0 .. mn0+63 (< mnlim) and K columns
// k0 .. k0+KB-1 (< klim) of a matrix whose element (mn, k) sits at
// base[mn + k*ld] (mn-contiguous) or base[k + mn*ld] (k-contiguous).
template <int KB>
__device__ __forceinline__ void pipe_load_tile(double* dst, const double* base, int ld, bool kcontig,
                                               bool vec, int mn0, int mnlim, int k0, int klim, int tid) {
  if (!kcontig) {
    if (vec) {
#pragma unroll
      for (int r = 0; r < KB / 4; ++r) {
        const int c = tid + NT * r, p = c >> 5, i = 2 * (c & 31);
        const int gi = mn0 + i, gp = k0 + p;
        const int bytes = gp < klim ? (gi + 1 < mnlim ? 16 : (gi < mnlim ? 8 : 0)) : 0;
        cp_async16(dst + p * PLD_MN + i, bytes ? base + (size_t)gp * ld + gi : base, bytes);
      }
    } else {
#pragma unroll
      for (int r = 0; r < KB / 2; ++r) {
        const int e = tid + NT * r, p = e >> 6, i = e & 63;
        const int gi = mn0 + i, gp = k0 + p;
        const bool ok = gi < mnlim && gp < klim;
        cp_async8(dst + p * PLD_MN + i, ok ? base + (size_t)gp * ld + gi : base, ok);
      }
    }
  } else {
    if (vec) {
#pragma unroll
      for (int r = 0; r < KB / 4; ++r) {
        const int c = tid + NT * r, i = c / (KB / 2), p = 2 * (c % (KB / 2));
        const int gi = mn0 + i, gp = k0 + p;
        const int bytes = gi < mnlim ? (gp + 1 < klim ? 16 : (gp < klim ? 8 : 0)) : 0;
        cp_async16(dst + pipe_kofs<KB>(i, p), bytes ? base + (size_t)gi * ld + gp : base, bytes);
      }
    } else {
#pragma unroll
      for (int r = 0; r < KB / 2; ++r) {
        const int e = tid + NT * r, i = e / KB, p = e % KB;
        const int gi = mn0 + i, gp = k0 + p;
        const bool ok = gi < mnlim && gp < klim;
        cp_async8(dst + pipe_kofs<KB>(i, p), ok ? base + (size_t)gi * ld + gp : base, ok);
      }
    }
  }
}

__device__ __forceinline__ bool pipe_vec_ok(const double* p, int ld) {
  return ((reinterpret_cast<uintptr_t>(p) & 15) == 0) && ((ld & 1) == 0);
}

// 128 registers at most, so that shared memory alone sets the CTAs per SM:
// four with KB = 16 and 3 stages (52 KB each), three with KB = 32 and 2
// stages (70 KB each)
template <int S, int KB>
__global__ void __launch_bounds__(NT, 4) gemm_grouped_pipe_kernel(const GemmProb* __restrict__ probs,
                                                               int nprob,
                                                               const GemmSeg* __restrict__ segs) {
  extern __shared__ __align__(16) double psm[];
  constexpr int PTILE = ptile<KB>();
  double* As = psm;                  // [S][PTILE]
  double* Bs = psm + S * PTILE;      // [S][PTILE]
  __shared__ double salpha[S];
  __shared__ int sflags[S];          // bit 0: A k-contiguous, bit 1: B k-contiguous

  const int tile = blockIdx.x;
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (probs[mid].tile0 <= tile) lo = mid; else hi = mid - 1;
  }
  const GemmProb P = probs[lo];
  const int ks = P.ksplit > 1 ? P.ksplit : 1;
  const int t = (tile - P.tile0) / ks;
  const int kc = (tile - P.tile0) % ks;
  const int row0 = (t / P.tiles_n) * BM;
  const int col0 = (t % P.tiles_n) * BN;
  const int m = P.m, n = P.n;
  if (row0 >= m || col0 >= n) return;  // shapes may be set on the device below the planned bound

  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tq = lane & 3;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;

  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

  // this CTA's share of the flattened (segment, K tile) sequence
  const int send = P.seg0 + P.nseg;
  int ktot = 0;
  for (int q = P.seg0; q < send; ++q) ktot += segs[q].k > 0 ? (segs[q].k + KB - 1) / KB : 0;
  const int per = (ktot + ks - 1) / ks;
  const int kt0 = kc * per;
  const int nk = max(0, min(ktot, kt0 + per) - kt0);
  int ls = P.seg0, lk0 = 0;
  {
    int kt = 0;
    while (ls < send) {
      const int nt = segs[ls].k > 0 ? (segs[ls].k + KB - 1) / KB : 0;
      if (kt + nt > kt0) break;
      kt += nt;
      ++ls;
    }
    lk0 = (kt0 - kt) * KB;
  }
  auto issue = [&](int stage) {
    const GemmSeg G = segs[ls];
    // op(A)[i, p]: A[i + p*lda] as stored, A[p + i*lda] transposed
    pipe_load_tile<KB>(As + stage * PTILE, G.A, G.lda, G.transA != 0, pipe_vec_ok(G.A, G.lda), row0, m, lk0, G.k,
                   tid);
    // op(B)[p, j]: B[p + j*ldb] as stored (k-contiguous), B[j + p*ldb] transposed
    pipe_load_tile<KB>(Bs + stage * PTILE, G.B, G.ldb, G.transB == 0, pipe_vec_ok(G.B, G.ldb), col0, n, lk0, G.k,
                   tid);
    if (tid == 0) {
      salpha[stage] = G.alpha;
      sflags[stage] = (G.transA != 0 ? 1 : 0) | (G.transB == 0 ? 2 : 0);
    }
    lk0 += KB;
    if (lk0 >= G.k) {
      ++ls;
      while (ls < send && segs[ls].k <= 0) ++ls;
      lk0 = 0;
    }
  };
#pragma unroll
  for (int st = 0; st < S - 1; ++st) {
    if (st < nk) issue(st);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    cp_async_wait<S - 2>();
    __syncthreads();
    const int nxt = kt + S - 1;
    if (nxt < nk) issue(nxt % S);
    cp_async_commit();
    const int stg = kt % S;
    const double* as = As + stg * PTILE;
    const double* bs = Bs + stg * PTILE;
    const double alpha = salpha[stg];
    const int fl = sflags[stg];
#pragma unroll
    for (int kk = 0; kk < KB; kk += 4) {
      double a[4], b[4];
      if (fl & 1) {
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = as[pipe_kofs<KB>(wm + i * 8 + g, kk + tq)];
      } else {
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = as[(kk + tq) * PLD_MN + wm + i * 8 + g];
      }
      if (fl & 2) {
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = bs[pipe_kofs<KB>(wn + j * 8 + g, kk + tq)];
      } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = bs[(kk + tq) * PLD_MN + wn + j * 8 + g];
      }
      if (alpha != 1.0) {
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] *= alpha;
      }
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
  }
  cp_async_wait<0>();

  const double beta = P.beta;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = row0 + wm + i * 8 + g;
    if (r >= m) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c = col0 + wn + j * 8 + 2 * tq + h;
        if (c < n) {
          double* dst = P.C + (size_t)c * P.ldc + r;
          const double v = acc[i][j][h];
          if (ks > 1) atomicAdd(dst, v);
          else *dst = (beta == 0.0) ? v : v + beta * (*dst);
        }
      }
    }
  }
}

template <int S, int KB>
constexpr size_t pipe_smem() { return 2 * (size_t)S * ptile<KB>() * sizeof(double); }

// Form of the grouped GEMM: the pipelined kernel with K step 16 and 3 stages
// by default (3).  Measured on B200: 28.0-29.2 TF/s on grouped 2048^3
// problems and 20.5-20.9 TF/s on 256^3 ones, over the four transpose
// combinations, against 24.8-28.2 and 14.5-19.0 TF/s for the register-staged
// kernel; over the eigensolver's own launches of a 12-block step (trailing
// updates, merges, back-transforms, basis changes) 4 % less GEMM time than
// either the register-staged kernel or K step 32 with 2 stages.  That last
// form (232) is 3 % faster on large square problems but up to 50 % slower on
// launches with short K.  NRGB_GEMM_PIPE selects another form: 4 (K step 16,
// 4 stages), 232, 332 (K step 32, 2 or 3 stages) or 0 (register-staged);
// read once per process.
int gemm_pipe_stages() {
  static const int s = [] {
    const char* e = getenv("NRGB_GEMM_PIPE");
    if (!e || !*e) return 3;
    const int v = atoi(e);
    return (v == 0 || v == 3 || v == 4 || v == 232 || v == 332) ? v : 3;
  }();
  return s;
}

template <int S, int KB>
cudaError_t pipe_launch(const GemmProb* d_probs, int nprob, const GemmSeg* d_segs, int total_tiles,
                        cudaStream_t stream, const char* tag) {
  static std::atomic<bool> attr[64];
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 64 || !attr[dev].load(std::memory_order_acquire)) {
    const cudaError_t e = cudaFuncSetAttribute(gemm_grouped_pipe_kernel<S, KB>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pipe_smem<S, KB>());
    if (e != cudaSuccess) return e;
    if (dev < 64) attr[dev].store(true, std::memory_order_release);
  }
  NRGB_LAUNCH(tag, stream,
              gemm_grouped_pipe_kernel<S, KB><<<total_tiles, NT, pipe_smem<S, KB>(), stream>>>(d_probs, nprob, d_segs));
  return cudaGetLastError();
}
// The 128x128 cp.async variant is used only where the device's schedule
// (schedule.cuh, set by the autotuner's measurements) says it wins: by
// default never (measured on B200 at first: 21-25 TF/s against 25-28 TF/s
// for the 64x64 register-staged kernel on the same shapes).

}  // namespace

void gemm_assign_tiles(GemmProb& p, int& tiles, int& stiles) {
  const int ks = p.ksplit > 1 ? p.ksplit : 1;
  p.tile0 = tiles;
  p.tiles_n = (p.n + GEMM_BN - 1) / GEMM_BN;
  tiles += ((p.m + GEMM_BM - 1) / GEMM_BM) * p.tiles_n * ks;
  p.stile0 = stiles;
  p.stiles_n = (p.n + LBN - 1) / LBN;
  stiles += ((p.m + LBM - 1) / LBM) * p.stiles_n * ks;
}

double gemm_flops(const GemmProb* probs, int nprob, const GemmSeg* segs) {
  double f = 0;
  for (int p = 0; p < nprob; ++p)
    for (int s = probs[p].seg0; s < probs[p].seg0 + probs[p].nseg; ++s)
      f += 2.0 * probs[p].m * (double)probs[p].n * segs[s].k;
  return f;
}

cudaError_t gemm_grouped_launch(const GemmProb* d_probs, int nprob, const GemmSeg* d_segs,
                                int total_tiles, cudaStream_t stream, const char* tag, int total_stiles) {
  if (total_tiles <= 0 || nprob <= 0) return cudaSuccess;
  // 128x128 tiles when the schedule selects them for this problem size,
  // they cover at most 30% more area than the 64x64 ones and they still give
  // enough CTAs to fill the GPU
  const int large_from = schedule_here().gemm_large_from.load(std::memory_order_relaxed);
  const double edge = GEMM_BM * sqrt((double)total_tiles / nprob);  // mean output edge per problem
  if (large_from > 0 && edge >= large_from && total_stiles > 0 && 4.0 * total_stiles <= 1.3 * total_tiles &&
      total_stiles >= 120) {
    // once per device (function attributes belong to the device's context);
    // every caller sets the same value, so threads that race here agree
    static std::atomic<bool> attr[64];
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 64 || !attr[dev].load(std::memory_order_acquire)) {
      const cudaError_t e =
          cudaFuncSetAttribute(gemm_grouped_large_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LSMEM);
      if (e != cudaSuccess) return e;
      if (dev < 64) attr[dev].store(true, std::memory_order_release);
    }
    NRGB_LAUNCH(tag, stream,
                gemm_grouped_large_kernel<<<total_stiles, LNT, LSMEM, stream>>>(d_probs, nprob, d_segs));
    return cudaGetLastError();
  }
  const int stages = gemm_pipe_stages();
  if (stages == 3) return pipe_launch<3, 16>(d_probs, nprob, d_segs, total_tiles, stream, tag);
  if (stages == 4) return pipe_launch<4, 16>(d_probs, nprob, d_segs, total_tiles, stream, tag);
  if (stages == 232) return pipe_launch<2, 32>(d_probs, nprob, d_segs, total_tiles, stream, tag);
  if (stages == 332) return pipe_launch<3, 32>(d_probs, nprob, d_segs, total_tiles, stream, tag);
  NRGB_LAUNCH(tag, stream, gemm_grouped_kernel<<<total_tiles, NT, 0, stream>>>(d_probs, nprob, d_segs));
  return cudaGetLastError();
}

cudaError_t gemm_grouped_launch_unaccounted(const GemmProb* d_probs, int nprob, const GemmSeg* d_segs,
                                            int total_tiles, cudaStream_t stream) {
  if (total_tiles <= 0 || nprob <= 0) return cudaSuccess;
  gemm_grouped_kernel<<<total_tiles, NT, 0, stream>>>(d_probs, nprob, d_segs);
  return cudaGetLastError();
}

}  // namespace nrgb
