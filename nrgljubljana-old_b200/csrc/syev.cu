// Batched FP64 symmetric eigensolver (see syev.cuh).
//
// Numerical methods (written from the published algorithms):
//  * Householder reflector H = I - tau v v^T, v(0) = 1, chosen so that
//    H x = beta e_1, beta = -sign(x_0) ||x||, tau = (beta - x_0)/beta.
//  * Blocked tridiagonalisation with the panel formulation A22 <- A22 - V W^T
//    - W V^T (Dongarra, Sorensen, Hammarling 1989).
//  * Implicit symmetric QR step with Wilkinson shift (Golub & Van Loan,
//    Matrix Computations, Alg. 8.3.2) for the leaves and the small path.
//  * Divide and conquer: Cuppen's rank-one tearing, deflation of small z_i
//    and of close d_i by Givens rotations, secular-equation roots by a
//    safeguarded two-pole rational iteration (Bunch-Nielsen-Sorensen / Li
//    "middle way" model) in coordinates relative to the nearer pole, and
//    eigenvectors from the Loewner-formula z-hat (Gu & Eisenstat 1995), which
//    keeps them orthogonal without extra precision.
#include <map>
#include <mutex>
#include <cooperative_groups.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <type_traits>

#include "gemm_f64.cuh"
#include "syev.cuh"
#include "schedule.cuh"

namespace nrgb {

namespace {

constexpr int SMALL_N = 32;     // warp-per-problem path
constexpr int LEAF = 16;        // D&C leaf size
constexpr int NB = 32;          // tridiagonalisation panel width
constexpr int NBB = 64;         // back-transformation block of reflectors
constexpr int TRD_NT = 256;     // threads of the panel kernel
constexpr int TRDC_NT = 256;    // threads of a CTA of the cluster kernel
constexpr size_t TRDC_SMEM = 227 * 1024;  // shared memory one CTA of the cluster kernel may use
constexpr int TRDC_CL_MAX = 16;           // largest cluster (non-portable above 8)
constexpr double EPS = 2.220446049250313e-16;

// --------------------------------------------------------------------------
// Small path: one warp per problem (n <= 32), everything in shared memory.
// --------------------------------------------------------------------------
struct SmallProb {
  const double* A;
  double* w;
  double* Z;
  int n;
};

constexpr int SMALL_WARPS = 2;

// Implicit symmetric QR with Wilkinson shift on tridiagonal (d, e),
// rotations accumulated into the columns of Z (Z <- Z G^T).  dn, en: 32
// doubles each of scratch (the step's new d, e).
__device__ void givens_qr_sweep_warp(double* d, double* e, double (*Z)[33], int n, int lane,
                                     double* cs, double* dn, double* en, int* fail) {
  int iter = 0;
  const int maxiter = 40 * n + 40;
  int hi = n - 1;
  while (hi > 0) {
    // lane 0 drives the sequential part; all lanes follow the same control flow
    int lo;
    if (lane == 0) {
      // deflate from the bottom
      while (hi > 0 && fabs(e[hi - 1]) <= EPS * (fabs(d[hi - 1]) + fabs(d[hi]))) {
        e[hi - 1] = 0.0;
        --hi;
      }
      lo = hi;
      while (lo > 0 && fabs(e[lo - 1]) > EPS * (fabs(d[lo - 1]) + fabs(d[lo]))) --lo;
      cs[2] = (double)hi;
      cs[3] = (double)lo;
    }
    __syncwarp();
    hi = (int)cs[2];
    lo = (int)cs[3];
    __syncwarp();
    if (hi <= 0) break;
    if (++iter > maxiter) {
      if (lane == 0) atomicExch(fail, 1);
      break;
    }
    // One implicit QR step on [lo, hi].  Every lane runs the same scalar
    // recurrence (so no lane waits for another's rotation), carrying the
    // running d[k], e[k], the bulge and the next x in registers.  The step
    // reads only d, e and stores only into dn, en (lane 0), which are copied
    // back after the step, so lanes need no synchronisation inside it.
    double a = d[lo], b = e[lo];
    double x, z = b;
    {
      const double dl = (d[hi - 1] - d[hi]) * 0.5;
      const double eh = e[hi - 1];
      const double den = dl + copysign(hypot(dl, eh), dl == 0.0 ? 1.0 : dl);
      x = a - (d[hi] - eh * eh / den);
    }
    for (int k = lo; k < hi; ++k) {
      const double dd = d[k + 1];
      const double ekn = (k + 1 < hi) ? e[k + 1] : 0.0;
      double c = 1.0, s = 0.0, r = 0.0;
      const double r2 = x * x + z * z;
      if (r2 > 0.0 && r2 < 1e300) {
        r = sqrt(r2);
        const double ri = 1.0 / r;
        c = x * ri;
        s = z * ri;
      } else if (x != 0.0 || z != 0.0) {  // squares out of range
        r = hypot(x, z);
        c = x / r;
        s = z / r;
      }
      const double cc = c * c, ss = s * s, csb = 2.0 * c * s * b;
      const double dk = cc * a + csb + ss * dd;
      const double dk1 = ss * a - csb + cc * dd;
      const double ek = c * s * (dd - a) + (cc - ss) * b;
      if (lane == 0) {
        if (k > lo) en[k - 1] = r;
        dn[k] = dk;
      }
      if (lane < n) {
        const double zk = Z[lane][k], zk1 = Z[lane][k + 1];
        Z[lane][k] = c * zk + s * zk1;
        Z[lane][k + 1] = -s * zk + c * zk1;
      }
      a = dk1;  // d[k+1]
      x = ek;   // e[k], the next rotation's x
      b = c * ekn;
      z = s * ekn;  // bulge
    }
    if (lane == 0) {
      dn[hi] = a;
      en[hi - 1] = x;
    }
    __syncwarp();
    if (lane >= lo && lane <= hi) d[lane] = dn[lane];
    if (lane >= lo && lane < hi) e[lane] = en[lane];
    __syncwarp();
  }
  __syncwarp();
}

__global__ void __launch_bounds__(32 * SMALL_WARPS) syev_small_kernel(const SmallProb* probs,
                                                                       int nprob, int* fail) {
  __shared__ double As[SMALL_WARPS][32][33];
  __shared__ double Zs[SMALL_WARPS][32][33];
  __shared__ double dv[SMALL_WARPS][32], ev[SMALL_WARPS][32], vv[SMALL_WARPS][32],
      wv[SMALL_WARPS][32], tv[SMALL_WARPS][32];
  __shared__ double csv[SMALL_WARPS][4];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int p = blockIdx.x * SMALL_WARPS + warp;
  if (p >= nprob) return;
  const SmallProb P = probs[p];
  const int n = P.n;
  double(*A)[33] = As[warp];
  double(*Z)[33] = Zs[warp];
  double *d = dv[warp], *e = ev[warp], *v = vv[warp], *w = wv[warp], *tau = tv[warp];
  for (int j = 0; j < n; ++j) A[lane][j] = (lane < n) ? P.A[lane + (size_t)j * n] : 0.0;
  __syncwarp();
  // Householder tridiagonalisation: columns c = 0 .. n-3
  for (int c = 0; c + 2 < n; ++c) {
    const double xi = (lane >= c + 2 && lane < n) ? A[lane][c] : 0.0;
    const double xn2 = warp_sum(xi * xi);
    const double alpha = A[c + 1][c];
    double tc = 0.0, beta = alpha, scal = 0.0;
    if (xn2 != 0.0) {
      beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
      tc = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
    const double vi = (lane == c + 1) ? 1.0 : ((lane >= c + 2 && lane < n) ? A[lane][c] * scal : 0.0);
    v[lane] = vi;
    __syncwarp();
    // p = tau A22 v
    double pi = 0.0;
    if (lane >= c + 1 && lane < n)
      for (int j = c + 1; j < n; ++j) pi += A[lane][j] * v[j];
    pi *= tc;
    const double pv = warp_sum(pi * vi);
    const double wi = pi - 0.5 * tc * pv * vi;
    w[lane] = wi;
    __syncwarp();
    if (lane >= c + 1 && lane < n)
      for (int j = c + 1; j < n; ++j) A[lane][j] -= vi * w[j] + wi * v[j];
    __syncwarp();
    if (lane >= c + 2 && lane < n) A[lane][c] = vi;  // store reflector
    if (lane == 0) {
      e[c] = beta;
      tau[c] = tc;
    }
    __syncwarp();
  }
  if (lane < n) d[lane] = A[lane][lane];
  if (lane == 0 && n >= 2) e[n - 2] = A[n - 1][n - 2];
  // Form Q = H_0 H_1 ... H_{n-3} explicitly (Z <- I, then Z <- H_c Z for c descending)
  for (int j = 0; j < n; ++j) Z[lane][j] = (lane == j) ? 1.0 : 0.0;
  __syncwarp();
  for (int c = n - 3; c >= 0; --c) {
    const double tc = tau[c];
    if (tc == 0.0) continue;
    // lane j handles column j of Z
    if (lane < n) {
      double s = Z[c + 1][lane];
      for (int i = c + 2; i < n; ++i) s += A[i][c] * Z[i][lane];
      s *= tc;
      Z[c + 1][lane] -= s;
      for (int i = c + 2; i < n; ++i) Z[i][lane] -= A[i][c] * s;
    }
    __syncwarp();
  }
  givens_qr_sweep_warp(d, e, Z, n, lane, csv[warp], v, w, fail);
  // sort ascending (selection sort by lane 0, swap columns by all lanes)
  for (int i = 0; i < n - 1; ++i) {
    if (lane == 0) {
      int kmin = i;
      for (int k = i + 1; k < n; ++k)
        if (d[k] < d[kmin]) kmin = k;
      csv[warp][0] = (double)kmin;
      if (kmin != i) {
        const double t = d[i];
        d[i] = d[kmin];
        d[kmin] = t;
      }
    }
    __syncwarp();
    const int kmin = (int)csv[warp][0];
    if (kmin != i && lane < n) {
      const double t = Z[lane][i];
      Z[lane][i] = Z[lane][kmin];
      Z[lane][kmin] = t;
    }
    __syncwarp();
  }
  if (lane < n) P.w[lane] = d[lane];
  for (int j = 0; j < n; ++j)
    if (lane < n) P.Z[lane + (size_t)j * n] = Z[lane][j];
}

// --------------------------------------------------------------------------
// Tridiagonalisation panel (cooperative persistent kernel).
// --------------------------------------------------------------------------
struct TrdProb {
  double* A;    // n x n, ld n
  double* d;    // n
  double* e;    // n-1
  double* tau;  // n-1
  double* Vp;   // n x NB panel reflectors, row-major (row i at Vp + i*NB)
  double* W;    // n x NB, row-major
  double* v;    // n
  double* y;    // n
  double* red;  // 2 slots x (2 + 2*NB)
  GridBarrier* bar;  // this problem's barrier: only its own CTAs synchronise
  int n;
  int cta0, ncta;
  int wait_log2;     // a barrier wait gives up after 2^wait_log2 polls
  int expect_extra;  // CTAs the barriers expect beyond ncta (0; 1 injects a lost CTA)
};

constexpr int RED = 2 + 2 * NB;

__device__ __forceinline__ double ld_volatile(const double* p) {
  return *reinterpret_cast<const volatile double*>(p);
}

// One panel of NB columns for every problem (cooperative launch).  Per column
// c two phases separated by grid barriers; every load of data written by
// other CTAs during the launch bypasses L1 (__ldcg).
//   A: finish the previous column: y = y' - V p - W q (p = W^T v, q = V^T v
//      of that column), W[:, jj-1] = tau y + a2 v with
//      a2 = -tau^2/2 * (y'^T v - 2 p^T q);  then
//      a = A[c:, c] - V W[c,:]^T - W V[c,:]^T and its norm below c+1.
//   B: Householder vector v of column c (every CTA forms all of it in shared
//      memory), partial p = W^T v, q = V^T v over this CTA's row chunk, and
//      y' = A22 v (one warp per column of A22), with y'^T v.
// Deferring the V p + W q correction of y to the next column's phase A saves
// the third grid barrier per column that an eager correction needs.  The
// entries below the subdiagonal of column c are overwritten with v one
// phase later too, because every CTA reads the updated column in phase B.
__global__ void __launch_bounds__(TRD_NT) trd_panel_kernel(const TrdProb* __restrict__ probs,
                                                           int nprob, int j0, int* fail) {
  extern __shared__ double sm[];
  double* scratch = sm;          // 32
  double* VWc = sm + 32;         // 2*NB: row c of V and W
  double* pq = VWc + 2 * NB;     // 2*NB: p, q of the previous column
  double* misc = pq + 2 * NB;    // 8
  double* pqw = misc + 8;        // (TRD_NT/32) x 2*NB partial p,q
  double* vs = pqw + (TRD_NT / 32) * 2 * NB;  // n_max
  const int b = blockIdx.x;
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (probs[mid].cta0 <= b) lo = mid; else hi = mid - 1;
  }
  const TrdProb P = probs[lo];
  const int rank = b - P.cta0;
  // Problems are independent: each synchronises only its own CTAs, so a
  // small problem does not wait for a large one inside a panel.
  GridBarrier* bar = P.bar;
  const unsigned nblocks = (unsigned)(P.ncta + P.expect_extra);
  const int n = P.n;
  const size_t ld = (size_t)n;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int nwarps = TRD_NT / 32;
  const int gw = rank * nwarps + warp, tw = P.ncta * nwarps;  // warp index within the problem

  for (int jj = 0; jj < NB; ++jj) {
    const int c = j0 + jj;
    const bool act = c < n;
    double* R = P.red + (c & 1) * RED;         // this column's sums
    double* Ro = P.red + ((c + 1) & 1) * RED;  // previous column's sums (next column's slot)
    // ---------------- phase A ----------------
    if (act) {
      const int kp = jj - 1;  // columns of V, W before the previous one
      double tprev = 0.0;
      if (jj > 0) tprev = __ldcg(&P.tau[c - 1]);
      if (tid < NB) {
        const int k = tid;
        pq[k] = (k < kp) ? ld_volatile(&Ro[2 + k]) : 0.0;
        pq[NB + k] = (k < kp) ? ld_volatile(&Ro[2 + NB + k]) : 0.0;
        VWc[k] = (k < jj) ? __ldcg(&P.Vp[(size_t)c * NB + k]) : 0.0;
        VWc[NB + k] = (k < kp) ? __ldcg(&P.W[(size_t)c * NB + k]) : 0.0;
      }
      __syncthreads();
      if (jj > 0 && warp == 0) {
        // scalar a2 and row c of the previous column of W (every CTA)
        const double ptq = warp_sum(pq[lane] * pq[NB + lane]);
        const double corr = warp_sum(VWc[lane] * pq[lane] + VWc[NB + lane] * pq[NB + lane]);
        const double a2 = -0.5 * tprev * tprev * (ld_volatile(&Ro[1]) - 2.0 * ptq);
        if (lane == 0) {
          misc[0] = a2;
          VWc[NB + kp] = tprev * (__ldcg(&P.y[c]) - corr) + a2 * __ldcg(&P.v[c]);
        }
      }
      __syncthreads();
      const double a2 = (jj > 0) ? misc[0] : 0.0;
      const double pk = pq[lane], qk = pq[NB + lane];
      const double vck = VWc[lane], wck = VWc[NB + lane];
      double ss = 0.0;
      for (int i = c + gw; i < n; i += tw) {
        double vik = 0.0, wik = 0.0;
        if (lane < jj) vik = __ldcg(&P.Vp[(size_t)i * NB + lane]);
        if (lane < kp) wik = __ldcg(&P.W[(size_t)i * NB + lane]);
        double wl = 0.0;
        if (jj > 0) {
          const double corr = warp_sum(vik * pk + wik * qk);
          wl = tprev * (__ldcg(&P.y[i]) - corr) + a2 * __ldcg(&P.v[i]);
          if (lane == kp) wik = wl;
        }
        const double t = warp_sum(vik * wck + wik * vck);
        if (lane == 0) {
          if (jj > 0) {
            P.W[(size_t)i * NB + kp] = wl;
            if (i >= c + 1) P.A[i + (size_t)(c - 1) * ld] = __ldcg(&P.v[i]);
          }
          const double a = __ldcg(&P.A[i + c * ld]) - t;
          P.A[i + c * ld] = a;
          if (i == c) P.d[c] = a;
          if (i >= c + 2) ss += a * a;
        }
      }
      ss = block_sum(ss, scratch);
      if (tid == 0 && ss != 0.0) atomicAdd(&R[0], ss);
    }
    if (grid_barrier(bar, nblocks, P.wait_log2)) {
      // a wait gave up: end the launch and report it (the host throws)
      if (tid == 0) atomicExch(fail, 1);
      return;
    }
    // ---------------- phase B ----------------
    if (act && c < n - 1) {
      const double alpha = __ldcg(&P.A[c + 1 + c * ld]);
      const double xn2 = ld_volatile(&R[0]);
      double beta = alpha, tc = 0.0, scal = 0.0;
      if (xn2 != 0.0) {
        beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
        tc = (beta - alpha) / beta;
        scal = 1.0 / (alpha - beta);
      }
      if (rank == 0 && tid == 0) {
        P.e[c] = beta;
        P.tau[c] = tc;
      }
      if (rank == 0 && tid < RED) Ro[tid] = 0.0;  // read in phase A, refilled from the next phase A on
      const int m = n - c - 1;
      for (int i = tid; i < m; i += TRD_NT) vs[i] = (i == 0) ? 1.0 : __ldcg(&P.A[c + 1 + i + c * ld]) * scal;
      __syncthreads();
      const int chunk = (m + P.ncta - 1) / P.ncta;
      const int r0 = c + 1 + rank * chunk, r1 = min(n, r0 + chunk);
      for (int i = r0 + tid; i < r1; i += TRD_NT) {
        const double vi = vs[i - c - 1];
        P.v[i] = vi;
        P.Vp[(size_t)i * NB + jj] = vi;
      }
      if (jj > 0) {
        double sp = 0.0, sq = 0.0;
        for (int i = r0 + warp; i < r1; i += nwarps) {
          const double vi = vs[i - c - 1];
          if (lane < jj) {
            sp += __ldcg(&P.W[(size_t)i * NB + lane]) * vi;
            sq += __ldcg(&P.Vp[(size_t)i * NB + lane]) * vi;
          }
        }
        pqw[warp * 2 * NB + lane] = sp;
        pqw[warp * 2 * NB + NB + lane] = sq;
        __syncthreads();
        if (tid < jj) {
          double a = 0.0, bq = 0.0;
          for (int w = 0; w < nwarps; ++w) {
            a += pqw[w * 2 * NB + tid];
            bq += pqw[w * 2 * NB + NB + tid];
          }
          if (a != 0.0) atomicAdd(&R[2 + tid], a);
          if (bq != 0.0) atomicAdd(&R[2 + NB + tid], bq);
        }
      }
      double yvp = 0.0;
      for (int j = c + 1 + gw; j < n; j += tw) {
        const double* col = P.A + (size_t)j * ld + (c + 1);
        double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int i = lane;
        for (; i + 480 < m; i += 512) {
          double x[16];
#pragma unroll
          for (int u = 0; u < 16; ++u) x[u] = __ldcg(&col[i + 32 * u]);
#pragma unroll
          for (int u = 0; u < 16; ++u) s[u & 7] += x[u] * vs[i + 32 * u];
        }
        for (; i + 224 < m; i += 256) {
#pragma unroll
          for (int u = 0; u < 8; ++u) s[u] += __ldcg(&col[i + 32 * u]) * vs[i + 32 * u];
        }
        for (; i < m; i += 32) s[0] += __ldcg(&col[i]) * vs[i];
        const double yj = warp_sum(((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7])));
        if (lane == 0) {
          P.y[j] = yj;
          yvp += yj * vs[j - c - 1];
        }
      }
      yvp = block_sum(yvp, scratch);
      if (tid == 0 && yvp != 0.0) atomicAdd(&R[1], yvp);
    }
    if (grid_barrier(bar, nblocks, P.wait_log2)) {
      // a wait gave up: end the launch and report it (the host throws)
      if (tid == 0) atomicExch(fail, 1);
      return;
    }
  }
  // finish the panel's last column: W[:, NB-1] for the trailing update and v
  // below its subdiagonal
  const int c = j0 + NB - 1;
  if (c < n - 1) {
    const double* R = P.red + (c & 1) * RED;
    const double tc = __ldcg(&P.tau[c]);
    if (tid < NB) {
      pq[tid] = (tid < NB - 1) ? ld_volatile(&R[2 + tid]) : 0.0;
      pq[NB + tid] = (tid < NB - 1) ? ld_volatile(&R[2 + NB + tid]) : 0.0;
    }
    __syncthreads();
    const double pk = pq[lane], qk = pq[NB + lane];
    const double a2 = -0.5 * tc * tc * (ld_volatile(&R[1]) - 2.0 * warp_sum(pk * qk));
    for (int i = c + 1 + gw; i < n; i += tw) {
      double corr = 0.0;
      if (lane < NB - 1)
        corr = __ldcg(&P.Vp[(size_t)i * NB + lane]) * pk + __ldcg(&P.W[(size_t)i * NB + lane]) * qk;
      corr = warp_sum(corr);
      if (lane == 0) {
        const double vi = __ldcg(&P.v[i]);
        P.W[(size_t)i * NB + NB - 1] = tc * (__ldcg(&P.y[i]) - corr) + a2 * vi;
        if (i >= c + 2) P.A[i + c * ld] = vi;
      }
    }
  }
  // a barrier that gave up is reported to the host (the barriers are reset per launch)
  if (tid == 0 && *reinterpret_cast<volatile int*>(&bar->error)) atomicExch(fail, 1);
}

// --------------------------------------------------------------------------
// Tridiagonalisation of a medium block inside one thread-block cluster.
// --------------------------------------------------------------------------
struct TrdClProb {
  double* A;    // n x n, leading dimension ld: input; on return the reflectors below the subdiagonal
  double* d;    // n
  double* e;    // n-1
  double* tau;  // n-1
  int n;
  int ld;       // n for a whole block; the block's size for its trailing part
};

// Leading dimension of a column held in shared memory: odd, so that 32 lanes
// reading the same row of 32 different columns hit 32 different banks.
__host__ __device__ inline int trdc_ld(int n) { return n | 1; }

// Doubles of dynamic shared memory one CTA needs for a block of size n on
// a cluster of cl CTAs: its columns (j = rank, rank + cl, ...) in full, then
// v and y (n each), one partial column dot per thread, one partial sum of
// y^T v per warp of every CTA, 2 x 4 scalars.
__host__ __device__ inline size_t trdc_smem_doubles(int n, int cl) {
  return (size_t)((n + cl - 1) / cl) * trdc_ld(n) + 2 * (size_t)n + TRDC_NT + (size_t)cl * (TRDC_NT / 32) + 8;
}

// Active held columns up to this count take the warp-per-column-group
// product (lanes across rows, shuffle reductions, no CTA barrier); more take
// lanes across columns (no shuffles) with a CTA barrier before the sums.
constexpr int TRDC_WARPCOL_MAX = 32;

// Barrier over the CTAs of the cluster (a plain CTA barrier for CL = 1).
template <int CL>
__device__ __forceinline__ void trdc_sync() {
  if constexpr (CL == 1) {
    __syncthreads();
  } else {
    cooperative_groups::this_cluster().sync();
  }
}

// Address of `p` in the shared memory of CTA `rank` of the cluster.
template <int CL, class T>
__device__ __forceinline__ T* trdc_at(T* p, int rank) {
  if constexpr (CL == 1) {
    return p;
  } else {
    return cooperative_groups::this_cluster().map_shared_rank(p, rank);
  }
}

// Reflector of column cc, held in shared memory (`col`), by one warp of its
// owner: beta, tau and the scale of v, written into every CTA's scalars
// `mc`; d, e, tau to global memory.
template <int CL>
__device__ __forceinline__ void trdc_reflector(const TrdClProb& P, const double* col, int cc, int n, double* mc,
                                               int lane) {
  double ss = 0.0;
  for (int i = cc + 2 + lane; i < n; i += 32) ss += col[i] * col[i];
  ss = warp_sum(ss);
  const double alpha = col[cc + 1];
  double beta = alpha, tc = 0.0, scal = 0.0;
  if (ss != 0.0) {
    beta = -copysign(sqrt(alpha * alpha + ss), alpha);
    tc = (beta - alpha) / beta;
    scal = 1.0 / (alpha - beta);
  }
  if (lane < CL) {
    double* rm = trdc_at<CL>(mc, lane);
    rm[0] = tc;
    rm[1] = scal;
  }
  if (lane == 0) {
    P.d[cc] = col[cc];
    P.e[cc] = beta;
    P.tau[cc] = tc;
  }
}

// Unblocked Householder tridiagonalisation (the dsytd2 recurrence, lower)
// of one block per cluster of CL CTAs.  The matrix lives in the CTAs'
// shared memory, distributed by columns (CTA r holds the columns j with
// j % CL == r, each in full), so the symmetric product y = A v needs no
// reduction across CTAs: y_j is the dot product of the held column j with v.
// Per column c, two cluster barriers:
//   a. every CTA reads the owner's column c through distributed shared
//      memory to form v (CTA barrier) and computes y_j for its columns:
//      with few active columns each warp takes four columns at a time
//      (lanes across rows, shuffle reductions); with many, lanes take
//      columns and warps row segments, summed after a CTA barrier.  Each
//      y_j goes into every CTA, and each warp's part of y^T v into its own
//      slot of every CTA; cluster barrier;
//   b. every warp sums the slots (all in the same order, so every CTA
//      holds the same y^T v) and applies A -= v w^T + w v^T to its columns
//      with w = tau y - tau^2/2 (y^T v) v formed on the fly (loads of four
//      columns and two rows issued before their stores).  Meanwhile warp 0
//      of the owner of column c+1 updates that column first and forms its
//      reflector (norm, beta, tau), writing the scalars into every CTA;
//      cluster barrier.
// Output as the panel kernel: d, e, tau, and v below the subdiagonal of A.
template <int CL>
__global__ void __launch_bounds__(TRDC_NT) trd_cluster_kernel(const TrdClProb* __restrict__ probs) {
  int r = 0;
  if constexpr (CL > 1) r = (int)cooperative_groups::this_cluster().block_rank();
  const TrdClProb P = probs[blockIdx.x / CL];
  const int n = P.n;
  const size_t ld = (size_t)P.ld;
  const int lds = trdc_ld(n);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int nwarps = TRDC_NT / 32;
  const int ncol = r < n ? (n - r + CL - 1) / CL : 0;
  extern __shared__ double sm[];
  double* Acol = sm;                                     // ncol columns, ld lds
  double* v = Acol + (size_t)((n + CL - 1) / CL) * lds;  // n
  double* y = v + n;                                     // n (written by every CTA)
  double* ypart = y + n;                                 // TRDC_NT partial column dots
  double* part = ypart + TRDC_NT;                        // CL x nwarps parts of y^T v
  double* misc = part + CL * nwarps;                     // 2 x 4 reflector scalars

  for (int l = 0; l < ncol; ++l) {
    const double* src = P.A + (size_t)(r + l * CL) * ld;
    for (int i = tid; i < n; i += TRDC_NT) Acol[(size_t)l * lds + i] = src[i];
  }
  // every CTA of the cluster has started (and loaded) before any of them
  // touches another's shared memory
  trdc_sync<CL>();
  if (n > 1 && r == 0 && warp == 0) trdc_reflector<CL>(P, Acol, 0, n, misc, lane);
  trdc_sync<CL>();

  for (int c = 0; c < n - 1; ++c) {
    const int o = c % CL;
    const double* mc = misc + (c & 1) * 4;
    // ---- a: v, y_j for the columns held here, parts of y^T v ----
    const double tc = mc[0], scal = mc[1];
    {
      const double* ocol = trdc_at<CL>(Acol, o) + (size_t)(c / CL) * lds;
      for (int i = c + 1 + tid; i < n; i += TRDC_NT) v[i] = (i == c + 1) ? 1.0 : ocol[i] * scal;
    }
    __syncthreads();
    // held columns after c: local indices l0 .. ncol-1
    const int l0 = (c + 1 - r + CL - 1) / CL > 0 ? (c + 1 - r + CL - 1) / CL : 0;
    const int nact = ncol > l0 ? ncol - l0 : 0;
    double sp = 0.0;
    if (nact <= TRDC_WARPCOL_MAX) {
      // warp w: active columns t = w, w + nwarps, ..., four at a time
      for (int t0 = warp; t0 < nact; t0 += 4 * nwarps) {
        const double* a[4];
        bool on[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int t = t0 + k * nwarps;
          on[k] = t < nact;
          a[k] = Acol + (size_t)(l0 + (on[k] ? t : t0)) * lds;
        }
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int i = c + 1 + lane; i < n; i += 32) {
          const double vi = v[i];
#pragma unroll
          for (int k = 0; k < 4; ++k) acc[k] += a[k][i] * vi;
        }
#pragma unroll
        for (int o2 = 16; o2 > 0; o2 >>= 1) {
#pragma unroll
          for (int k = 0; k < 4; ++k) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o2);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          if (!on[k]) continue;
          const int j = r + (l0 + t0 + k * nwarps) * CL;
          if (lane < CL) trdc_at<CL>(y, lane)[j] = acc[k];
          sp += acc[k] * v[j];
        }
      }
    } else {
      // lanes across 32 columns, warps across column groups and row segments
      const int chunks = (nact + 31) >> 5;
      const int segs = max(1, nwarps / chunks);
      if (warp < chunks * segs) {
        const int ch = warp % chunks, sg = warp / chunks;
        const int m = n - c - 1;
        const int per = (m + segs - 1) / segs;
        const int i0 = c + 1 + sg * per, i1 = min(n, i0 + per);
        const int t = ch * 32 + lane;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        if (t < nact) {
          const double* a = Acol + (size_t)(l0 + t) * lds;
          int i = i0;
          for (; i + 3 < i1; i += 4) {
            s0 += a[i] * v[i];
            s1 += a[i + 1] * v[i + 1];
            s2 += a[i + 2] * v[i + 2];
            s3 += a[i + 3] * v[i + 3];
          }
          for (; i < i1; ++i) s0 += a[i] * v[i];
        }
        ypart[sg * (chunks * 32) + t] = (s0 + s1) + (s2 + s3);
      }
      __syncthreads();
      for (int t = tid; t < nact; t += TRDC_NT) {
        double yj = 0.0;
        for (int sg = 0; sg < segs; ++sg) yj += ypart[sg * (chunks * 32) + t];
        const int j = r + (l0 + t) * CL;
#pragma unroll
        for (int q = 0; q < CL; ++q) trdc_at<CL>(y, q)[j] = yj;
        sp += yj * v[j];
      }
      sp = warp_sum(sp);
    }
    if (lane < CL) trdc_at<CL>(part, lane)[r * nwarps + warp] = sp;
    trdc_sync<CL>();
    // ---- b: the rank-2 update with w on the fly, the next reflector ----
    double ytv = 0.0;
    for (int q = lane; q < CL * nwarps; q += 32) ytv += part[q];
    ytv = warp_sum(ytv);
    const double a2 = -0.5 * tc * tc * ytv;
    if (r == o)
      for (int i = c + 2 + tid; i < n; i += TRDC_NT) P.A[i + (size_t)c * ld] = v[i];
    const int cn = c + 1;
    const bool own_next = cn < n - 1 && r == cn % CL;  // column cn is then local column l0
    const int wfirst = own_next ? 1 : 0;
    if (tc != 0.0 && warp >= wfirst) {
      const int nw = nwarps - wfirst;
      for (int l = l0 + wfirst + 4 * (warp - wfirst); l < ncol; l += 4 * nw) {
        const int nl = min(4, ncol - l);
        double vj[4], wj[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int j = r + (l + min(k, nl - 1)) * CL;
          vj[k] = v[j];
          wj[k] = tc * y[j] + a2 * v[j];
        }
        double* a0 = Acol + (size_t)l * lds;
        int i = c + 1 + lane;
        for (; i + 32 < n; i += 64) {
          const double v0 = v[i], v1 = v[i + 32];
          const double w0 = tc * y[i] + a2 * v0, w1 = tc * y[i + 32] + a2 * v1;
          double x[8];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            x[k] = k < nl ? a0[(size_t)k * lds + i] : 0.0;
            x[4 + k] = k < nl ? a0[(size_t)k * lds + i + 32] : 0.0;
          }
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            x[k] -= v0 * wj[k] + w0 * vj[k];
            x[4 + k] -= v1 * wj[k] + w1 * vj[k];
          }
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (k < nl) {
              a0[(size_t)k * lds + i] = x[k];
              a0[(size_t)k * lds + i + 32] = x[4 + k];
            }
        }
        if (i < n) {
          const double v0 = v[i];
          const double w0 = tc * y[i] + a2 * v0;
          double x[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) x[k] = k < nl ? a0[(size_t)k * lds + i] : 0.0;
#pragma unroll
          for (int k = 0; k < 4; ++k) x[k] -= v0 * wj[k] + w0 * vj[k];
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (k < nl) a0[(size_t)k * lds + i] = x[k];
        }
      }
    }
    if (own_next && warp == 0) {
      double* col = Acol + (size_t)l0 * lds;
      if (tc != 0.0) {
        const double vj = v[cn], wj = tc * y[cn] + a2 * v[cn];
        for (int i = c + 1 + lane; i < n; i += 32) col[i] -= v[i] * wj + (tc * y[i] + a2 * v[i]) * vj;
        __syncwarp();
      }
      trdc_reflector<CL>(P, col, cn, n, misc + (cn & 1) * 4, lane);
    }
    trdc_sync<CL>();
  }
  if (n >= 1 && r == (n - 1) % CL && tid == 0) P.d[n - 1] = Acol[(size_t)((n - 1) / CL) * lds + (n - 1)];
  // no CTA leaves while another may still read its shared memory
  trdc_sync<CL>();
}

// Threads of a CTA of the one-barrier kernel (8 warps; 16 measured slower,
// and so did splitting the rank-2 update into column x row-segment tasks).
constexpr int TRDC1_NT = 256;
// Rows of the next column each thread of the one-barrier kernel reads from
// its owner before the rank-2 update and finishes after it.
constexpr int TRDC1_ROWS = 4;

// Doubles of dynamic shared memory of the one-barrier kernel: the held
// columns, v, the running copy of the next column, y twice (alternating by
// column parity), one partial column dot per thread, the parts of y^T v
// twice, one partial norm per warp, scalars.
__host__ __device__ inline size_t trdc1_smem_doubles(int n, int cl) {
  return (size_t)((n + cl - 1) / cl) * trdc_ld(n) + 4 * (size_t)n + TRDC1_NT + 2 * (size_t)cl * (TRDC1_NT / 32) +
         (TRDC1_NT / 32) + 8;
}



// The same recurrence with one cluster barrier per column.  Every CTA keeps
// its own copy of the column being reduced and forms each reflector itself
// (all CTAs run the same arithmetic on the same values, so they agree to the
// bit); the owner of a column therefore never broadcasts it, and the second
// cluster barrier of trd_cluster_kernel is gone.  Per column c:
//   a. beta, tau and v of column c from the local copy (the norm's partial
//      sums were left by step c-1); y_j of the held columns j > c into
//      every CTA's y buffer of this parity, parts of y^T v likewise; cluster
//      barrier;
//   b. every CTA reads column c+1 from its owner's shared memory (which the
//      owner no longer updates from this step on), applies this step's
//      rank-2 correction to it and leaves the partial norms for step c+1;
//      the held columns j > c+1 take the rank-2 update; CTA barrier.
// y and the parts alternate by parity: a CTA writes step c+1's values only
// after the cluster barrier of step c+1, which every CTA reaches after it has
// read step c-1's.  Output as trd_cluster_kernel.
template <int CL>
__global__ void __launch_bounds__(TRDC1_NT) trd_cluster1_kernel(const TrdClProb* __restrict__ probs) {
  int r = 0;
  if constexpr (CL > 1) r = (int)cooperative_groups::this_cluster().block_rank();
  const TrdClProb P = probs[blockIdx.x / CL];
  const int n = P.n;
  const size_t ld = (size_t)P.ld;
  const int lds = trdc_ld(n);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int nwarps = TRDC1_NT / 32;
  const int ncol = r < n ? (n - r + CL - 1) / CL : 0;
  extern __shared__ double sm[];
  double* Acol = sm;                                     // ncol columns, ld lds
  double* v = Acol + (size_t)((n + CL - 1) / CL) * lds;  // n
  double* cur = v + n;                                   // n: column c (rows c .. n-1)
  double* ybuf = cur + n;                                // 2 x n (written by every CTA)
  double* ypart = ybuf + 2 * (size_t)n;                  // TRDC1_NT partial column dots
  double* pbuf = ypart + TRDC1_NT;                        // 2 x CL x nwarps parts of y^T v
  double* psq = pbuf + 2 * CL * nwarps;                  // nwarps partial norms

  for (int l = 0; l < ncol; ++l) {
    const double* src = P.A + (size_t)(r + l * CL) * ld;
    for (int i = tid; i < n; i += TRDC1_NT) Acol[(size_t)l * lds + i] = src[i];
  }
  // every CTA of the cluster has loaded before any of them reads another's
  // shared memory; then column 0 from CTA 0
  trdc_sync<CL>();
  {
    const double* c0 = trdc_at<CL>(Acol, 0);
    double sq = 0.0;
    for (int i = tid; i < n; i += TRDC1_NT) {
      const double x = c0[i];
      cur[i] = x;
      if (i >= 2) sq += x * x;
    }
    sq = warp_sum(sq);
    if (lane == 0) psq[warp] = sq;
  }
  __syncthreads();

  for (int c = 0; c < n - 1; ++c) {
    double* y = ybuf + (size_t)(c & 1) * n;
    double* part = pbuf + (c & 1) * CL * nwarps;
    // ---- a: reflector of column c, v, y_j for the columns held here ----
    double ss = 0.0;
#pragma unroll
    for (int q = 0; q < nwarps; ++q) ss += psq[q];
    const double alpha = cur[c + 1];
    double beta = alpha, tc = 0.0, scal = 0.0;
    if (ss != 0.0) {
      beta = -copysign(sqrt(alpha * alpha + ss), alpha);
      tc = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
    if (r == 0 && tid == 0) {
      P.d[c] = cur[c];
      P.e[c] = beta;
      P.tau[c] = tc;
    }
    const bool own = r == c % CL;
    for (int i = c + 1 + tid; i < n; i += TRDC1_NT) {
      const double vi = (i == c + 1) ? 1.0 : cur[i] * scal;
      v[i] = vi;
      if (own && i >= c + 2) P.A[i + (size_t)c * ld] = vi;
    }
    __syncthreads();
    // held columns after c: local indices l0 .. ncol-1
    const int l0 = (c + 1 - r + CL - 1) / CL > 0 ? (c + 1 - r + CL - 1) / CL : 0;
    const int nact = ncol > l0 ? ncol - l0 : 0;
    double sp = 0.0;
    if (nact <= TRDC_WARPCOL_MAX) {
      for (int t0 = warp; t0 < nact; t0 += 4 * nwarps) {
        const double* a[4];
        bool on[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int t = t0 + k * nwarps;
          on[k] = t < nact;
          a[k] = Acol + (size_t)(l0 + (on[k] ? t : t0)) * lds;
        }
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int i = c + 1 + lane; i < n; i += 32) {
          const double vi = v[i];
#pragma unroll
          for (int k = 0; k < 4; ++k) acc[k] += a[k][i] * vi;
        }
#pragma unroll
        for (int o2 = 16; o2 > 0; o2 >>= 1) {
#pragma unroll
          for (int k = 0; k < 4; ++k) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o2);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          if (!on[k]) continue;
          const int j = r + (l0 + t0 + k * nwarps) * CL;
          if (lane < CL) trdc_at<CL>(y, lane)[j] = acc[k];
          sp += acc[k] * v[j];
        }
      }
    } else {
      const int chunks = (nact + 31) >> 5;
      const int segs = max(1, nwarps / chunks);
      if (warp < chunks * segs) {
        const int ch = warp % chunks, sg = warp / chunks;
        const int m = n - c - 1;
        const int per = (m + segs - 1) / segs;
        const int i0 = c + 1 + sg * per, i1 = min(n, i0 + per);
        const int t = ch * 32 + lane;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        if (t < nact) {
          const double* a = Acol + (size_t)(l0 + t) * lds;
          int i = i0;
          for (; i + 3 < i1; i += 4) {
            s0 += a[i] * v[i];
            s1 += a[i + 1] * v[i + 1];
            s2 += a[i + 2] * v[i + 2];
            s3 += a[i + 3] * v[i + 3];
          }
          for (; i < i1; ++i) s0 += a[i] * v[i];
        }
        ypart[sg * (chunks * 32) + t] = (s0 + s1) + (s2 + s3);
      }
      __syncthreads();
      for (int t = tid; t < nact; t += TRDC1_NT) {
        double yj = 0.0;
        for (int sg = 0; sg < segs; ++sg) yj += ypart[sg * (chunks * 32) + t];
        const int j = r + (l0 + t) * CL;
#pragma unroll
        for (int q = 0; q < CL; ++q) trdc_at<CL>(y, q)[j] = yj;
        sp += yj * v[j];
      }
      sp = warp_sum(sp);
    }
    if (lane < CL) trdc_at<CL>(part, lane)[r * nwarps + warp] = sp;
    trdc_sync<CL>();
    // ---- b: column c+1 from its owner, the rank-2 update ----
    const int cn = c + 1;
    double xr[TRDC1_ROWS];
    {
      const double* ocol = trdc_at<CL>(Acol, cn % CL) + (size_t)(cn / CL) * lds;
#pragma unroll
      for (int k = 0; k < TRDC1_ROWS; ++k) {
        const int i = cn + tid + k * TRDC1_NT;
        xr[k] = i < n ? ocol[i] : 0.0;
      }
    }
    double ytv = 0.0;
    for (int q = lane; q < CL * nwarps; q += 32) ytv += part[q];
    ytv = warp_sum(ytv);
    const double a2 = -0.5 * tc * tc * ytv;
    // held columns after c+1: local indices l1 .. ncol-1
    const int l1 = (c + 2 - r + CL - 1) / CL > 0 ? (c + 2 - r + CL - 1) / CL : 0;
    if (tc != 0.0) {
      for (int l = l1 + 4 * warp; l < ncol; l += 4 * nwarps) {
        const int nl = min(4, ncol - l);
        double vj[4], wj[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int j = r + (l + min(k, nl - 1)) * CL;
          vj[k] = v[j];
          wj[k] = tc * y[j] + a2 * v[j];
        }
        double* a0 = Acol + (size_t)l * lds;
        int i = c + 1 + lane;
        for (; i + 32 < n; i += 64) {
          const double v0 = v[i], v1 = v[i + 32];
          const double w0 = tc * y[i] + a2 * v0, w1 = tc * y[i + 32] + a2 * v1;
          double x[8];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            x[k] = k < nl ? a0[(size_t)k * lds + i] : 0.0;
            x[4 + k] = k < nl ? a0[(size_t)k * lds + i + 32] : 0.0;
          }
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            x[k] -= v0 * wj[k] + w0 * vj[k];
            x[4 + k] -= v1 * wj[k] + w1 * vj[k];
          }
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (k < nl) {
              a0[(size_t)k * lds + i] = x[k];
              a0[(size_t)k * lds + i + 32] = x[4 + k];
            }
        }
        if (i < n) {
          const double v0 = v[i];
          const double w0 = tc * y[i] + a2 * v0;
          double x[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) x[k] = k < nl ? a0[(size_t)k * lds + i] : 0.0;
#pragma unroll
          for (int k = 0; k < 4; ++k) x[k] -= v0 * wj[k] + w0 * vj[k];
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (k < nl) a0[(size_t)k * lds + i] = x[k];
        }
      }
    }
    {
      // column c+1 after this step (rows c+1 .. n-1) and its partial norm
      // over rows c+3 .. n-1 (v[c+1] = 1)
      const double wn = tc * y[cn] + a2;
      double sq = 0.0;
#pragma unroll
      for (int k = 0; k < TRDC1_ROWS; ++k) {
        const int i = cn + tid + k * TRDC1_NT;
        if (i < n) {
          double x = xr[k];
          if (tc != 0.0) x -= v[i] * wn + (tc * y[i] + a2 * v[i]);
          cur[i] = x;
          if (i >= cn + 2) sq += x * x;
        }
      }
      sq = warp_sum(sq);
      if (lane == 0) psq[warp] = sq;
    }
    __syncthreads();
  }
  if (n >= 1 && r == 0 && tid == 0) P.d[n - 1] = cur[n - 1];
  // no CTA leaves while another may still read its shared memory
  trdc_sync<CL>();
}

// Doubles of dynamic shared memory of the fused kernel: the held columns, v
// twice, the running copy of the next column, y twice, the parts of y^T v
// twice, one partial norm per warp, scalars.
__host__ __device__ inline size_t trdc2_smem_doubles(int n, int cl) {
  return (size_t)((n + cl - 1) / cl) * trdc_ld(n) + 5 * (size_t)n + 2 * (size_t)cl * (TRDC1_NT / 32) +
         (TRDC1_NT / 32) + 8;
}

// The one-barrier recurrence with the rank-2 update of step c and the
// products of step c+1 in one pass over the held columns.  Right after the
// cluster barrier of step c every CTA holds y_c, v_c and the parts of
// y_c^T v_c, so it can finish column c+1 (read from its owner) and form
// v_{c+1} before it touches its own columns; then each held column j > c+1
// is updated and, while its rows are in registers, dotted with v_{c+1}.
// Per column: one pass over the held columns, one CTA barrier (after the
// next column's partial norms) and one cluster barrier (after y_{c+1} and
// the parts of y_{c+1}^T v_{c+1} reach every CTA).  v, y and the parts
// alternate between two buffers by column parity.  The loop starts at
// c = -1 (no update; column 0 read raw), so the first products need no
// separate pass.  Rows above c+2 of a held column are dead after step c and
// are not updated.  Output as trd_cluster_kernel.
template <int CL>
__global__ void __launch_bounds__(TRDC1_NT) trd_cluster2_kernel(const TrdClProb* __restrict__ probs) {
  int r = 0;
  if constexpr (CL > 1) r = (int)cooperative_groups::this_cluster().block_rank();
  const TrdClProb P = probs[blockIdx.x / CL];
  const int n = P.n;
  const size_t ld = (size_t)P.ld;
  const int lds = trdc_ld(n);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  constexpr int nwarps = TRDC1_NT / 32;
  const int ncol = r < n ? (n - r + CL - 1) / CL : 0;
  extern __shared__ double sm[];
  double* Acol = sm;                                        // ncol columns, ld lds
  double* vbuf = Acol + (size_t)((n + CL - 1) / CL) * lds;  // 2 x n
  double* cur = vbuf + 2 * (size_t)n;                       // n: column c+1 (rows c+1 .. n-1)
  double* ybuf = cur + n;                                   // 2 x n (written by every CTA)
  double* pbuf = ybuf + 2 * (size_t)n;                      // 2 x CL x nwarps parts of y^T v
  double* psq = pbuf + 2 * CL * nwarps;                     // nwarps partial norms

  for (int l = 0; l < ncol; ++l) {
    const double* src = P.A + (size_t)(r + l * CL) * ld;
    for (int i = tid; i < n; i += TRDC1_NT) Acol[(size_t)l * lds + i] = src[i];
  }
  // every CTA of the cluster has loaded before any of them reads another's
  trdc_sync<CL>();

  double tc = 0.0;  // tau of column c (0 for c = -1)
  for (int c = -1; c < n - 1; ++c) {
    const int cn = c + 1;
    const double* v = vbuf + (size_t)((c + 2) & 1) * n;  // v_c (parity of c, kept non-negative)
    double* vn = vbuf + (size_t)((c + 1) & 1) * n;        // v_{c+1}
    const double* y = ybuf + (size_t)((c + 2) & 1) * n;
    double* yn = ybuf + (size_t)((c + 1) & 1) * n;
    const double* part = pbuf + ((c + 2) & 1) * CL * nwarps;
    double* partn = pbuf + ((c + 1) & 1) * CL * nwarps;
    // ---- column c+1 from its owner, corrected by step c; its partial norm ----
    double xr[TRDC1_ROWS];
    {
      const double* ocol = trdc_at<CL>(Acol, cn % CL) + (size_t)(cn / CL) * lds;
#pragma unroll
      for (int k = 0; k < TRDC1_ROWS; ++k) {
        const int i = cn + tid + k * TRDC1_NT;
        xr[k] = i < n ? ocol[i] : 0.0;
      }
    }
    double a2 = 0.0;
    if (c >= 0 && tc != 0.0) {
      double ytv = 0.0;
      for (int q = lane; q < CL * nwarps; q += 32) ytv += part[q];
      ytv = warp_sum(ytv);
      a2 = -0.5 * tc * tc * ytv;
    }
    {
      const double wn = (c >= 0 && tc != 0.0) ? tc * y[cn] + a2 : 0.0;
      double sq = 0.0;
#pragma unroll
      for (int k = 0; k < TRDC1_ROWS; ++k) {
        const int i = cn + tid + k * TRDC1_NT;
        if (i < n) {
          double x = xr[k];
          if (c >= 0 && tc != 0.0) x -= v[i] * wn + (tc * y[i] + a2 * v[i]);
          cur[i] = x;
          if (i >= cn + 2) sq += x * x;
        }
      }
      sq = warp_sum(sq);
      if (lane == 0) psq[warp] = sq;
    }
    __syncthreads();
    if (cn == n - 1) {
      if (r == 0 && tid == 0) P.d[n - 1] = cur[n - 1];
      break;
    }
    // ---- reflector of column c+1 (every thread, same arithmetic) ----
    double ss = 0.0;
#pragma unroll
    for (int q = 0; q < nwarps; ++q) ss += psq[q];
    const double alpha = cur[cn + 1];
    double beta = alpha, tcn = 0.0, scal = 0.0;
    if (ss != 0.0) {
      beta = -copysign(sqrt(alpha * alpha + ss), alpha);
      tcn = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
    if (r == 0 && tid == 0) {
      P.d[cn] = cur[cn];
      P.e[cn] = beta;
      P.tau[cn] = tcn;
    }
    const bool own = r == cn % CL;
    for (int i = cn + 1 + tid; i < n; i += TRDC1_NT) {
      const double vi = (i == cn + 1) ? 1.0 : cur[i] * scal;
      vn[i] = vi;
      if (own && i >= cn + 2) P.A[i + (size_t)cn * ld] = vi;
    }
    // ---- update of the held columns j > c+1 by step c, products with v_{c+1} ----
    const int l1 = (c + 2 - r + CL - 1) / CL > 0 ? (c + 2 - r + CL - 1) / CL : 0;
    const bool upd = c >= 0 && tc != 0.0;
    double sp = 0.0;
    for (int l = l1 + 4 * warp; l < ncol; l += 4 * nwarps) {
      const int nl = min(4, ncol - l);
      double vj[4], wj[4], acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int j = r + (l + min(k, nl - 1)) * CL;
        vj[k] = upd ? v[j] : 0.0;
        wj[k] = upd ? tc * y[j] + a2 * v[j] : 0.0;
      }
      double* a0 = Acol + (size_t)l * lds;
      int i = cn + 1 + lane;
      for (; i + 32 < n; i += 64) {
        const double p0 = (i == cn + 1) ? 1.0 : cur[i] * scal;
        const double p1 = cur[i + 32] * scal;
        double x[8];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          x[k] = k < nl ? a0[(size_t)k * lds + i] : 0.0;
          x[4 + k] = k < nl ? a0[(size_t)k * lds + i + 32] : 0.0;
        }
        if (upd) {
          const double v0 = v[i], v1 = v[i + 32];
          const double w0 = tc * y[i] + a2 * v0, w1 = tc * y[i + 32] + a2 * v1;
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            x[k] -= v0 * wj[k] + w0 * vj[k];
            x[4 + k] -= v1 * wj[k] + w1 * vj[k];
          }
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (k < nl) {
              a0[(size_t)k * lds + i] = x[k];
              a0[(size_t)k * lds + i + 32] = x[4 + k];
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[k] += x[k] * p0 + x[4 + k] * p1;
      }
      if (i < n) {
        const double p0 = (i == cn + 1) ? 1.0 : cur[i] * scal;
        double x[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) x[k] = k < nl ? a0[(size_t)k * lds + i] : 0.0;
        if (upd) {
          const double v0 = v[i];
          const double w0 = tc * y[i] + a2 * v0;
#pragma unroll
          for (int k = 0; k < 4; ++k) x[k] -= v0 * wj[k] + w0 * vj[k];
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (k < nl) a0[(size_t)k * lds + i] = x[k];
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[k] += x[k] * p0;
      }
#pragma unroll
      for (int o2 = 16; o2 > 0; o2 >>= 1) {
#pragma unroll
        for (int k = 0; k < 4; ++k) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o2);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (k >= nl) continue;
        const int j = r + (l + k) * CL;
        if (lane < CL) trdc_at<CL>(yn, lane)[j] = acc[k];
        sp += acc[k] * ((j == cn + 1) ? 1.0 : cur[j] * scal);
      }
    }
    if (lane < CL) trdc_at<CL>(partn, lane)[r * nwarps + warp] = sp;
    tc = tcn;
    trdc_sync<CL>();
  }
  // no CTA leaves while another may still read its shared memory
  trdc_sync<CL>();
}

// Launch configuration of the cluster kernel for `nprob` blocks.  The
// kernel's attributes (largest dynamic shared memory, non-portable cluster
// size) are set once per device, at the largest size any launch uses, by the
// solver's constructor (set_attr): setting them per launch to the launch's
// own size would race between solver instances on other threads.
// The cluster kernel of CL CTAs: 0 two cluster barriers per column, 1 one,
// 2 one with the update and the next products fused.  The default (1) is
// built for every cluster size 1..16, the comparison forms for the powers
// of two only.
template <int CL>
void (*trdc_kernel(int variant))(const TrdClProb*) {
  if constexpr ((CL & (CL - 1)) == 0) {
    if (variant == 2) return trd_cluster2_kernel<CL>;
    if (variant == 0) return trd_cluster_kernel<CL>;
  }
  return trd_cluster1_kernel<CL>;
}

// Whether the cluster kernel of this variant is built for CL CTAs.
inline bool trdc_size_built(int variant, int CL) {
  return CL >= 1 && CL <= TRDC_CL_MAX && (variant == 1 || (CL & (CL - 1)) == 0);
}

// f(std::integral_constant<int, CL>{}) for a runtime cluster size 1..16.
template <class F>
auto trdc_with_cl(int CL, F&& f) {
  switch (CL) {
    case 1: return f(std::integral_constant<int, 1>{});
    case 2: return f(std::integral_constant<int, 2>{});
    case 3: return f(std::integral_constant<int, 3>{});
    case 4: return f(std::integral_constant<int, 4>{});
    case 5: return f(std::integral_constant<int, 5>{});
    case 6: return f(std::integral_constant<int, 6>{});
    case 7: return f(std::integral_constant<int, 7>{});
    case 8: return f(std::integral_constant<int, 8>{});
    case 9: return f(std::integral_constant<int, 9>{});
    case 10: return f(std::integral_constant<int, 10>{});
    case 11: return f(std::integral_constant<int, 11>{});
    case 12: return f(std::integral_constant<int, 12>{});
    case 13: return f(std::integral_constant<int, 13>{});
    case 14: return f(std::integral_constant<int, 14>{});
    case 15: return f(std::integral_constant<int, 15>{});
    default: return f(std::integral_constant<int, 16>{});
  }
}

template <int CL>
cudaError_t trdc_config(int one, size_t smem, cudaLaunchConfig_t& cfg, cudaLaunchAttribute* at, int nprob,
                        cudaStream_t st, bool set_attr) {
  cfg = cudaLaunchConfig_t{};
  cfg.gridDim = dim3((unsigned)(nprob * CL));
  cfg.blockDim = dim3(one ? TRDC1_NT : TRDC_NT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CL;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  if (!set_attr) return cudaSuccess;
  cudaError_t e = cudaFuncSetAttribute(trdc_kernel<CL>(one), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess && CL > 8)
    e = cudaFuncSetAttribute(trdc_kernel<CL>(one), cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  return e;
}

// Clusters of CL CTAs with `smem` bytes each that can be resident at once
// (0: this cluster size is not usable here); sets the kernel's attributes
// for launches of up to `smem` bytes.
template <int CL>
int trdc_max_clusters(int one, size_t smem) {
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute at[1];
  if (trdc_config<CL>(one, smem, cfg, at, 1, nullptr, true) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  int nc = 0;
  if (cudaOccupancyMaxActiveClusters(&nc, trdc_kernel<CL>(one), &cfg) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return nc;
}

template <int CL>
cudaError_t trdc_launch(int one, const TrdClProb* d, int nprob, size_t smem, cudaStream_t st) {
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute at[1];
  cudaError_t e = trdc_config<CL>(one, smem, cfg, at, nprob, st, false);
  if (e != cudaSuccess) return e;
  return cudaLaunchKernelEx(&cfg, trdc_kernel<CL>(one), d);
}

// A kernel's largest dynamic shared memory on the current device only grows:
// solvers on other threads may launch it with more than this call needs, and
// lowering the attribute under them would fail their launches.
cudaError_t raise_smem_attr(const void* func, int bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, int> set;  // (device, kernel) -> bytes set
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(mu);
  int& cur = set[{dev, func}];
  if (bytes <= cur) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) cur = bytes;
  return e;
}

// --------------------------------------------------------------------------
// Zero fill of many device ranges in one launch (one CTA per range of at
// most ZERO_CHUNK doubles).
// --------------------------------------------------------------------------
struct ZeroSeg {
  double* p;
  long long n;
};
constexpr long long ZERO_CHUNK = 32768;

__global__ void zero_kernel(const ZeroSeg* __restrict__ segs) {
  const ZeroSeg z = segs[blockIdx.x];
  for (long long i = threadIdx.x; i < z.n; i += blockDim.x) z.p[i] = 0.0;
}

void zero_add(std::vector<ZeroSeg>& v, double* p, long long n) {
  for (long long o = 0; o < n; o += ZERO_CHUNK) v.push_back(ZeroSeg{p + o, std::min(ZERO_CHUNK, n - o)});
}

// --------------------------------------------------------------------------
// Divide and conquer
// --------------------------------------------------------------------------
struct DcProb {
  int n;
  double* D;      // eigenvalues in progress (n)
  const double* dT;  // tridiagonal diagonal (n)
  const double* e;   // off-diagonal (n-1)
  double* Q;      // n x n (ld n): eigenvectors of T
  double* W1;     // n x n workspace
  double* U;      // n x n workspace
  double* ds;     // n sorted d (then compacted dK in [lo, lo+k))
  double* zs;     // n sorted z (then zK)
  double* dD;     // n deflated values (at [lo+k, hi))
  int* src;       // n source column of sorted position
  int* flag;      // n per sorted position: 1 = nondeflated, 0 = deflated
  double* tau;    // n
  int* orig;      // n
  double* zhat;   // n
  int* kcnt;      // n (value at index lo of a node)
  double* rho;    // n (value at index lo)
  int* rank;      // n final position
  int* rotp;      // n rotation pairs (p index)
  int* rotj;      // n
  double* rotc;   // n
  double* rots;   // n
  int* nrot;      // n (value at index lo)
};

struct DcNode {
  int prob, lo, mid, hi;
};

// Leaf: tridiagonal QR on [lo, hi) of one problem, one warp per leaf.
__global__ void __launch_bounds__(64) dc_leaf_kernel(const DcProb* __restrict__ probs,
                                                     const DcNode* __restrict__ leaves, int nleaf,
                                                     int* fail) {
  __shared__ double Zs[2][32][33];
  __shared__ double dv[2][32], ev[2][32], csv[2][4], dnv[2][32], env[2][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int li = blockIdx.x * 2 + warp;
  if (li >= nleaf) return;
  const DcNode L = leaves[li];
  const DcProb P = probs[L.prob];
  const int n = P.n, lo = L.lo, s = L.hi - L.lo;
  double* d = dv[warp];
  double* e = ev[warp];
  double(*Z)[33] = Zs[warp];
  if (lane < s) {
    double dd = P.dT[lo + lane];
    if (lane == 0 && lo > 0) dd -= fabs(P.e[lo - 1]);
    if (lane == s - 1 && L.hi < n) dd -= fabs(P.e[L.hi - 1]);
    d[lane] = dd;
    if (lane < s - 1) e[lane] = P.e[lo + lane];
  }
  for (int j = 0; j < s; ++j) Z[lane][j] = (lane == j) ? 1.0 : 0.0;
  __syncwarp();
  givens_qr_sweep_warp(d, e, Z, s, lane, csv[warp], dnv[warp], env[warp], fail);
  for (int i = 0; i < s - 1; ++i) {
    if (lane == 0) {
      int kmin = i;
      for (int k = i + 1; k < s; ++k)
        if (d[k] < d[kmin]) kmin = k;
      csv[warp][0] = (double)kmin;
      if (kmin != i) {
        const double t = d[i];
        d[i] = d[kmin];
        d[kmin] = t;
      }
    }
    __syncwarp();
    const int kmin = (int)csv[warp][0];
    if (kmin != i && lane < s) {
      const double t = Z[lane][i];
      Z[lane][i] = Z[lane][kmin];
      Z[lane][kmin] = t;
    }
    __syncwarp();
  }
  if (lane < s) P.D[lo + lane] = d[lane];
  for (int j = 0; j < s; ++j)
    if (lane < s) P.Q[(size_t)(lo + lane) + (size_t)(lo + j) * n] = Z[lane][j];
}

// Merge, step 1: z, sort, deflation, rotations, compaction.  One CTA per node.
// The sorted d and z and the deflation flags live in a work area: dynamic
// shared memory when the node has at most `cap` entries (the launch's
// shared memory holds 2 cap doubles and cap ints), else the node's slices
// of zhat, tau and flag in global memory, which are free at this point.  The
// two sequential scans (deflation, compaction order) run on the work area.
constexpr int DC_NT = 256;
constexpr int DC_PREP_CAP = 8192;  // largest node staged in shared memory (160 KB)

__host__ __device__ inline size_t dc_prep_smem(int cap) { return (size_t)cap * (2 * sizeof(double) + sizeof(int)); }

__global__ void __launch_bounds__(DC_NT) dc_prep_kernel(const DcProb* __restrict__ probs,
                                                        const DcNode* __restrict__ nodes,
                                                        GemmProb* gprob, GemmSeg* gseg, int cap) {
  extern __shared__ double dcsm[];
  __shared__ double mx[2][DC_NT / 32];
  __shared__ int sk[2];
  const DcNode N = nodes[blockIdx.x];
  const DcProb P = probs[N.prob];
  const int n = P.n, lo = N.lo, mid = N.mid, hi = N.hi;
  const int n1 = mid - lo, np = hi - lo;
  const size_t ld = (size_t)n;
  const int tid = threadIdx.x;
  const bool staged = np <= cap;
  double* wd = staged ? dcsm : P.zhat + lo;
  double* wz = staged ? dcsm + cap : P.tau + lo;
  int* wf = staged ? reinterpret_cast<int*>(dcsm + 2 * (size_t)cap) : P.flag + lo;
  const double beta = P.e[mid - 1];
  const double rho = 2.0 * fabs(beta);
  const double sgn = beta >= 0.0 ? 1.0 : -1.0;
  const double isq2 = 0.70710678118654752440;
  // sorted positions by merging the two ascending halves
  double dmax = 0.0, zmax = 0.0;
  for (int i = tid; i < np; i += DC_NT) {
    const double di = P.D[lo + i];
    double zi;
    int pos;
    if (i < n1) {
      zi = P.Q[(size_t)(mid - 1) + (size_t)(lo + i) * ld] * isq2;
      // count of second-half values strictly less than di
      int a = 0, b = np - n1;
      while (a < b) {
        const int m = (a + b) >> 1;
        if (P.D[mid + m] < di) a = m + 1; else b = m;
      }
      pos = i + a;
    } else {
      zi = sgn * P.Q[(size_t)mid + (size_t)(lo + i) * ld] * isq2;
      int a = 0, b = n1;
      while (a < b) {
        const int m = (a + b) >> 1;
        if (P.D[lo + m] <= di) a = m + 1; else b = m;
      }
      pos = (i - n1) + a;
    }
    wd[pos] = di;
    wz[pos] = zi;
    P.src[lo + pos] = i;
    dmax = fmax(dmax, fabs(di));
    zmax = fmax(zmax, fabs(zi));
  }
  // block max of |d| and |z|
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    zmax = fmax(zmax, __shfl_xor_sync(0xffffffffu, zmax, o));
  }
  if ((tid & 31) == 0) {
    mx[0][tid >> 5] = dmax;
    mx[1][tid >> 5] = zmax;
  }
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < DC_NT / 32; ++w) {
      dmax = fmax(dmax, mx[0][w]);
      zmax = fmax(zmax, mx[1][w]);
    }
    // deflation scan (sequential)
    const double tol = 8.0 * EPS * fmax(dmax, rho * zmax);
    int nr = 0, k = 0, prev = -1;
    for (int j = 0; j < np; ++j) {
      wf[j] = 0;
      if (rho * fabs(wz[j]) <= tol) continue;  // deflated by small z
      if (prev < 0) {
        prev = j;
        continue;
      }
      // |dt c s| <= tol with c = z_j / t, s = -z_p / t, t = |(z_j, z_p)|,
      // tested as |dt z_j z_p| <= tol t^2: no root or division for the
      // entries that stay (both |z| exceed tol / rho here, so t^2 is normal)
      const double zp = wz[prev], zj = wz[j];
      const double dt = wd[j] - wd[prev];
      if (fabs(dt * zj * zp) <= tol * (zj * zj + zp * zp)) {
        const double t = hypot(zj, zp);
        const double c = zj / t, s = -zp / t;
        wz[j] = t;
        wz[prev] = 0.0;
        const double dp = wd[prev], dj = wd[j];
        wd[prev] = dp * c * c + dj * s * s;
        wd[j] = dp * s * s + dj * c * c;
        P.rotp[lo + nr] = prev;
        P.rotj[lo + nr] = j;
        P.rotc[lo + nr] = c;
        P.rots[lo + nr] = s;
        ++nr;
        prev = j;  // prev deflated (flag stays 0)
      } else {
        wf[prev] = 1;
        ++k;
        prev = j;
      }
    }
    if (prev >= 0) {
      wf[prev] = 1;
      ++k;
    }
    sk[0] = k;
    sk[1] = nr;
    P.kcnt[lo] = k;
    P.rho[lo] = rho;
    P.nrot[lo] = nr;
    // compaction order: nondeflated first (in order), then deflated (in
    // order); rank holds, for now, the sorted position of each target
    int kk = 0, dd = 0;
    for (int j = 0; j < np; ++j) {
      if (wf[j]) {
        P.rank[lo + kk] = j;
        ++kk;
      } else {
        P.rank[lo + k + dd] = j;
        ++dd;
      }
    }
  }
  __syncthreads();
  const int k = sk[0];
  // compact the values out of the work area
  for (int a = tid; a < np; a += DC_NT) {
    const int j = P.rank[lo + a];
    if (a < k) {
      P.ds[lo + a] = wd[j];
      P.zs[lo + a] = wz[j];
    } else {
      P.dD[lo + a] = wd[j];
    }
  }
  // GEMM descriptor: W1[lo:hi, lo:lo+k] = Q[lo:hi, lo:lo+k] * U[lo:lo+k, lo:lo+k]
  if (tid == 0) {
    GemmProb g = gprob[blockIdx.x];  // tile0/tiles_n preset by the host
    g.C = P.W1 + lo + (size_t)lo * ld;
    g.ldc = n;
    g.m = np;
    g.n = k;
    g.beta = 0.0;
    gprob[blockIdx.x] = g;
    GemmSeg s;
    s.A = P.Q + lo + (size_t)lo * ld;
    s.lda = n;
    s.B = P.U + lo + (size_t)lo * ld;
    s.ldb = n;
    s.k = k;
    s.transA = 0;
    s.transB = 0;
    s.alpha = 1.0;
    gseg[g.seg0] = s;
  }
}

// Merge, step 2, in three launches over the node's block Q[lo:hi, lo:hi]
// (rows independent throughout):
//   gather:  W1[:, pos] = Q[:, src[pos]], the child eigenvector columns in
//            sorted order (a CTA per 128 rows x DC_PCOLS columns);
//   rotate:  the deflation rotations in order, one thread per row (nothing
//            to do when the node has none);
//   compact: Q[:, a] = W1[:, rank[a]], nondeflated columns first.
constexpr int DC_PCOLS = 8;

__global__ void dc_gather_kernel(const DcProb* __restrict__ probs, const DcNode* __restrict__ nodes, int compact) {
  const DcNode N = nodes[blockIdx.z];
  const DcProb P = probs[N.prob];
  const int lo = N.lo, np = N.hi - N.lo;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int c0 = blockIdx.y * DC_PCOLS;
  if (r >= np || c0 >= np) return;
  const size_t ld = (size_t)P.n;
  const int* map = compact ? P.rank + lo : P.src + lo;
  const double* from = (compact ? P.W1 : P.Q) + (size_t)(lo + r) + (size_t)lo * ld;
  double* to = (compact ? P.Q : P.W1) + (size_t)(lo + r) + (size_t)lo * ld;
  const int c1 = min(np, c0 + DC_PCOLS);
  for (int c = c0; c < c1; ++c) to[(size_t)c * ld] = from[(size_t)map[c] * ld];
}

__global__ void dc_rotate_kernel(const DcProb* __restrict__ probs, const DcNode* __restrict__ nodes) {
  const DcNode N = nodes[blockIdx.y];
  const DcProb P = probs[N.prob];
  const int lo = N.lo, np = N.hi - N.lo;
  const int nr = P.nrot[lo];
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (nr == 0 || r >= np) return;
  const size_t ld = (size_t)P.n;
  double* w1 = P.W1 + (size_t)(lo + r) + (size_t)lo * ld;  // row r, columns lo..hi
  for (int t = 0; t < nr; ++t) {
    const size_t pc = (size_t)P.rotp[lo + t] * ld, jc = (size_t)P.rotj[lo + t] * ld;
    const double c = P.rotc[lo + t], s = P.rots[lo + t];
    const double x = w1[pc], y = w1[jc];
    w1[pc] = c * x + s * y;
    w1[jc] = c * y - s * x;
  }
}

// Secular equation roots, one warp per root: lanes share the pole sums.
__global__ void dc_secular_warp_kernel(const DcProb* __restrict__ probs, const DcNode* __restrict__ nodes,
                                       int* fail) {
  const int node = blockIdx.y;
  const int j = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const DcNode N = nodes[node];
  const DcProb P = probs[N.prob];
  const int lo = N.lo;
  const int k = P.kcnt[lo];
  if (j >= k) return;
  const double* d = P.ds + lo;
  const double* z = P.zs + lo;
  const double rho = P.rho[lo];
  int o;
  double tlo, thi;
  if (j < k - 1) {
    const double mid = 0.5 * (d[j + 1] - d[j]);
    double f = 0.0;
    for (int i = lane; i < k; i += 32) f += z[i] * z[i] / ((d[i] - d[j]) - mid);
    f = 1.0 + rho * warp_sum(f);
    if (f >= 0.0) {
      o = j;
      tlo = 0.0;
      thi = mid;
    } else {
      o = j + 1;
      tlo = -mid;
      thi = 0.0;
    }
  } else {
    double zz = 0.0;
    for (int i = lane; i < k; i += 32) zz += z[i] * z[i];
    zz = warp_sum(zz);
    o = j;
    tlo = 0.0;
    thi = rho * zz;
  }
  const double dorig = d[o];
  const double dL = d[j] - dorig;
  const double dR = (j < k - 1) ? d[j + 1] - dorig : 0.0;
  double t = 0.5 * (tlo + thi);
  bool done = false;
  for (int it = 0; it < 400; ++it) {
    double psi = 0.0, dpsi = 0.0, phi = 0.0, dphi = 0.0;
    for (int i = lane; i < k; i += 32) {
      const double del = (d[i] - dorig) - t;
      const double q = z[i] / del;
      if (i <= j) {
        psi += z[i] * q;
        dpsi += q * q;
      } else {
        phi += z[i] * q;
        dphi += q * q;
      }
    }
    psi = warp_sum(psi);
    dpsi = warp_sum(dpsi);
    phi = warp_sum(phi);
    dphi = warp_sum(dphi);
    // all lanes hold identical sums and run the same scalar update
    const double f = 1.0 + rho * (psi + phi);
    if (f == 0.0) {
      done = true;
      break;
    }
    if (f < 0.0) tlo = t; else thi = t;
    double tn;
    const double DL = dL - t;
    if (j < k - 1) {
      const double DR = dR - t;
      const double sL = rho * dpsi * DL * DL, sR = rho * dphi * DR * DR;
      const double cc = f - sL / DL - sR / DR;
      const double bb = cc * (DL + DR) + sL + sR;
      const double c0 = DL * DR * f;
      double eta;
      if (cc == 0.0) {
        eta = c0 / bb;
      } else {
        const double sq = sqrt(fmax(bb * bb - 4.0 * cc * c0, 0.0));
        const double qq = (bb >= 0.0) ? bb + sq : bb - sq;
        const double e1 = qq / (2.0 * cc), e2 = 2.0 * c0 / qq;
        eta = (e1 > DL && e1 < DR) ? e1 : e2;
      }
      tn = t + eta;
    } else {
      const double sL = rho * dpsi * DL * DL;
      const double cc = f - sL / DL;
      tn = (cc > 0.0) ? t + DL + sL / cc : 0.5 * (tlo + thi);
    }
    if (fabs(tn - t) <= 2.0 * EPS * fabs(t) || fabs(f) <= EPS * (8.0 + 8.0 * rho * (phi - psi))) {
      done = true;
      break;
    }
    if (!(tn > tlo && tn < thi)) tn = 0.5 * (tlo + thi);
    if (thi - tlo <= 4.0 * EPS * fmax(fabs(tlo), fabs(thi))) {
      t = tn;
      done = true;
      break;
    }
    t = tn;
  }
  if (lane == 0) {
    if (!done && thi - tlo > 1e-10 * fmax(fabs(tlo), fabs(thi))) atomicExch(fail, 2);
    P.tau[lo + j] = t;
    P.orig[lo + j] = o;
  }
}

// Loewner z-hat.  One warp per i; lanes share the product over j.
__global__ void dc_lowner_kernel(const DcProb* __restrict__ probs, const DcNode* __restrict__ nodes) {
  const int node = blockIdx.y;
  const int i = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const DcNode N = nodes[node];
  const DcProb P = probs[N.prob];
  const int lo = N.lo;
  const int k = P.kcnt[lo];
  if (i >= k) return;
  const double* d = P.ds + lo;
  const double rho = P.rho[lo];
  const double di = d[i];
  auto lam_minus = [&](int j) { return (d[P.orig[lo + j]] - di) + P.tau[lo + j]; };
  double prod = 1.0;
  for (int j = lane; j < k - 1; j += 32) prod *= lam_minus(j) / ((j < i ? d[j] : d[j + 1]) - di);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) prod *= __shfl_xor_sync(0xffffffffu, prod, o);
  prod *= lam_minus(k - 1) / rho;
  if (lane == 0) P.zhat[lo + i] = copysign(sqrt(fmax(prod, 0.0)), P.zs[lo + i]);
}

// Eigenvectors of the rank-one problem.  One warp per column j.
__global__ void dc_vectors_kernel(const DcProb* __restrict__ probs, const DcNode* __restrict__ nodes) {
  const int node = blockIdx.y;
  const int j = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const DcNode N = nodes[node];
  const DcProb P = probs[N.prob];
  const int lo = N.lo;
  const int k = P.kcnt[lo];
  if (j >= k) return;
  const double* d = P.ds + lo;
  const double dor = d[P.orig[lo + j]];
  const double tj = P.tau[lo + j];
  double* col = P.U + lo + (size_t)(lo + j) * P.n;
  double ss = 0.0;
  for (int i = lane; i < k; i += 32) {
    const double u = -P.zhat[lo + i] / ((dor - d[i]) + tj);
    col[i] = u;
    ss += u * u;
  }
  ss = warp_sum(ss);
  const double inv = 1.0 / sqrt(ss);
  for (int i = lane; i < k; i += 32) col[i] *= inv;
}

// Final order: rank of every eigenvalue of the node (one warp per value,
// lanes share the comparisons); writes D and the rank.
__global__ void dc_rank_kernel(const DcProb* __restrict__ probs, const DcNode* __restrict__ nodes) {
  const int node = blockIdx.y;
  const int a = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const DcNode N = nodes[node];
  const DcProb P = probs[N.prob];
  const int lo = N.lo, np = N.hi - N.lo;
  if (a >= np) return;
  const int k = P.kcnt[lo];
  const double* d = P.ds + lo;
  auto val = [&](int b) {
    return b < k ? d[P.orig[lo + b]] + P.tau[lo + b] : P.dD[lo + b];
  };
  const double x = val(a);
  unsigned r = 0;
  for (int b = lane; b < np; b += 32) {
    const double y = val(b);
    r += (y < x) || (y == x && b < a);
  }
  r = __reduce_add_sync(0xffffffffu, r);
  if (lane == 0) {
    P.rank[lo + a] = (int)r;
    P.D[lo + r] = x;
  }
}

// Deflated columns Q[:, lo+a] (a >= k) -> W1[:, lo+a]; then all columns of
// W1 -> Q[:, lo + rank[a]].  Two launches of the same kernel (mode 0/1).
__global__ void dc_copy_kernel(const DcProb* __restrict__ probs, const DcNode* __restrict__ nodes,
                               int mode) {
  const int node = blockIdx.y;
  const int a = blockIdx.x;
  const DcNode N = nodes[node];
  const DcProb P = probs[N.prob];
  const int lo = N.lo, np = N.hi - N.lo;
  if (a >= np) return;
  const int k = P.kcnt[lo];
  const size_t ld = (size_t)P.n;
  if (mode == 0) {
    if (a < k) return;
    const double* s = P.Q + lo + (size_t)(lo + a) * ld;
    double* t = P.W1 + lo + (size_t)(lo + a) * ld;
    for (int i = threadIdx.x; i < np; i += blockDim.x) t[i] = s[i];
  } else {
    const double* s = P.W1 + lo + (size_t)(lo + a) * ld;
    double* t = P.Q + lo + (size_t)(lo + P.rank[lo + a]) * ld;
    for (int i = threadIdx.x; i < np; i += blockDim.x) t[i] = s[i];
  }
}

// --------------------------------------------------------------------------
// Back-transformation helpers
// --------------------------------------------------------------------------
struct BtProb {
  int n;
  const double* A;    // reflectors below the subdiagonal
  const double* tau;  // n-1
  double* V;          // n x n (ld n): reflector c in column c, c <= n-2
  double* G;          // nblk blocks of NBB x NBB: V_k^T V_k
  double* T;          // nblk blocks of NBB x NBB: the WY factors
};

// Reflectors of block k (columns j0 = k NBB .. j0 + nb - 1, nb <= NBB).
__host__ __device__ inline int bt_nblk(int n) { return n > 1 ? (n - 2) / NBB + 1 : 0; }

// V[:, c] = (0, .., 0, 1, A[c+2:, c]) for every reflector c of every problem
// (a CTA per column).
__global__ void bt_buildV_kernel(const BtProb* __restrict__ probs) {
  const BtProb P = probs[blockIdx.y];
  const int c = blockIdx.x;
  const int n = P.n;
  if (c > n - 2) return;
  double* col = P.V + (size_t)c * n;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double v = 0.0;
    if (i == c + 1) v = 1.0;
    else if (i > c + 1) v = P.A[i + (size_t)c * n];
    col[i] = v;
  }
}

// T of the compact WY form of the reflectors j0 .. j0+nb-1 (the dlarft
// recurrence T[0:j, j] = -tau_j T[0:j, 0:j] G[0:j, j], G = V^T V), with G and
// T in shared memory; four threads per row of T share its dot products.
constexpr int BT_T_NT = 4 * NBB;
constexpr size_t BT_T_SMEM = 2 * (size_t)NBB * (NBB + 1) * sizeof(double);

// One CTA per block k (x) of every problem (y).
__global__ void __launch_bounds__(BT_T_NT) bt_T_kernel(const BtProb* __restrict__ probs) {
  const BtProb P = probs[blockIdx.y];
  const int n = P.n;
  const int j0 = blockIdx.x * NBB;
  const int nb = min(NBB, n - 1 - j0);
  if (nb <= 0) return;
  const double* G = P.G + (size_t)blockIdx.x * NBB * NBB;
  double* T = P.T + (size_t)blockIdx.x * NBB * NBB;
  extern __shared__ double btsm[];
  double(*Ts)[NBB + 1] = reinterpret_cast<double(*)[NBB + 1]>(btsm);
  double(*Gs)[NBB + 1] = reinterpret_cast<double(*)[NBB + 1]>(btsm + NBB * (NBB + 1));
  for (int idx = threadIdx.x; idx < NBB * NBB; idx += BT_T_NT) {
    const int r = idx % NBB, c = idx / NBB;
    Ts[r][c] = 0.0;
    Gs[r][c] = G[r + c * NBB];
  }
  __syncthreads();
  const int i = threadIdx.x >> 2, q = threadIdx.x & 3;
  for (int j = 0; j < nb; ++j) {
    double acc = 0.0;
    for (int l = i + q; l < j; l += 4) acc += Ts[i][l] * Gs[l][j];
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    // column j is written here and read only from step j+1 on
    if (q == 0) {
      const double tj = P.tau[j0 + j];
      if (i < j) Ts[i][j] = -tj * acc;
      else if (i == j) Ts[j][j] = tj;
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < NBB * NBB; idx += BT_T_NT) {
    const int r = idx % NBB, c = idx / NBB;
    T[r + c * NBB] = Ts[r][c];
  }
}

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }

// Host helper that batches GEMM problems and launches them.
// Launch descriptors of several launches gathered on the host and sent to
// the device in one copy (instead of one small copy per launch).
class DescPack {
 public:
  template <class T>
  size_t add(const std::vector<T>& v) {
    const size_t off = (buf_.size() + 255) & ~size_t(255);
    buf_.resize(off + v.size() * sizeof(T));
    if (!v.empty()) memcpy(buf_.data() + off, v.data(), v.size() * sizeof(T));
    return off;
  }
  // device copy (stream-ordered); offsets from add() index into it
  char* upload(DeviceArena& arena, cudaStream_t st) {
    char* dev = static_cast<char*>(arena.alloc(buf_.size() + 256));
    if (!buf_.empty()) NRGB_CUDA(cudaMemcpyAsync(dev, buf_.data(), buf_.size(), cudaMemcpyHostToDevice, st));
    return dev;
  }

 private:
  std::vector<char> buf_;
};

struct GemmBatch {
  std::vector<GemmProb> probs;
  std::vector<GemmSeg> segs;
  int tiles = 0, stiles = 0;
  void add(double* C, int ldc, int m, int n, double beta, const std::vector<GemmSeg>& ss, int ksplit = 1) {
    if (m <= 0 || n <= 0) return;
    GemmProb p{};
    p.ksplit = ksplit;
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
  bool empty() const { return probs.empty(); }
};

}  // namespace

// ------------------------------------------------------------------------
// host orchestration
// ------------------------------------------------------------------------

SyevBatched::SyevBatched() {
  NRGB_CUDA(cudaMalloc(&d_err_, 4 * sizeof(int)));
  NRGB_CUDA(cudaMalloc(&d_bar_, sizeof(GridBarrier)));
  int dev = 0;
  NRGB_CUDA(cudaGetDevice(&dev));
  NRGB_CUDA(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev));
  int optin = 0;
  NRGB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cl_smem_ = std::min(TRDC_SMEM, (size_t)optin);
  // NRGB_TRD_PATH=panel keeps every block on the cooperative panel path
  // (comparisons, or a device where cluster launches are unavailable)
  const char* path = getenv("NRGB_TRD_PATH");
  if (path && strcmp(path, "panel") == 0) cl_smem_ = 0;
  // the cluster kernel (default: one barrier per column); for comparisons
  // NRGB_TRDC_BARRIERS=2 selects the form with two cluster barriers per
  // column and NRGB_TRDC_FUSED=1 the one-barrier form with the update and
  // the next products fused (faster for a block alone, slower when many
  // clusters run at once)
  const char* nb = getenv("NRGB_TRDC_BARRIERS");
  const char* nf = getenv("NRGB_TRDC_FUSED");
  cl_one_ = (nb && strcmp(nb, "2") == 0) ? 0 : (nf && strcmp(nf, "1") == 0) ? 2 : 1;
  // NRGB_TRDC_POW2=1 restricts the default kernel to clusters of 1, 2, 4, 8
  // and 16 CTAs (comparisons); otherwise a block takes the smallest cluster
  // of any size that holds it
  const char* np2 = getenv("NRGB_TRDC_POW2");
  const bool pow2 = np2 && strcmp(np2, "1") == 0;
  if (cl_smem_ > 0) {
    for (int cl = 1; cl <= TRDC_CL_MAX; ++cl) {
      if (!trdc_size_built(cl_one_, cl) || (pow2 && (cl & (cl - 1)) != 0)) continue;
      cl_max_[cl] = trdc_with_cl(cl, [&](auto c) { return trdc_max_clusters<decltype(c)::value>(cl_one_, cl_smem_); });
    }
  }
  // largest block the cluster kernel holds (the one-barrier kernels also
  // read at most TRDC1_ROWS rows of a column per thread)
  for (int cl = TRDC_CL_MAX; cl >= 1 && cl_nmax_ == 0; --cl) {
    if (cl_max_[cl] <= 0) continue;
    int n = 1;
    while (trdc_bytes(n + 1, cl) <= cl_smem_ && (!cl_one_ || n + 1 <= TRDC1_ROWS * TRDC1_NT)) ++n;
    cl_nmax_ = n > SMALL_N ? n : 0;
  }
  // one side stream per launch group of the cluster kernel (up to 19
  // groups: single-CTA launches in four shared-memory sizes and one per
  // cluster size), so that no group waits behind another on a shared stream
  if (const char* ns = getenv("NRGB_SIDE_STREAMS")) naux_ = std::max(1, std::min(NAUX, atoi(ns)));
  for (int i = 0; i < NAUX; ++i) {
    NRGB_CUDA(cudaStreamCreateWithFlags(&aux_[i], cudaStreamNonBlocking));
    NRGB_CUDA(cudaEventCreateWithFlags(&join_[i], cudaEventDisableTiming));
  }
  NRGB_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
  NRGB_CUDA(cudaStreamCreateWithFlags(&small_st_, cudaStreamNonBlocking));
  NRGB_CUDA(cudaEventCreateWithFlags(&small_done_, cudaEventDisableTiming));
}

SyevBatched::~SyevBatched() {
  if (d_err_) cudaFree(d_err_);
  if (d_bar_) cudaFree(d_bar_);
  for (int i = 0; i < NAUX; ++i) {
    if (aux_[i]) cudaStreamDestroy(aux_[i]);
    if (join_[i]) cudaEventDestroy(join_[i]);
  }
  if (fork_) cudaEventDestroy(fork_);
  if (small_done_) cudaEventDestroy(small_done_);
  if (small_st_) cudaStreamDestroy(small_st_);
}

namespace {
struct Plan {
  std::vector<int> small, big;
};

void plan_tree(int prob, int lo, int hi, std::vector<DcNode>& leaves,
               std::vector<std::pair<int, DcNode>>& merges, int& height) {
  if (hi - lo <= LEAF) {
    leaves.push_back(DcNode{prob, lo, lo, hi});
    height = 0;
    return;
  }
  const int mid = lo + (hi - lo) / 2;
  int h1, h2;
  plan_tree(prob, lo, mid, leaves, merges, h1);
  plan_tree(prob, mid, hi, leaves, merges, h2);
  height = std::max(h1, h2) + 1;
  merges.push_back({height, DcNode{prob, lo, mid, hi}});
}
}  // namespace

size_t SyevBatched::workspace_bytes(const std::vector<int>& ns) {
  ArenaPlan pl;
  for (int n : ns) {
    if (n <= SMALL_N) continue;
    const size_t nn = (size_t)n * n;
    pl.add<double>(nn);   // W1
    pl.add<double>(nn);   // U
    pl.add<double>((size_t)n * NB * 2);
    pl.add<double>((size_t)n * 16);
    pl.add<int>((size_t)n * 10);
    pl.add<double>(2 * RED);
    pl.add<double>((size_t)NBB * NBB * std::max(1, bt_nblk(n)));  // G
    pl.add<double>((size_t)NBB * NBB * std::max(1, bt_nblk(n)));  // T
    pl.add<double>((size_t)NBB * n * 2);                          // X (last block), Y
  }
  pl.add<double>(64 * 1024);
  int nmx = 0;
  for (int n : ns) nmx = std::max(nmx, n);
  // per-panel launch descriptors
  pl.add<char>((size_t)(nmx / NB + 2) * (ns.size() * (sizeof(TrdProb) + 2 * sizeof(GemmSeg) + sizeof(GemmProb)) + 2048));
  // zero-fill descriptors: the per-problem buffers once, the split-K
  // outputs of the back-transformation once; cluster descriptors
  size_t zs = 0;
  for (int n : ns)
    zs += 6 + (size_t)n * n / ZERO_CHUNK + (size_t)NBB * NBB * bt_nblk(n) / ZERO_CHUNK +
          (NBB * (size_t)n / ZERO_CHUNK + 2) * (n / NBB + 3);
  pl.add<ZeroSeg>(zs);
  // divide-and-conquer descriptors (one copy): problems, leaves, and per
  // merge node a node, a GEMM problem and a segment; 3 aligned arrays per level
  size_t ndc = 0;
  for (int n : ns) ndc += 2 * (size_t)(n / LEAF + 2);
  pl.add<char>(ns.size() * sizeof(DcProb) + ndc * (sizeof(DcNode) + sizeof(GemmProb) + sizeof(GemmSeg)) +
               256 * 3 * 40 + 1024);
  // back-transformation GEMM descriptors (4 batches per block of reflectors)
  size_t nbt = 0;
  for (int n : ns) nbt += 4 * (size_t)(bt_nblk(n) + 1);
  pl.add<char>(ns.size() * sizeof(BtProb) + nbt * (sizeof(GemmProb) + sizeof(GemmSeg)) +
               256 * 6 * (size_t)(nmx / NBB + 4));
  pl.add<TrdClProb>(2 * ns.size() + 16);
  return pl.bytes + (size_t)ns.size() * 4096 + (1 << 20);
}

size_t SyevBatched::trdc_bytes(int n, int cl) const {
  return (cl_one_ == 2 ? trdc2_smem_doubles(n, cl) : cl_one_ == 1 ? trdc1_smem_doubles(n, cl)
                                                                   : trdc_smem_doubles(n, cl)) *
         sizeof(double);
}

int SyevBatched::cl_use() const {
  const int lim = schedule_here().cluster_limit.load(std::memory_order_relaxed);
  return (lim > 0 && lim < cl_nmax_) ? lim : cl_nmax_;
}

void SyevBatched::run(const std::vector<SyevDesc>& probs, cudaStream_t st) {
  launches_ = 0;
  NRGB_CUDA(cudaMemsetAsync(d_err_, 0, 4 * sizeof(int), st));
  NRGB_CUDA(cudaMemsetAsync(d_bar_, 0, sizeof(GridBarrier), st));
  std::vector<int> small, big;
  for (int i = 0; i < (int)probs.size(); ++i) {
    if (probs[i].n <= 0) continue;
    (probs[i].n <= SMALL_N ? small : big).push_back(i);
  }
  std::vector<int> ns;
  for (int i : big) ns.push_back(probs[i].n);
  // plus descriptor storage
  const size_t need = workspace_bytes(ns) + probs.size() * 512 + (1 << 20);
  if (arena_.capacity() < need) {
    NRGB_CUDA(cudaStreamSynchronize(st));
    arena_.reserve(need + need / 4);
  }
  arena_.reset();

  // ---------------- small problems ----------------
  if (!small.empty()) {
    std::vector<SmallProb> sp;
    for (int i : small) sp.push_back(SmallProb{probs[i].A, probs[i].w, probs[i].Z, probs[i].n});
    SmallProb* d_sp = arena_.alloc_n<SmallProb>(sp.size());
    NRGB_CUDA(cudaMemcpyAsync(d_sp, sp.data(), sp.size() * sizeof(SmallProb), cudaMemcpyHostToDevice, st));
    // on its own stream, beside the larger blocks; joined before the flags are read
    NRGB_CUDA(cudaEventRecord(fork_, st));
    NRGB_CUDA(cudaStreamWaitEvent(small_st_, fork_, 0));
    NRGB_LAUNCH("syev_small", small_st_,
                syev_small_kernel<<<ceil_div((int)sp.size(), SMALL_WARPS), 32 * SMALL_WARPS, 0, small_st_>>>(
                    d_sp, (int)sp.size(), d_err_));
    NRGB_CUDA(cudaGetLastError());
    NRGB_CUDA(cudaEventRecord(small_done_, small_st_));
    ++launches_;
  }

  if (!big.empty()) {
    const int nbig = (int)big.size();
    int nmax = 0;
    for (int i : big) nmax = std::max(nmax, probs[i].n);
    // per-problem workspaces
    std::vector<TrdProb> tp(nbig);
    std::vector<DcProb> dp(nbig);
    std::vector<BtProb> bp(nbig);
    std::vector<double*> dT(nbig), eT(nbig), tauT(nbig), bt_X(nbig), bt_Y(nbig);
    std::vector<ZeroSeg> zeros;  // ranges that must start at zero, cleared in one launch
    for (int b = 0; b < nbig; ++b) {
      const SyevDesc& S = probs[big[b]];
      const int n = S.n;
      const size_t nn = (size_t)n * n;
      double* W1 = arena_.alloc_n<double>(nn);
      double* U = arena_.alloc_n<double>(nn);
      double* Vp = arena_.alloc_n<double>((size_t)n * NB);
      double* Wp = arena_.alloc_n<double>((size_t)n * NB);
      double* vec = arena_.alloc_n<double>((size_t)n * 16);
      int* ivec = arena_.alloc_n<int>((size_t)n * 10);
      double* red = arena_.alloc_n<double>(2 * RED);
      const int nblk = std::max(1, bt_nblk(n));
      double* G = arena_.alloc_n<double>((size_t)NBB * NBB * nblk);
      double* T = arena_.alloc_n<double>((size_t)NBB * NBB * nblk);
      bt_X[b] = arena_.alloc_n<double>((size_t)NBB * n);
      bt_Y[b] = arena_.alloc_n<double>((size_t)NBB * n);
      dT[b] = vec;
      eT[b] = vec + n;
      tauT[b] = vec + 2 * n;
      TrdProb& t = tp[b];
      t.A = S.A;
      t.d = dT[b];
      t.e = eT[b];
      t.tau = tauT[b];
      t.Vp = Vp;
      t.W = Wp;
      t.v = vec + 3 * n;
      t.y = vec + 4 * n;
      t.red = red;
      t.n = n;
      DcProb& q = dp[b];
      q.n = n;
      q.D = S.w;
      q.dT = dT[b];
      q.e = eT[b];
      q.Q = S.Z;
      q.W1 = W1;
      q.U = U;
      q.ds = vec + 5 * n;
      q.zs = vec + 6 * n;
      q.dD = vec + 7 * n;
      q.tau = vec + 8 * n;
      q.zhat = vec + 9 * n;
      q.rho = vec + 10 * n;
      q.rotc = vec + 11 * n;
      q.rots = vec + 12 * n;
      q.src = ivec;
      q.flag = ivec + n;
      q.orig = ivec + 2 * n;
      q.kcnt = ivec + 3 * n;
      q.rank = ivec + 4 * n;
      q.rotp = ivec + 5 * n;
      q.rotj = ivec + 6 * n;
      q.nrot = ivec + 7 * n;
      BtProb& bt = bp[b];
      bt.n = n;
      bt.A = S.A;
      bt.tau = tauT[b];
      bt.V = W1;  // free once divide and conquer is done
      bt.G = G;
      bt.T = T;
      zero_add(zeros, red, 2 * RED);
      zero_add(zeros, tauT[b], n);
      zero_add(zeros, S.Z, (long long)nn);
    }
    if (!zeros.empty()) {
      ZeroSeg* d_z = arena_.alloc_n<ZeroSeg>(zeros.size());
      NRGB_CUDA(cudaMemcpyAsync(d_z, zeros.data(), zeros.size() * sizeof(ZeroSeg), cudaMemcpyHostToDevice, st));
      NRGB_LAUNCH("zero_fill", st, zero_kernel<<<(unsigned)zeros.size(), 256, 0, st>>>(d_z));
      NRGB_CUDA(cudaGetLastError());
      ++launches_;
    }
    // ---------------- 1) tridiagonalisation ----------------
    // Blocks whose matrix fits in the shared memory of a cluster of at most
    // 16 CTAs: one cluster each (smallest cluster that holds the block).
    // Launches of different cluster sizes (and, for single-CTA clusters, of
    // different shared-memory sizes, so that small blocks share an SM) run
    // concurrently on side streams; the panel launches for the larger
    // blocks follow on the main stream.
    std::vector<char> via_cluster(nbig, 0);
    // Launch the cluster tridiagonalisation for `list`: groups by cluster size
    // (the smallest cluster whose shared memory holds the block; single-CTA
    // clusters split at n = 64, 96, 128), concurrently on side streams,
    // joined into `st`.  Every entry must fit some cluster size.
    auto launch_clusters = [&](const std::vector<TrdClProb>& list) {
      constexpr int NG = TRDC_CL_MAX + 3;  // group 0..3: one CTA; group CL + 2: CL CTAs
      std::vector<TrdClProb> grp[NG];
      size_t gsmem[NG] = {};
      for (const TrdClProb& t : list) {
        const int n = t.n;
        for (int cl = 1; cl <= TRDC_CL_MAX; ++cl) {
          const size_t bytes = trdc_bytes(n, cl);
          if (cl_max_[cl] > 0 && bytes <= cl_smem_) {
            const int g = cl > 1 ? cl + 2 : (n <= 64 ? 0 : n <= 96 ? 1 : n <= 128 ? 2 : 3);
            grp[g].push_back(t);
            gsmem[g] = std::max(gsmem[g], bytes);
            break;
          }
        }
      }
      int used = 0;
      TrdClProb* dg[NG] = {};
      for (int g = NG - 1; g >= 0; --g) {
        if (grp[g].empty()) continue;
        dg[g] = arena_.alloc_n<TrdClProb>(grp[g].size());
        NRGB_CUDA(cudaMemcpyAsync(dg[g], grp[g].data(), grp[g].size() * sizeof(TrdClProb), cudaMemcpyHostToDevice, st));
      }
      NRGB_CUDA(cudaEventRecord(fork_, st));
      for (int g = NG - 1; g >= 0; --g) {
        if (grp[g].empty()) continue;
        cudaStream_t sx = aux_[used % naux_];
        if (used < naux_) NRGB_CUDA(cudaStreamWaitEvent(sx, fork_, 0));
        double fl = 0, by = 0;
        for (const TrdClProb& t : grp[g]) {
          fl += 4.0 / 3.0 * (double)t.n * t.n * t.n;
          by += 8.0 * (double)t.n * t.n;  // the block, read from HBM once
        }
        KernelStats::get().add_work("trd_cluster", fl);
        KernelStats::get().add_work("trd_cluster_hbm", by);
        const int np = (int)grp[g].size();
        const int cl = g > 3 ? g - 2 : 1;
        cudaError_t e = cudaSuccess;
        NRGB_LAUNCH("trd_cluster", sx, e = trdc_with_cl(cl, [&](auto c) {
                      return trdc_launch<decltype(c)::value>(cl_one_, dg[g], np, gsmem[g], sx);
                    }));
        NRGB_CUDA(e);
        ++launches_;
        ++used;
      }
      for (int i = 0; i < std::min(used, naux_); ++i) {
        NRGB_CUDA(cudaEventRecord(join_[i], aux_[i]));
        NRGB_CUDA(cudaStreamWaitEvent(st, join_[i], 0));
      }
    };
    // Larger blocks: panel launches for their leading columns until the
    // trailing block fits a cluster, whose tridiagonalisation finishes it.
    std::vector<int> jstop(nbig);
    const int clim = cl_use();
    {
      std::vector<TrdClProb> whole;
      for (int b = 0; b < nbig; ++b) {
        const int n = tp[b].n;
        jstop[b] = n;
        if (clim > 0 && n <= clim) {
          whole.push_back(TrdClProb{tp[b].A, tp[b].d, tp[b].e, tp[b].tau, n, n});
          via_cluster[b] = 1;
        } else if (clim > 0) {
          jstop[b] = ((n - clim + NB - 1) / NB) * NB;
        }
      }
      launch_clusters(whole);
    }
    {
      const size_t smem = (size_t)(32 + 4 * NB + 8 + (TRD_NT / 32) * 2 * NB + nmax) * sizeof(double);
      NRGB_CUDA(raise_smem_attr((const void*)trd_panel_kernel, (int)smem));
      int per_sm = 0;
      NRGB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trd_panel_kernel, TRD_NT, smem));
      per_sm = std::max(1, std::min(per_sm, 4));
      const int cap = per_sm * sms_;
      // One cooperative launch per panel of NB columns.  All problems advance
      // column by column in lockstep, so a column costs the maximum over
      // problems of (trailing size)^2 / CTAs: the CTAs of each launch are
      // shared among the problems that still have columns left in
      // proportion to (n - j0)^2, and finished problems get none.
      std::vector<int> order(nbig);
      std::iota(order.begin(), order.end(), 0);
      GridBarrier* bars = arena_.alloc_n<GridBarrier>(nbig);
      for (int j0 = 0; j0 < nmax; j0 += NB) {
        std::vector<int> act;
        for (int b : order)
          if (tp[b].n > j0 && !via_cluster[b] && j0 < jstop[b]) act.push_back(b);
        for (size_t s0 = 0; s0 < act.size(); s0 += cap) {
          const size_t s1 = std::min(act.size(), s0 + cap);
          const int cnt = (int)(s1 - s0);
          double wsum = 0.0;
          for (size_t q = s0; q < s1; ++q) wsum += pow((double)(tp[act[q]].n - j0), 2.0);
          const int extra = cap - cnt;
          std::vector<TrdProb> sub;
          int tot = 0;
          NRGB_CUDA(cudaMemsetAsync(bars, 0, sizeof(GridBarrier) * nbig, st));
          for (size_t q = s0; q < s1; ++q) {
            TrdProb t = tp[act[q]];
            t.bar = bars + act[q];
            t.wait_log2 = wait_log2_;
            t.expect_extra = inject_shortfall_ ? 1 : 0;
            const double w = pow((double)(t.n - j0), 2.0) / wsum;
            int nc = 1 + (int)floor(w * extra);
            nc = std::min(nc, std::max(1, (t.n - j0) / 8));
            t.cta0 = tot;
            t.ncta = nc;
            tot += nc;
            sub.push_back(t);
          }
          TrdProb* d_tp = arena_.alloc_n<TrdProb>(sub.size());
          NRGB_CUDA(cudaMemcpyAsync(d_tp, sub.data(), sub.size() * sizeof(TrdProb), cudaMemcpyHostToDevice, st));
          int np_ = cnt;
          int j0_ = j0;
          int* fail = d_err_ + 3;
          void* args[] = {(void*)&d_tp, (void*)&np_, (void*)&j0_, (void*)&fail};
          {
            // algorithmic bytes: column c reads its trailing (n-c-1)^2 block once
            double wb = 0;
            for (const TrdProb& t : sub)
              for (int c = j0; c < std::min(j0 + NB, t.n - 1); ++c) wb += 8.0 * (double)(t.n - c - 1) * (t.n - c - 1);
            KernelStats::get().add_work("trd_panel", wb);
          }
          NRGB_LAUNCH("trd_panel", st,
                      NRGB_CUDA(cudaLaunchCooperativeKernel((void*)trd_panel_kernel, dim3(tot), dim3(TRD_NT),
                                                            args, smem, st)));
          ++launches_;
          // trailing update A22 -= V W^T + W V^T for rows/cols >= j0+NB
          GemmBatch gb;
          for (const TrdProb& t : sub) {
            const int n = t.n;
            const int r0 = j0 + NB;
            if (r0 >= n) continue;
            const int m2 = n - r0;
            // Vp, W are row-major n x NB: as column-major matrices they are
            // NB x n with ld NB, so op(A) = stored^T and op(B) = stored.
            GemmSeg s1{}, s2{};
            s1.A = t.Vp + (size_t)r0 * NB;
            s1.lda = NB;
            s1.B = t.W + (size_t)r0 * NB;
            s1.ldb = NB;
            s1.k = NB;
            s1.transA = 1;
            s1.transB = 0;
            s1.alpha = -1.0;
            s2 = s1;
            s2.A = t.W + (size_t)r0 * NB;
            s2.B = t.Vp + (size_t)r0 * NB;
            gb.add(t.A + r0 + (size_t)r0 * n, n, m2, m2, 1.0, {s1, s2});
          }
          if (!gb.empty()) {
            GemmProb* d_gp = arena_.alloc_n<GemmProb>(gb.probs.size());
            GemmSeg* d_gs = arena_.alloc_n<GemmSeg>(gb.segs.size());
            NRGB_CUDA(cudaMemcpyAsync(d_gp, gb.probs.data(), gb.probs.size() * sizeof(GemmProb),
                                      cudaMemcpyHostToDevice, st));
            NRGB_CUDA(cudaMemcpyAsync(d_gs, gb.segs.data(), gb.segs.size() * sizeof(GemmSeg),
                                      cudaMemcpyHostToDevice, st));
            KernelStats::get().add_work("gemm_f64_trailing",
                                        gemm_flops(gb.probs.data(), (int)gb.probs.size(), gb.segs.data()));
            NRGB_CUDA(gemm_grouped_launch(d_gp, (int)gb.probs.size(), d_gs, gb.tiles, st, "gemm_f64_trailing", gb.stiles));
            ++launches_;
          }
        }
      }
    }
    if (inject_shortfall_) {
      // fault injection (the barriers expected a CTA that was never
      // launched): report the timed-out wait here, before any later stage
      // reads the unfinished reduction, and leave no work of this call in
      // flight on any stream
      int f = 0;
      NRGB_CUDA(cudaMemcpyAsync(&f, d_err_ + 3, sizeof(int), cudaMemcpyDeviceToHost, st));
      NRGB_CUDA(cudaStreamSynchronize(st));
      if (small_st_) NRGB_CUDA(cudaStreamSynchronize(small_st_));
      for (int i = 0; i < NAUX; ++i)
        if (aux_[i]) NRGB_CUDA(cudaStreamSynchronize(aux_[i]));
      if (f) throw CudaError("syev: grid barrier timed out");
    }
    // the trailing blocks A[j:, j:] (j = jstop) of the larger blocks, fully
    // updated by the last trailing update, tridiagonalised in clusters
    {
      std::vector<TrdClProb> tails;
      for (int b = 0; b < nbig; ++b) {
        const int j = jstop[b], n = tp[b].n;
        if (via_cluster[b] || j >= n) continue;
        tails.push_back(TrdClProb{tp[b].A + j + (size_t)j * n, tp[b].d + j, tp[b].e + j, tp[b].tau + j, n - j, n});
      }
      launch_clusters(tails);
    }
    // ---------------- 2) divide and conquer ----------------
    // Leaves in one launch, then the merges level by level (all problems'
    // nodes of a level together); every level's descriptors go to the
    // device in one copy up front.
    {
      std::vector<DcNode> leaves;
      std::vector<std::pair<int, DcNode>> merges;
      int hmax = 0;
      for (int b = 0; b < nbig; ++b) {
        int h;
        plan_tree(b, 0, dp[b].n, leaves, merges, h);
        hmax = std::max(hmax, h);
      }
      struct Level {
        std::vector<DcNode> nodes;
        GemmBatch gb;
        int maxnp = 0;
        size_t o_nodes = 0, o_gp = 0, o_gs = 0;
      };
      std::vector<Level> levels(hmax + 1);
      for (auto& m : merges) levels[m.first].nodes.push_back(m.second);
      DescPack pk;
      const size_t o_dp = pk.add(dp);
      const size_t o_leaves = pk.add(leaves);
      for (int h = 1; h <= hmax; ++h) {
        Level& L = levels[h];
        for (auto& nd : L.nodes) {
          const int np = nd.hi - nd.lo;
          L.maxnp = std::max(L.maxnp, np);
          GemmSeg sg{};
          L.gb.add(nullptr, 0, np, np, 0.0, {sg});  // shapes fixed on device (n = k <= np)
        }
        // segments too, even though dc_prep fills them in: the copy sizes them
        L.o_nodes = pk.add(L.nodes);
        L.o_gp = pk.add(L.gb.probs);
        L.o_gs = pk.add(L.gb.segs);
      }
      char* dev = pk.upload(arena_, st);
      const DcProb* d_dp = reinterpret_cast<const DcProb*>(dev + o_dp);
      NRGB_LAUNCH("dc_leaf", st,
                  dc_leaf_kernel<<<ceil_div((int)leaves.size(), 2), 64, 0, st>>>(
                      d_dp, reinterpret_cast<const DcNode*>(dev + o_leaves), (int)leaves.size(), d_err_ + 1));
      NRGB_CUDA(cudaGetLastError());
      ++launches_;
      NRGB_CUDA(raise_smem_attr((const void*)dc_prep_kernel, (int)dc_prep_smem(DC_PREP_CAP)));
      for (int h = 1; h <= hmax; ++h) {
        Level& L = levels[h];
        if (L.nodes.empty()) continue;
        const int nn = (int)L.nodes.size();
        const int maxnp = L.maxnp;
        const DcNode* d_nodes = reinterpret_cast<const DcNode*>(dev + L.o_nodes);
        GemmProb* d_gp = reinterpret_cast<GemmProb*>(dev + L.o_gp);
        GemmSeg* d_gs = reinterpret_cast<GemmSeg*>(dev + L.o_gs);
        const int cap = maxnp <= DC_PREP_CAP ? maxnp : 0;
        NRGB_LAUNCH("dc_prep", st,
                    dc_prep_kernel<<<nn, DC_NT, dc_prep_smem(cap), st>>>(d_dp, d_nodes, d_gp, d_gs, cap));
        NRGB_CUDA(cudaGetLastError());
        dim3 g1(ceil_div(maxnp, 128), nn);
        dim3 gp(ceil_div(maxnp, 128), ceil_div(maxnp, DC_PCOLS), nn);
        NRGB_LAUNCH("dc_permute", st, dc_gather_kernel<<<gp, 128, 0, st>>>(d_dp, d_nodes, 0));
        NRGB_CUDA(cudaGetLastError());
        NRGB_LAUNCH("dc_permute", st, dc_rotate_kernel<<<g1, 128, 0, st>>>(d_dp, d_nodes));
        NRGB_CUDA(cudaGetLastError());
        NRGB_LAUNCH("dc_permute", st, dc_gather_kernel<<<gp, 128, 0, st>>>(d_dp, d_nodes, 1));
        NRGB_CUDA(cudaGetLastError());
        dim3 gw(ceil_div(maxnp, 8), nn);
        NRGB_LAUNCH("dc_secular", st, dc_secular_warp_kernel<<<gw, 256, 0, st>>>(d_dp, d_nodes, d_err_ + 2));
        NRGB_CUDA(cudaGetLastError());
        NRGB_LAUNCH("dc_lowner", st, dc_lowner_kernel<<<gw, 256, 0, st>>>(d_dp, d_nodes));
        NRGB_CUDA(cudaGetLastError());
        dim3 g2(ceil_div(maxnp, 8), nn);
        NRGB_LAUNCH("dc_vectors", st, dc_vectors_kernel<<<g2, 256, 0, st>>>(d_dp, d_nodes));
        NRGB_CUDA(cudaGetLastError());
        NRGB_CUDA(gemm_grouped_launch(d_gp, nn, d_gs, L.gb.tiles, st, "gemm_f64_dc", L.gb.stiles));
        NRGB_LAUNCH("dc_rank", st, dc_rank_kernel<<<gw, 256, 0, st>>>(d_dp, d_nodes));
        NRGB_CUDA(cudaGetLastError());
        dim3 g3(maxnp, nn);
        NRGB_LAUNCH("dc_copy", st, dc_copy_kernel<<<g3, 128, 0, st>>>(d_dp, d_nodes, 0));
        NRGB_CUDA(cudaGetLastError());
        NRGB_LAUNCH("dc_copy", st, dc_copy_kernel<<<g3, 128, 0, st>>>(d_dp, d_nodes, 1));
        NRGB_CUDA(cudaGetLastError());
        launches_ += 11;
      }
      // problems that are a single leaf already have D, Q in place
    }
    // ---------------- 3) back-transformation ----------------
    // Z = H_0 H_1 ... H_{n-2} Z in blocks of NBB reflectors, last block
    // first: Z[r0:, :] -= V_k T_k (V_k^T Z[r0:, :]).  V (all reflectors, in
    // W1), every G_k = V_k^T V_k and every T_k are formed up front in four
    // launches; then three GEMMs per block.  Split-K outputs X_k live in
    // their own slots (U, free after divide and conquer, holds blocks
    // k with (k+1) NBB <= n; the last block uses X), zeroed once.  All
    // descriptors go to the device in one copy.
    {
      int kmax = 0;
      for (int b = 0; b < nbig; ++b) kmax = std::max(kmax, bt_nblk(bp[b].n));
      auto xslot = [&](int b, int k) {
        const int n = bp[b].n;
        return (k + 1) * NBB <= n ? dp[b].U + (size_t)k * NBB * n : bt_X[b];
      };
      auto xsplit = [](int mrows) { return std::max(1, std::min(16, mrows / 128)); };
      auto gsplit = [](int mrows) { return std::max(1, std::min(16, mrows / 256)); };
      std::vector<ZeroSeg> bz;
      GemmBatch gg;  // every G_k
      for (int b = 0; b < nbig; ++b) {
        const BtProb& P = bp[b];
        const int n = P.n;
        for (int k = 0; k < bt_nblk(n); ++k) {
          const int j0 = k * NBB, nb = std::min(NBB, n - 1 - j0), r0 = j0 + 1, mrows = n - r0;
          GemmSeg s{};
          s.A = P.V + r0 + (size_t)j0 * n;
          s.lda = n;
          s.transA = 1;
          s.B = s.A;
          s.ldb = n;
          s.transB = 0;
          s.k = mrows;
          s.alpha = 1.0;
          const int kg = gsplit(mrows);
          double* Gk = P.G + (size_t)k * NBB * NBB;
          if (kg > 1) zero_add(bz, Gk, (long long)NBB * NBB);
          gg.add(Gk, NBB, nb, nb, 0.0, {s}, kg);
          if (xsplit(mrows) > 1) zero_add(bz, xslot(b, k), (long long)NBB * n);
        }
      }
      // per block k (descending): X_k = V_k^T Z, Y = T_k X_k, Z -= V_k Y
      struct Step {
        GemmBatch gx, gy, gz;
      };
      std::vector<Step> steps(kmax);
      for (int k = kmax - 1; k >= 0; --k) {
        Step& S = steps[k];
        for (int b = 0; b < nbig; ++b) {
          const BtProb& P = bp[b];
          const int n = P.n;
          if (k >= bt_nblk(n)) continue;
          const int j0 = k * NBB, nb = std::min(NBB, n - 1 - j0), r0 = j0 + 1, mrows = n - r0;
          double* Z = probs[big[b]].Z;
          double* Xk = xslot(b, k);
          GemmSeg s{};
          s.A = P.V + r0 + (size_t)j0 * n;
          s.lda = n;
          s.transA = 1;
          s.B = Z + r0;
          s.ldb = n;
          s.transB = 0;
          s.k = mrows;
          s.alpha = 1.0;
          S.gx.add(Xk, NBB, nb, n, 0.0, {s}, xsplit(mrows));
          GemmSeg t{};
          t.A = P.T + (size_t)k * NBB * NBB;
          t.lda = NBB;
          t.transA = 0;
          t.B = Xk;
          t.ldb = NBB;
          t.transB = 0;
          t.k = nb;
          t.alpha = 1.0;
          S.gy.add(bt_Y[b], NBB, nb, n, 0.0, {t});
          GemmSeg u{};
          u.A = P.V + r0 + (size_t)j0 * n;
          u.lda = n;
          u.transA = 0;
          u.B = bt_Y[b];
          u.ldb = NBB;
          u.transB = 0;
          u.k = nb;
          u.alpha = -1.0;
          S.gz.add(Z + r0, n, mrows, n, 1.0, {u});
        }
      }
      // one upload: problems, zero ranges, then the GEMM batches
      DescPack pk;
      const size_t o_bp = pk.add(bp);
      const size_t o_bz = pk.add(bz);
      std::vector<std::pair<size_t, size_t>> og;  // (probs, segs) offsets, batch order below
      auto put = [&](const GemmBatch& g) { og.push_back({pk.add(g.probs), pk.add(g.segs)}); };
      put(gg);
      for (int k = kmax - 1; k >= 0; --k) {
        put(steps[k].gx);
        put(steps[k].gy);
        put(steps[k].gz);
      }
      char* dev = pk.upload(arena_, st);
      const BtProb* d_bp = reinterpret_cast<const BtProb*>(dev + o_bp);
      size_t gi = 0;
      auto gemm = [&](const GemmBatch& g) {
        const std::pair<size_t, size_t> o = og[gi++];
        if (g.empty()) return;
        KernelStats::get().add_work("gemm_f64_bt", gemm_flops(g.probs.data(), (int)g.probs.size(), g.segs.data()));
        NRGB_CUDA(gemm_grouped_launch(reinterpret_cast<const GemmProb*>(dev + o.first), (int)g.probs.size(),
                                      reinterpret_cast<const GemmSeg*>(dev + o.second), g.tiles, st, "gemm_f64_bt",
                                      g.stiles));
        ++launches_;
      };
      if (kmax > 0) {
        NRGB_LAUNCH("bt_buildV", st, bt_buildV_kernel<<<dim3(std::max(1, nmax - 1), nbig), 128, 0, st>>>(d_bp));
        NRGB_CUDA(cudaGetLastError());
        ++launches_;
        if (!bz.empty()) {
          NRGB_LAUNCH("zero_fill", st,
                      zero_kernel<<<(unsigned)bz.size(), 256, 0, st>>>(reinterpret_cast<const ZeroSeg*>(dev + o_bz)));
          NRGB_CUDA(cudaGetLastError());
          ++launches_;
        }
        gemm(gg);
        NRGB_CUDA(raise_smem_attr((const void*)bt_T_kernel, (int)BT_T_SMEM));
        NRGB_LAUNCH("bt_T", st, bt_T_kernel<<<dim3(kmax, nbig), BT_T_NT, BT_T_SMEM, st>>>(d_bp));
        NRGB_CUDA(cudaGetLastError());
        ++launches_;
        for (int k = kmax - 1; k >= 0; --k) {
          gemm(steps[k].gx);
          gemm(steps[k].gy);
          gemm(steps[k].gz);
        }
      }
    }
  }
  if (!small.empty()) NRGB_CUDA(cudaStreamWaitEvent(st, small_done_, 0));
  // error flags
  int herr[4] = {0, 0, 0, 0};
  GridBarrier hb{};
  NRGB_CUDA(cudaMemcpyAsync(herr, d_err_, sizeof(herr), cudaMemcpyDeviceToHost, st));
  NRGB_CUDA(cudaMemcpyAsync(&hb, d_bar_, sizeof(hb), cudaMemcpyDeviceToHost, st));
  NRGB_CUDA(cudaStreamSynchronize(st));
  hb.error |= herr[3];
  if (herr[0] || herr[1]) throw CudaError("syev: QR iteration did not converge");
  if (herr[2]) throw CudaError("syev: secular equation iteration did not converge");
  if (hb.error) throw CudaError("syev: grid barrier timed out");
}

}  // namespace nrgb
