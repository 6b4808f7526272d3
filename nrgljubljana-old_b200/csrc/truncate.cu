// Truncation of one NRG step on the device (see truncate.cuh).
//
// Ordering: every block's values are ascending, so the position of value v
// (block b, index i) in the sorted list of all values is
//   i + sum_{b' < b} #{w_b' <= v} + sum_{b' > b} #{w_b' < v},
// a stable merge found by binary searches, no sort.
//
// Splitting correction (find_clusters, src/splitting.cc:45-77).  The
// reference scans the sorted list once: a cluster starts at e0 and takes
// every following value with v - e0 < fixeps; a cluster whose values are
// not all equal maps each value different from its first onto the first.
// Values at least fixeps above their predecessor always start a new cluster,
// so the list splits into independent runs, and one thread replays the scan
// over each run (runs are a handful of nearly equal values).  The last
// cluster of the list is not processed, as in the reference.  New mappings
// come out in key order (the list is sorted); equal keys are adjacent and
// map to the same value, so the first of them is kept; keys already mapped
// keep their old value (the reference inserts into a std::map).  The new
// entries are merged into the sorted map; fix_splittings then replaces every
// value found among the keys.
#include "truncate.cuh"

#include <math.h>

#include "common.cuh"

namespace nrgb {

namespace {

constexpr int TR_NT = 256;
constexpr int SCAN_NT = 1024;

__device__ __forceinline__ int ub(const double* a, int n, double v) {  // first a[i] > v
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] <= v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ int lb(const double* a, int n, double v) {  // first a[i] >= v
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

struct Work {
  double* es;    // sorted values
  double* cval;  // candidate replacement value at its key's sorted position
  int* cflag;    // 1: es[k] is a new key
  double* nkey;  // compacted new keys (ascending)
  double* nval;
  int* scal;     // [0] number of new keys
};

Work carve(void* work, int wtot) {
  char* p = static_cast<char*>(work);
  auto take = [&](size_t bytes) {
    char* q = p;
    p += (bytes + 255) & ~size_t(255);
    return q;
  };
  Work w;
  w.es = reinterpret_cast<double*>(take(sizeof(double) * wtot));
  w.cval = reinterpret_cast<double*>(take(sizeof(double) * wtot));
  w.cflag = reinterpret_cast<int*>(take(sizeof(int) * wtot));
  w.nkey = reinterpret_cast<double*>(take(sizeof(double) * wtot));
  w.nval = reinterpret_cast<double*>(take(sizeof(double) * wtot));
  w.scal = reinterpret_cast<int*>(take(sizeof(int) * 8));
  return w;
}

// ground state: the lowest first value of all blocks (find_groundstate)
__global__ void tr_gs_kernel(const TruncBlock* __restrict__ bl, int nb, TruncTail* tail) {
  __shared__ double red[TR_NT];
  double m = INFINITY;
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
    if (bl[b].n > 0) m = fmin(m, bl[b].w[0]);
  red[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmin(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    tail->Egs = red[0];
    tail->flags = 0;
  }
}

__global__ void tr_shift_kernel(double* __restrict__ w, int n, const TruncTail* __restrict__ tail) {
  const double e = tail->Egs;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) w[i] -= e;
}

__global__ void tr_rank_kernel(const TruncBlock* __restrict__ bl, int nb, const double* __restrict__ wall, int wtot,
                               double* __restrict__ es, TruncTail* tail) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= wtot) return;
  int lo = 0, hi = nb - 1;  // block of g: last with off <= g
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (bl[mid].off <= g) lo = mid; else hi = mid - 1;
  }
  const int b = lo, i = g - bl[b].off;
  const double v = wall[g];
  if (i > 0 && wall[g - 1] > v) atomicOr(&tail->flags, 2);
  int r = i;
  for (int c = 0; c < nb; ++c) {
    if (c == b || bl[c].n == 0) continue;
    r += (c < b) ? ub(bl[c].w, bl[c].n, v) : lb(bl[c].w, bl[c].n, v);
  }
  es[r] = v;
}

// one thread per run start: replay the reference's cluster scan over the run
__global__ void tr_cluster_kernel(const double* __restrict__ es, int wtot, double eps, double* __restrict__ cval,
                                  int* __restrict__ cflag) {
  const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (i0 >= wtot) return;
  if (i0 > 0 && !(es[i0] - es[i0 - 1] >= eps)) return;  // not the start of a run
  int i1 = i0 + 1;
  while (i1 < wtot && !(es[i1] - es[i1 - 1] >= eps)) ++i1;
  int c0 = i0;
  double e0 = es[i0];
  for (int i = i0 + 1; i <= i1; ++i) {
    const bool in = (i < i1) && (es[i] - e0 < eps);
    if (in) continue;
    // the cluster [c0, i) closes; the one reaching the end of the list is
    // never processed
    if (i < wtot) {
      bool split = false;
      for (int k = c0 + 1; k < i && !split; ++k) split = es[k] != es[c0];
      if (split)
        for (int k = c0 + 1; k < i; ++k)
          if (es[k] != es[c0] && es[k] != es[k - 1]) {
            cflag[k] = 1;
            cval[k] = es[c0];
          }
    }
    if (i < i1) {
      c0 = i;
      e0 = es[i];
    }
  }
}

// keep the new keys that are not mapped yet, compacted in key order
__global__ void __launch_bounds__(SCAN_NT) tr_compact_kernel(const double* __restrict__ es,
                                                             const double* __restrict__ cval,
                                                             const int* __restrict__ cflag, int wtot,
                                                             const double* __restrict__ mk, const int* __restrict__ mcount,
                                                             double* __restrict__ nkey, double* __restrict__ nval,
                                                             int* __restrict__ scal) {
  __shared__ int part[SCAN_NT];
  const int t = threadIdx.x;
  const int per = (wtot + SCAN_NT - 1) / SCAN_NT;
  const int a = min(wtot, t * per), b = min(wtot, a + per);
  const int mc = *mcount;
  auto keep = [&](int k) {
    if (!cflag[k]) return false;
    const int p = lb(mk, mc, es[k]);
    return !(p < mc && mk[p] == es[k]);
  };
  int cnt = 0;
  for (int k = a; k < b; ++k) cnt += keep(k);
  part[t] = cnt;
  __syncthreads();
  for (int s = 1; s < SCAN_NT; s <<= 1) {  // inclusive scan (Hillis-Steele)
    const int v = t >= s ? part[t - s] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  int pos = part[t] - cnt;
  for (int k = a; k < b; ++k)
    if (keep(k)) {
      nkey[pos] = es[k];
      nval[pos] = cval[k];
      ++pos;
    }
  if (t == SCAN_NT - 1) scal[0] = part[t];
}

// merge the sorted map (mk, mv; *mcount entries) with the new entries into
// (ok, ov); grid covers at least count + new entries
__global__ void tr_merge_kernel(const double* __restrict__ mk, const double* __restrict__ mv, int* mcount,
                                const double* __restrict__ nkey, const double* __restrict__ nval,
                                const int* __restrict__ scal, double* __restrict__ ok, double* __restrict__ ov) {
  const int mc = *mcount, nn = scal[0];
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < mc) {
    const int p = g + lb(nkey, nn, mk[g]);
    ok[p] = mk[g];
    ov[p] = mv[g];
  } else if (g < mc + nn) {
    const int j = g - mc;
    const int p = j + lb(mk, mc, nkey[j]);
    ok[p] = nkey[j];
    ov[p] = nval[j];
  }
}

__global__ void tr_count_kernel(int* mcount, const int* __restrict__ scal) { *mcount += scal[0]; }

// fix_splittings: replace every value found among the keys
__global__ void tr_fix_kernel(double* __restrict__ w, int n, const double* __restrict__ mk,
                              const double* __restrict__ mv, const int* __restrict__ mcount) {
  const int mc = *mcount;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = w[i];
    const int p = lb(mk, mc, v);
    if (p < mc && mk[p] == v) w[i] = mv[p];
  }
}

// highest_retained_energy (src/nrg.cc:1919-1948) and the kept counts
__global__ void tr_retain_kernel(const TruncBlock* __restrict__ bl, int nb, const double* __restrict__ es, int wtot,
                                 TruncRules R, TruncTail* tail, const int* __restrict__ mcount) {
  __shared__ double emax;
  if (threadIdx.x == 0) {
    if (es[0] != 0.0) atomicOr(&tail->flags, 1);
    long long nrkeep;
    if (R.keepenergy <= 0.0) {
      nrkeep = R.keep;
    } else {
      nrkeep = 1 + ub(es, wtot, R.keepenergy);
      nrkeep = min(max(nrkeep, (long long)R.keepmin), (long long)R.keep);
    }
    if (R.safeguard > 0.0) {
      int extra = 0;
      while (nrkeep < wtot && es[nrkeep] - es[nrkeep - 1] <= R.safeguard && extra < R.safeguardmax) {
        ++nrkeep;
        ++extra;
      }
    }
    nrkeep = min(max(nrkeep, 1ll), (long long)wtot);
    emax = es[nrkeep - 1];
    tail->Emax = emax;
    tail->map_count = *mcount;
  }
  __syncthreads();
  int* kept = reinterpret_cast<int*>(tail + 1);
  for (int b = threadIdx.x; b < nb; b += blockDim.x) kept[b] = R.keep_all ? bl[b].n : ub(bl[b].w, bl[b].n, emax);
}

// partial sums of the thermodynamics per block: one warp per block
__global__ void tr_sums_kernel(const TruncBlock* __restrict__ bl, int nb, double f, double* __restrict__ sums) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= nb) return;
  const TruncBlock B = bl[warp];
  double z = 0, e = 0, e2 = 0;
  for (int i = lane; i < B.n; i += 32) {
    const double be = f * B.w[i], ex = exp(-be);
    z += ex;
    e += be * ex;
    e2 += be * be * ex;
  }
  for (int o = 16; o > 0; o >>= 1) {
    z += __shfl_xor_sync(0xffffffffu, z, o);
    e += __shfl_xor_sync(0xffffffffu, e, o);
    e2 += __shfl_xor_sync(0xffffffffu, e2, o);
  }
  if (lane == 0) {
    sums[3 * warp] = z;
    sums[3 * warp + 1] = e;
    sums[3 * warp + 2] = e2;
  }
}

int nblk(int n, int t) { return (n + t - 1) / t; }

}  // namespace

size_t trunc_tail_bytes(int nblocks) {
  return sizeof(TruncTail) + (((size_t)nblocks * sizeof(int) + 7) & ~size_t(7)) + 3 * (size_t)nblocks * sizeof(double);
}

const double* trunc_tail_sums(const void* tail, int nblocks) {
  return reinterpret_cast<const double*>(static_cast<const char*>(tail) + sizeof(TruncTail) +
                                         (((size_t)nblocks * sizeof(int) + 7) & ~size_t(7)));
}

size_t trunc_work_bytes(int wtot, int) { return 5 * (((size_t)wtot * 8 + 255) & ~size_t(255)) + 4096; }

cudaError_t truncate_step(const TruncBlock* d_blocks, int nb, double* wall, int wtot, const TruncRules& R,
                          TruncState& S, void* work, void* tail_dev, cudaStream_t st) {
  if (wtot <= 0 || nb <= 0) return cudaErrorInvalidValue;
  Work W = carve(work, wtot);
  TruncTail* tail = static_cast<TruncTail*>(tail_dev);
  double* sums = reinterpret_cast<double*>(static_cast<char*>(tail_dev) + sizeof(TruncTail) +
                                           (((size_t)nb * sizeof(int) + 7) & ~size_t(7)));
  cudaError_t e;
  const int gw = std::min(nblk(wtot, TR_NT), 148 * 8);
  NRGB_LAUNCH("truncate", st, tr_gs_kernel<<<1, TR_NT, 0, st>>>(d_blocks, nb, tail));
  NRGB_LAUNCH("truncate", st, tr_shift_kernel<<<gw, TR_NT, 0, st>>>(wall, wtot, tail));
  // two passes of find_clusters, with fix_splittings after the first (the
  // second finds nothing new when the first changed nothing)
  for (int pass = 0; pass < 2; ++pass) {
    NRGB_LAUNCH("truncate", st, tr_rank_kernel<<<nblk(wtot, TR_NT), TR_NT, 0, st>>>(d_blocks, nb, wall, wtot, W.es, tail));
    if ((e = cudaMemsetAsync(W.cflag, 0, sizeof(int) * wtot, st)) != cudaSuccess) return e;
    NRGB_LAUNCH("truncate", st, tr_cluster_kernel<<<nblk(wtot, TR_NT), TR_NT, 0, st>>>(W.es, wtot, R.fixeps, W.cval, W.cflag));
    const int c = S.cur;
    NRGB_LAUNCH("truncate", st, tr_compact_kernel<<<1, SCAN_NT, 0, st>>>(W.es, W.cval, W.cflag, wtot, S.map_k[c], S.d_count,
                                                                          W.nkey, W.nval, W.scal));
    NRGB_LAUNCH("truncate", st, tr_merge_kernel<<<std::max(1, nblk(S.map_count + (pass + 1) * wtot, TR_NT)), TR_NT, 0, st>>>(
                                    S.map_k[c], S.map_v[c], S.d_count, W.nkey, W.nval, W.scal, S.map_k[1 - c],
                                    S.map_v[1 - c]));
    NRGB_LAUNCH("truncate", st, tr_count_kernel<<<1, 1, 0, st>>>(S.d_count, W.scal));
    S.cur = 1 - c;
    if (pass == 0)
      NRGB_LAUNCH("truncate", st, tr_fix_kernel<<<gw, TR_NT, 0, st>>>(wall, wtot, S.map_k[S.cur], S.map_v[S.cur], S.d_count));
  }
  NRGB_LAUNCH("truncate", st, tr_retain_kernel<<<1, TR_NT, 0, st>>>(d_blocks, nb, W.es, wtot, R, tail, S.d_count));
  NRGB_LAUNCH("truncate", st, tr_sums_kernel<<<nblk(nb * 32, TR_NT), TR_NT, 0, st>>>(d_blocks, nb, R.betabar, sums));
  return cudaGetLastError();
}

}  // namespace nrgb
