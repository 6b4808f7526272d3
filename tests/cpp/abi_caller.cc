// A compiled C++ caller of libnrgb.so that binds the library the way the
// reference's code would (include/nrgb.h, linked with -lnrgb):
//
//  * seam 1, the eigensolver (src/diag.h:54-89 dsyev_, called per block from
//    nrg_diagonalisations_OpenMP, src/nrg.cc:2484-2507): the blocks of a step
//    arrive as row-major matrices with the upper triangle filled (what
//    nrg_prepare_task_for_diag builds); both triangles are written, one
//    batched call replaces the per-block dsyev_, and column r of the returned
//    eigenvectors becomes row r of matrix0 (src/diag.h:80-84).  A nonzero
//    status takes the reference's my_error exit path (src/diag.h:76-77).
//  * seam 3, the whole run (start_calculation, src/nrg.cc:3429-3469):
//    nrgb_run on a work directory, its status mapped the same way.
//
//   abi_caller <workdir> <outdir>   diagonalise test blocks, then run workdir
//   abi_caller --bad-run <dir>      nrgb_run on a directory without inputs
//
// Exit status: 0 success, 1 an error reported by the library (message on
// stderr, as my_error prints it), 2 no usable CUDA device, 3 a wrong result.
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "nrgb.h"

namespace {

// The reference's Matrix is a row-major ublas matrix; this stand-in keeps
// the same indexing.
struct Matrix {
  int n = 0;
  std::vector<double> a;
  explicit Matrix(int n_) : n(n_), a((size_t)n_ * n_, 0.0) {}
  double& operator()(int r, int c) { return a[(size_t)r * n + c]; }
  double operator()(int r, int c) const { return a[(size_t)r * n + c]; }
};

struct Eigen {
  std::vector<double> value;
  Matrix matrix0;  // row r = eigenvector r
  explicit Eigen(int n) : value(n), matrix0(n) {}
};

[[noreturn]] void my_error(const char* what, const char* msg) {
  fprintf(stderr, "ERROR: %s: %s\n", what, msg);
  exit(1);
}

// A test block: a tridiagonal-plus-rank-one symmetric matrix, upper triangle
// only (the reference fills the upper triangle, src/matrix.cc:86-137).
Matrix test_block(int n, int seed) {
  Matrix h(n);
  unsigned s = 12345u + 977u * (unsigned)seed;
  auto rnd = [&] {
    s = s * 1664525u + 1013904223u;
    return (double)(s >> 8) / (double)(1u << 24) - 0.5;
  };
  std::vector<double> u(n);
  for (int i = 0; i < n; ++i) u[i] = rnd();
  for (int r = 0; r < n; ++r)
    for (int c = r; c < n; ++c) {
      double x = 0.1 * u[r] * u[c];
      if (c == r) x += (double)r / n + rnd();
      if (c == r + 1) x += 0.5 + rnd();
      h(r, c) = x;
    }
  return h;
}

// The batched drop-in for one step's diagonalisations.
std::vector<Eigen> diagonalise_all(nrgb_ctx* ctx, const std::vector<Matrix>& hs) {
  const size_t nb = hs.size();
  std::vector<int> n(nb);
  std::vector<std::vector<double>> a(nb), w(nb);
  std::vector<double*> pa(nb), pw(nb);
  for (size_t i = 0; i < nb; ++i) {
    n[i] = hs[i].n;
    a[i].assign((size_t)n[i] * n[i], 0.0);
    for (int r = 0; r < n[i]; ++r)  // symmetrise: both triangles, column-major
      for (int c = r; c < n[i]; ++c) a[i][r + (size_t)c * n[i]] = a[i][c + (size_t)r * n[i]] = hs[i](r, c);
    w[i].resize(n[i]);
    pa[i] = a[i].data();
    pw[i] = w[i].data();
  }
  if (nrgb_syev_batched(ctx, (int)nb, n.data(), pa.data(), pw.data()) != 0)
    my_error("nrgb_syev_batched", nrgb_last_error(ctx));
  std::vector<Eigen> out;
  for (size_t i = 0; i < nb; ++i) {
    Eigen e(n[i]);
    for (int r = 0; r < n[i]; ++r) {
      e.value[r] = w[i][r];
      for (int j = 0; j < n[i]; ++j) e.matrix0(r, j) = a[i][j + (size_t)r * n[i]];
    }
    out.push_back(std::move(e));
  }
  return out;
}

// checkdiag (src/diag.h:329-349): orthonormal rows of matrix0 and
// H v_r = lambda_r v_r, within n-scaled bounds.
bool check(const Matrix& h, const Eigen& e) {
  const int n = h.n;
  double hmax = 0;
  for (double x : h.a) hmax = fmax(hmax, fabs(x));
  auto H = [&](int r, int c) { return r <= c ? h(r, c) : h(c, r); };
  for (int r = 0; r < n; ++r) {
    if (r && e.value[r] < e.value[r - 1]) return false;
    for (int i = 0; i < n; ++i) {
      double s = 0;
      for (int j = 0; j < n; ++j) s += H(i, j) * e.matrix0(r, j);
      if (fabs(s - e.value[r] * e.matrix0(r, i)) > 1e-12 * n * (1 + hmax)) return false;
    }
    for (int q = r; q < n; ++q) {
      double s = 0;
      for (int j = 0; j < n; ++j) s += e.matrix0(r, j) * e.matrix0(q, j);
      if (fabs(s - (q == r ? 1.0 : 0.0)) > 1e-12 * n) return false;
    }
  }
  return true;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    fprintf(stderr, "usage: %s <workdir> <outdir> | --bad-run <dir>\n", argv[0]);
    return 1;
  }
  printf("%s\n", nrgb_version());
  nrgb_ctx* ctx = nullptr;
  if (nrgb_create(0, &ctx) != 0) {
    fprintf(stderr, "no usable CUDA device\n");
    return 2;
  }
  if (strcmp(argv[1], "--bad-run") == 0) {
    double stats[8];
    if (nrgb_run(ctx, argv[2], argv[2], stats) != 0) my_error("nrgb_run", nrgb_last_error(ctx));
    nrgb_destroy(ctx);
    return 0;
  }
  // seam 1: one step of blocks of uneven sizes (warp, cluster and panel paths)
  std::vector<Matrix> hs;
  const int sizes[] = {1, 7, 32, 45, 160, 300, 700};
  for (int k = 0; k < (int)(sizeof sizes / sizeof sizes[0]); ++k) hs.push_back(test_block(sizes[k], k));
  const std::vector<Eigen> es = diagonalise_all(ctx, hs);
  for (size_t i = 0; i < hs.size(); ++i)
    if (!check(hs[i], es[i])) {
      fprintf(stderr, "block %zu (n = %d): wrong eigen-decomposition\n", i, hs[i].n);
      return 3;
    }
  printf("diagonalised %zu blocks\n", hs.size());
  // seam 3: the whole run
  double stats[8];
  if (nrgb_run(ctx, argv[1], argv[2], stats) != 0) my_error("nrgb_run", nrgb_last_error(ctx));
  printf("run: %.3f s, %.0f kernels\n", stats[0], stats[5]);
  nrgb_destroy(ctx);
  return 0;
}
