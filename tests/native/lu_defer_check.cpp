// Checks the deferred dense block of the host factorisation: the Schur
// complement returned by sparse_lu_factor(..., defer_dense = true) is
// factorised here (partial pivoting, largest magnitude, first row on a tie,
// unblocked) and handed back through sparse_lu_finish; the row-oriented
// factors must match those of the non-deferred factorisation (the host's
// blocked dense LU): structure and permutations exactly, values to rounding.
// Input on stdin: n nnz, then colptr, rowind, val.  Prints "ok" or the first
// mismatch.
#include <cmath>
#include <cstdio>
#include <vector>

#include "sparse_lu.h"

using namespace andfn;

int main() {
  int n, nnz;
  if (scanf("%d %d", &n, &nnz) != 2) return 2;
  CscMatrix A;
  A.n = n;
  A.colptr.resize(n + 1);
  A.rowind.resize(nnz);
  A.val.resize(nnz);
  for (auto &x : A.colptr) scanf("%d", &x);
  for (auto &x : A.rowind) scanf("%d", &x);
  for (auto &x : A.val) scanf("%lf", &x);
  int dense = 0;
  std::vector<int> q = column_min_degree_order(A, &dense, 0.4, 1 << 30);
  if (dense == 0) {
    printf("no dense tail\n");
    return 3;
  }
  LuFactors H, D;
  if (sparse_lu_factor(A, q, 1.0, H, dense) != 0) return 4;
  if (sparse_lu_factor(A, q, 1.0, D, dense, true) != 0 || !D.schur) return 5;
  const int K = D.dense;
  std::vector<double> S(D.schur, D.schur + (size_t)K * K);
  std::vector<int> piv(K);
  std::vector<double> dg(K);
  for (int j = 0; j < K; j++) {
    int p = j;
    double amax = std::fabs(S[(size_t)j * K + j]);
    for (int i = j + 1; i < K; i++)
      if (std::fabs(S[(size_t)j * K + i]) > amax) {
        amax = std::fabs(S[(size_t)j * K + i]);
        p = i;
      }
    piv[j] = p;
    for (int c = 0; c < K; c++) std::swap(S[(size_t)c * K + j], S[(size_t)c * K + p]);
    const double inv = 1.0 / S[(size_t)j * K + j];
    for (int i = j + 1; i < K; i++) S[(size_t)j * K + i] *= inv;
    for (int c = j + 1; c < K; c++) {
      const double u = S[(size_t)c * K + j];
      for (int i = j + 1; i < K; i++) S[(size_t)c * K + i] -= S[(size_t)j * K + i] * u;
    }
    dg[j] = S[(size_t)j * K + j];
  }
  if (sparse_lu_finish(D, piv, dg) != 0) return 6;
  if (H.pinv != D.pinv || H.q != D.q || H.l_ptr != D.l_ptr || H.l_col != D.l_col || H.u_ptr != D.u_ptr ||
      H.u_col != D.u_col) {
    printf("structure differs\n");
    return 1;
  }
  auto close = [](const std::vector<double> &a, const std::vector<double> &b) {
    for (size_t i = 0; i < a.size(); i++)
      if (std::fabs(a[i] - b[i]) > 1e-9 * (1.0 + std::fabs(a[i]))) return false;
    return a.size() == b.size();
  };
  if (!close(H.l_val, D.l_val) || !close(H.u_val, D.u_val) || !close(H.u_inv_diag, D.u_inv_diag)) {
    printf("values differ\n");
    return 1;
  }
  // the dense block: the host keeps L22 / U22; here they are in S
  for (int c = 0; c < K; c++)
    for (int i = 0; i < K; i++) {
      const double h = (i > c) ? H.l22[(size_t)c * K + i] : (i < c ? H.u22[(size_t)c * K + i] : 0.0);
      const double d = (i == c) ? 0.0 : S[(size_t)c * K + i];
      if (std::fabs(h - d) > 1e-9 * (1.0 + std::fabs(h))) {
        printf("dense block differs at %d %d: %g %g\n", i, c, h, d);
        return 1;
      }
    }
  printf("ok K %d\n", K);
  return 0;
}
