// Checks the factorisation that follows a column order still being computed:
// column_min_degree_order runs on a second thread and publishes its order
// (OrderProgress), lu_leading_follow takes the leading pivot steps as the
// columns arrive, sparse_lu_factor_rest finishes.  The order, the dense tail
// and every array of the (deferred and non-deferred) factors must equal,
// bit for bit, those of the sequential path (order, then sparse_lu_factor).
// Input on stdin: n nnz, then colptr, rowind, val.  Prints "ok <dense>" or
// the first mismatch.
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "sparse_lu.h"

using namespace andfn;

template <class T>
static bool same(const std::vector<T> &a, const std::vector<T> &b) {
  return a.size() == b.size() && (a.empty() || std::memcmp(a.data(), b.data(), sizeof(T) * a.size()) == 0);
}

static bool same_factors(const LuFactors &a, const LuFactors &b, int K) {
  if (a.n != b.n || a.dense != b.dense || !same(a.q, b.q) || !same(a.pinv, b.pinv)) return false;
  if (!same(a.l_ptr, b.l_ptr) || !same(a.l_col, b.l_col) || !same(a.l_val, b.l_val)) return false;
  if (!same(a.u_ptr, b.u_ptr) || !same(a.u_col, b.u_col) || !same(a.u_val, b.u_val)) return false;
  if (!same(a.u_inv_diag, b.u_inv_diag) || !same(a.l22, b.l22) || !same(a.u22, b.u22)) return false;
  const LuPending &p = a.pending, &r = b.pending;
  if (!same(p.Lcp, r.Lcp) || !same(p.Lri, r.Lri) || !same(p.Lv, r.Lv) || !same(p.Ucp, r.Ucp) ||
      !same(p.Uri, r.Uri) || !same(p.Uv, r.Uv) || !same(p.diag, r.diag) || !same(p.prow, r.prow) ||
      !same(p.tail_rows, r.tail_rows))
    return false;
  if ((a.schur == nullptr) != (b.schur == nullptr)) return false;
  if (a.schur && std::memcmp(a.schur, b.schur, sizeof(double) * (size_t)K * K) != 0) return false;
  return true;
}

int main() {
  int n, nnz;
  if (scanf("%d %d", &n, &nnz) != 2) return 2;
  CscMatrix A;
  A.n = n;
  A.colptr.resize(n + 1);
  A.rowind.resize(nnz);
  A.val.resize(nnz);
  for (auto &x : A.colptr)
    if (scanf("%d", &x) != 1) return 2;
  for (auto &x : A.rowind)
    if (scanf("%d", &x) != 1) return 2;
  for (auto &x : A.val)
    if (scanf("%lf", &x) != 1) return 2;
  const double frac = 0.15;
  int dense = 0;
  const std::vector<int> q = column_min_degree_order(A, &dense, frac);
  for (int defer = 0; defer < 2; defer++) {
    LuFactors S;
    if (sparse_lu_factor(A, q, 1.0, S, dense, defer != 0) != 0) {
      printf("sequential factorisation failed\n");
      return 4;
    }
    for (int rep = 0; rep < 4; rep++) {
      OrderProgress prog;
      prog.reset(n);
      int dense2 = 0;
      std::vector<int> q2;
      std::thread th([&] { q2 = column_min_degree_order(A, &dense2, frac, 3072, &prog); });
      LuLeading st;
      lu_leading_init(st, n);
      const int rc = lu_leading_follow(A, prog, st);
      th.join();
      if (rc != 0 || q2 != q || dense2 != dense || prog.lead.load() != n - dense || prog.count.load() != n ||
          !prog.done.load() || prog.order != q) {
        printf("order or leading steps differ (rc %d, dense %d / %d)\n", rc, dense2, dense);
        return 1;
      }
      LuFactors P;
      if (sparse_lu_factor_rest(A, q2, st, P, dense2, defer != 0, nullptr) != 0) {
        printf("rest failed\n");
        return 5;
      }
      if (!same_factors(S, P, dense)) {
        printf("factors differ (defer %d, repetition %d)\n", defer, rep);
        return 1;
      }
    }
  }
  printf("ok %d\n", dense);
  return 0;
}
