// Host-side sparse LU for the discharge system (see sparse_lu.h).
//
// The reference factorises its discharge matrix once per solve with SuperLU
// (scipy.sparse.linalg.splu, andfn/hpc/hpc_solve.py:121; COLAMD column order,
// partial pivoting) and re-solves it every iteration (hpc_solve.py:651).  The
// matrix has a structurally zero diagonal (an element's own log term vanishes
// on its own segment, hpc_solve.py:1148 skips it), so pivoting is required.
//
// This file is our own implementation of the same two published algorithms:
//   * a column minimum-degree order on the quotient graph of A^T A, with the
//     rows of A as the initial elements and approximate external degrees
//     (Davis, Gilbert, Larimore & Ng, "A column approximate minimum degree
//     ordering algorithm", ACM TOMS 30(3), 2004; Amestoy, Davis & Duff,
//     "An approximate minimum degree ordering algorithm", SIMAX 17(4), 1996);
//   * left-looking LU with partial pivoting, one sparse triangular solve per
//     column whose pattern is found by depth-first search (Gilbert & Peierls,
//     "Sparse partial pivoting in time proportional to arithmetic
//     operations", SISSC 9(5), 1988).
#include "sparse_lu.h"

#include <algorithm>
#include <cmath>
#include <thread>
#include <utility>

namespace andfn {

// Degree-bucketed priority queue with O(1) insert / remove / decrease.
struct DegreeBuckets {
  std::vector<int> head, next, prev, deg;
  int mindeg = 0;
  explicit DegreeBuckets(int n) : head(n + 1, -1), next(n, -1), prev(n, -1), deg(n, 0) {}
  void insert(int i, int d) {
    deg[i] = d;
    prev[i] = -1;
    next[i] = head[d];
    if (head[d] >= 0) prev[head[d]] = i;
    head[d] = i;
    if (d < mindeg) mindeg = d;
  }
  void remove(int i) {
    const int d = deg[i];
    if (prev[i] >= 0)
      next[prev[i]] = next[i];
    else
      head[d] = next[i];
    if (next[i] >= 0) prev[next[i]] = prev[i];
  }
  int pop_min() {
    while (head[mindeg] < 0) mindeg++;
    int i = head[mindeg];
    // smallest index among the minimum-degree columns (deterministic order)
    for (int j = next[i]; j >= 0; j = next[j])
      if (j < i) i = j;
    remove(i);
    return i;
  }
};

// Variables are supervariables: columns found indistinguishable (the same
// set of adjacent elements, hence the same neighbours) after an elimination
// step are merged into one principal column of weight nv (the sum of their
// weights), which is then updated and eliminated as one.  Degrees, element
// sizes and |Lp| are weighted sums.  When a principal column is eliminated,
// the order receives it and then the columns merged into it.
std::vector<int> column_min_degree_order(const CscMatrix &A, int *dense_tail, double dense_frac, int max_dense,
                                         OrderProgress *prog) {
  const int n = A.n;
  if (dense_tail) *dense_tail = 0;
  if (prog && (int)prog->order.size() != n) prog->reset(n);
  // Ei[j]: the distinct rows of column j (the initial elements of variable j);
  // Le[r]: the columns of row r in increasing order (row r is the initial
  // element r, a clique of its columns); elements n.. are created by pivots.
  std::vector<std::vector<int>> Le(2 * (size_t)n + 1);
  std::vector<std::vector<int>> Ei(n);
  {
    std::vector<int> mk(n, -1), cnt(n, 0);
    for (int j = 0; j < n; j++) {
      auto &E = Ei[j];
      E.reserve(A.colptr[j + 1] - A.colptr[j]);
      for (int p = A.colptr[j]; p < A.colptr[j + 1]; p++) {
        const int r = A.rowind[p];
        if (mk[r] == j) continue;
        mk[r] = j;
        E.push_back(r);
        cnt[r]++;
      }
    }
    for (int r = 0; r < n; r++) Le[r].reserve(cnt[r]);
    for (int j = 0; j < n; j++)
      for (int r : Ei[j]) Le[r].push_back(j);
  }
  // per element: the stamp and value of w (below), its weighted size and
  // whether it is active, side by side (one cache line per visit)
  struct ElemInfo {
    int stamp, w, len, active;
  };
  std::vector<ElemInfo> ei(2 * (size_t)n + 1, ElemInfo{-1, 0, 0, 0});
  for (int r = 0; r < n; r++) {
    ei[r].active = !Le[r].empty();
    ei[r].len = (int)Le[r].size();
  }
  // nv: weight of a principal column (0 once merged or eliminated);
  // svnext / svtail: the chain of columns merged into a principal
  std::vector<int> nv(n, 1), svnext(n, -1), svtail(n);
  for (int j = 0; j < n; j++) svtail[j] = j;
  std::vector<char> alive(n, 1);  // a principal column not yet eliminated
  std::vector<int> mark(n, -1);
  DegreeBuckets queue(n);
  // Exact initial degree |union of row cliques containing j| - 1 (columns in
  // parallel, each thread with its own marks), inserted in column order.
  std::vector<int> deg0(n);
#pragma omp parallel
  {
    std::vector<int> mk(n, -1);
#pragma omp for schedule(static, 64)
    for (int j = 0; j < n; j++) {
      int d = 0;
      for (int e : Ei[j])
        for (int v : Le[e])
          if (v != j && mk[v] != j) {
            mk[v] = j;
            d++;
          }
      deg0[j] = std::min(d, n - 1);
    }
  }
  for (int j = 0; j < n; j++) queue.insert(j, deg0[j]);
  queue.mindeg = 0;

  std::vector<int> order;
  order.reserve(n);
  auto emit = [&](int p) {
    for (int v = p; v >= 0; v = svnext[v]) {
      if (prog) prog->order[order.size()] = v;
      order.push_back(v);
    }
  };
  // the leading columns are published after every pivot step, the tail at once
  auto publish_done = [&](int lead) {
    if (!prog) return;
    prog->lead.store(lead, std::memory_order_release);
    prog->count.store((int)order.size(), std::memory_order_release);
    prog->done.store(1, std::memory_order_release);
  };
  int stamp = 0, estamp = 0, eliminated = 0;
  std::vector<int> emark(2 * (size_t)n + 1, -1);
  std::vector<int> Lp, dnew(n, 0);
  std::vector<unsigned> hsh(n, 0);
  std::vector<int> byhash;
  for (int step = 0; eliminated < n; step++) {
    const int remaining = n - eliminated;
    while (queue.head[queue.mindeg] < 0) queue.mindeg++;
    if (dense_tail && remaining >= 64 && remaining <= max_dense && queue.mindeg >= dense_frac * (remaining - 1)) {
      // The remaining graph is nearly complete: it is factorised as a dense
      // block, where the column order does not change the fill.  Append the
      // remaining principal columns by (degree, index), each followed by the
      // columns merged into it.
      *dense_tail = remaining;
      const int lead = (int)order.size();
      if (prog) prog->lead.store(lead, std::memory_order_release);
      std::vector<std::pair<int, int>> rest;
      for (int j = 0; j < n; j++)
        if (alive[j]) rest.push_back({queue.deg[j], j});
      std::sort(rest.begin(), rest.end());
      for (auto &pr : rest) emit(pr.second);
      publish_done(lead);
      return order;
    }
    const int p = queue.pop_min();
    emit(p);
    if (prog) prog->count.store((int)order.size(), std::memory_order_release);
    eliminated += nv[p];
    alive[p] = 0;
    // New element: union of the active elements adjacent to p, minus p.
    stamp++;
    Lp.clear();
    int lpw = 0;
    for (int e : Ei[p]) {
      if (!ei[e].active) continue;
      for (int v : Le[e])
        if (alive[v] && mark[v] != stamp) {
          mark[v] = stamp;
          Lp.push_back(v);
          lpw += nv[v];
        }
      ei[e].active = 0;  // absorbed into the new element
      std::vector<int>().swap(Le[e]);
    }
    std::vector<int>().swap(Ei[p]);
    const int ne = n + step;
    if (Lp.empty()) continue;
    std::sort(Lp.begin(), Lp.end());
    Le[ne] = Lp;
    ei[ne].active = 1;
    ei[ne].len = lpw;
    // Prune absorbed elements from the neighbours' lists and add the new one;
    // w(e) = weighted |Le \ Lp| for every other element touching Lp (one pass).
    const int wst = step;
    for (int i : Lp) {
      auto &E = Ei[i];
      size_t o = 0;
      for (size_t a = 0; a < E.size(); a++) {
        const int e = E[a];
        ElemInfo &x = ei[e];
        if (!x.active) continue;
        E[o++] = e;
        if (x.stamp != wst) {
          x.stamp = wst;
          x.w = x.len;
        }
        x.w -= nv[i];
      }
      E.resize(o);
      E.push_back(ne);
    }
    // Aggressive absorption of elements contained in Lp, then approximate
    // external degrees and a hash of each list for the supervariable test.
    for (int i : Lp) {
      auto &E = Ei[i];
      size_t o = 0;
      long d = lpw - nv[i];
      unsigned h = 0;
      for (size_t a = 0; a < E.size(); a++) {
        int e = E[a];
        ElemInfo &x = ei[e];
        if (e != ne && x.stamp == wst && x.w == 0) {
          if (x.active) {
            x.active = 0;
            std::vector<int>().swap(Le[e]);
          }
          continue;
        }
        if (!x.active) continue;
        E[o++] = e;
        h += (unsigned)e;
        if (e != ne) d += x.w;
      }
      E.resize(o);
      long bound = (long)queue.deg[i] + lpw - nv[i];
      if (d > bound) d = bound;
      if (d > remaining - nv[p] - nv[i]) d = remaining - nv[p] - nv[i];
      if (d < 0) d = 0;
      dnew[i] = (int)d;
      hsh[i] = h;
      queue.remove(i);
    }
    // Supervariables: columns of Lp with the same element set are merged
    // into the first of them (by index); the principal's external degree
    // no longer counts the merged weight.
    byhash.assign(Lp.begin(), Lp.end());
    std::sort(byhash.begin(), byhash.end(), [&](int a, int b) {
      if (hsh[a] != hsh[b]) return hsh[a] < hsh[b];
      if (Ei[a].size() != Ei[b].size()) return Ei[a].size() < Ei[b].size();
      return a < b;
    });
    for (size_t a = 0; a < byhash.size();) {
      size_t b = a + 1;
      while (b < byhash.size() && hsh[byhash[b]] == hsh[byhash[a]] &&
             Ei[byhash[b]].size() == Ei[byhash[a]].size())
        b++;
      for (size_t u = a; u + 1 < b; u++) {
        const int i = byhash[u];
        if (!nv[i]) continue;
        estamp++;
        for (int e : Ei[i]) emark[e] = estamp;
        for (size_t t = u + 1; t < b; t++) {
          const int j = byhash[t];
          if (!nv[j]) continue;
          bool same = true;
          for (int e : Ei[j])
            if (emark[e] != estamp) {
              same = false;
              break;
            }
          if (!same) continue;
          nv[i] += nv[j];
          dnew[i] = std::max(0, dnew[i] - nv[j]);
          nv[j] = 0;
          alive[j] = 0;
          svnext[svtail[i]] = j;
          svtail[i] = svtail[j];
          std::vector<int>().swap(Ei[j]);
        }
      }
      a = b;
    }
    for (int i : Lp)
      if (nv[i]) queue.insert(i, dnew[i]);
  }
  publish_done((int)order.size());
  return order;
}

// Blocked right-looking LU with partial pivoting of a column-major n x n
// matrix (unit lower L and U overwrite S); piv[j] = row swapped with row j.
static int dense_lu(double *S, int n, std::vector<int> &piv, double &min_piv) {
  const int NB = 48;
  piv.assign(n, 0);
  for (int j0 = 0; j0 < n; j0 += NB) {
    const int jb = std::min(NB, n - j0);
    // panel factorisation, columns j0 .. j0+jb-1
    for (int j = j0; j < j0 + jb; j++) {
      double *cj = S + (size_t)j * n;
      int p = j;
      double amax = std::fabs(cj[j]);
      for (int i = j + 1; i < n; i++)
        if (std::fabs(cj[i]) > amax) {
          amax = std::fabs(cj[i]);
          p = i;
        }
      piv[j] = p;
      if (amax == 0.0 || !std::isfinite(amax)) return 3;
      min_piv = std::min(min_piv, amax);
      if (p != j)
        for (int c = 0; c < n; c++) std::swap(S[(size_t)c * n + j], S[(size_t)c * n + p]);
      const double inv = 1.0 / cj[j];
      for (int i = j + 1; i < n; i++) cj[i] *= inv;
      for (int c = j + 1; c < j0 + jb; c++) {
        double *cc = S + (size_t)c * n;
        const double u = cc[j];
        if (u != 0.0)
          for (int i = j + 1; i < n; i++) cc[i] -= cj[i] * u;
      }
    }
    const int c0 = j0 + jb;
    if (c0 >= n) break;
    // U12 = L11^-1 A12 and trailing update A22 -= L21 U12, by columns
#pragma omp parallel for schedule(dynamic, 8)
    for (int c = c0; c < n; c++) {
      double *cc = S + (size_t)c * n;
      for (int j = j0; j < c0; j++) {
        const double u = cc[j];
        if (u == 0.0) continue;
        const double *cj = S + (size_t)j * n;
        for (int i = j + 1; i < c0; i++) cc[i] -= cj[i] * u;
      }
      for (int j = j0; j < c0; j++) {
        const double u = cc[j];
        if (u == 0.0) continue;
        const double *cj = S + (size_t)j * n;
        for (int i = c0; i < n; i++) cc[i] -= cj[i] * u;
      }
    }
  }
  return 0;
}

static int finish_factors(LuFactors &F, LuPending &W, const std::vector<int> &dpiv, const double *S,
                          const double *tail_diag);

void lu_leading_init(LuLeading &st, int n) {
  st.n = n;
  st.k = 0;
  st.pinv.assign(n, -1);
  st.prow.assign(n, -1);
  st.Lcp.assign(1, 0);
  st.Lri.clear();
  st.Lv.clear();
  st.Ucp.assign(1, 0);
  st.Uri.clear();
  st.Uv.clear();
  st.diag.assign(n, 0.0);
  st.x.assign(n, 0.0);
  st.touched.assign(n, -1);
  st.visited.assign(n, -1);
  st.pattern.clear();
  st.pattern.reserve(n);
  st.topo.clear();
  st.topo.reserve(n);
  st.stack.clear();
  st.childpos.clear();
  st.min_piv = INFINITY;
}

int lu_leading_step(const CscMatrix &A, LuLeading &st, int col) {
  const int k = st.k;
  std::vector<int> &pinv = st.pinv, &prow = st.prow, &Lcp = st.Lcp, &Lri = st.Lri, &Ucp = st.Ucp, &Uri = st.Uri;
  std::vector<double> &Lv = st.Lv, &Uv = st.Uv, &diag = st.diag, &x = st.x;
  std::vector<int> &touched = st.touched, &visited = st.visited, &pattern = st.pattern, &topo = st.topo,
                   &stack = st.stack, &childpos = st.childpos;
  double &min_piv = st.min_piv;
  pattern.clear();
  topo.clear();
  // Scatter A(:, col) and find the reach of its pivoted rows in L's graph.
  for (int p = A.colptr[col]; p < A.colptr[col + 1]; p++) {
    int r = A.rowind[p];
    if (touched[r] != k) {
      touched[r] = k;
      pattern.push_back(r);
      x[r] = 0.0;
    }
    x[r] += A.val[p];
    int j = pinv[r];
    if (j >= 0 && visited[j] != k) {
      // iterative DFS from pivot step j over L's column structure
      stack.clear();
      childpos.clear();
      stack.push_back(j);
      childpos.push_back(Lcp[j]);
      visited[j] = k;
      while (!stack.empty()) {
        int jj = stack.back();
        int &cp = childpos.back();
        bool pushed = false;
        while (cp < Lcp[jj + 1]) {
          int rr = Lri[cp++];
          int j2 = pinv[rr];
          if (j2 >= 0 && visited[j2] != k) {
            visited[j2] = k;
            stack.push_back(j2);
            childpos.push_back(Lcp[j2]);
            pushed = true;
            break;
          }
        }
        if (!pushed) {
          topo.push_back(jj);
          stack.pop_back();
          childpos.pop_back();
        }
      }
    }
  }
  // Numeric: apply the reached columns of L in topological order.
  for (int t = (int)topo.size() - 1; t >= 0; t--) {
    int j = topo[t];
    const int rj = prow[j];
    double xj = (touched[rj] == k) ? x[rj] : 0.0;
    if (xj == 0.0) continue;
    for (int p = Lcp[j]; p < Lcp[j + 1]; p++) {
      int r = Lri[p];
      if (touched[r] != k) {
        touched[r] = k;
        pattern.push_back(r);
        x[r] = 0.0;
      }
      x[r] -= Lv[p] * xj;
    }
  }
  // U(:, k): the pivoted rows, in topological order (dependency order).
  for (int t = (int)topo.size() - 1; t >= 0; t--) {
    int j = topo[t];
    const int rj = prow[j];
    double v = (touched[rj] == k) ? x[rj] : 0.0;
    if (v != 0.0) {
      Uri.push_back(j);
      Uv.push_back(v);
    }
  }
  Ucp.push_back((int)Uri.size());
  // Partial pivoting over the not-yet-pivoted rows.
  int piv = -1;
  double amax = 0.0;
  for (int r : pattern)
    if (pinv[r] < 0) {
      double a = std::fabs(x[r]);
      if (a > amax || (a == amax && piv >= 0 && r < piv && a > 0)) {
        amax = a;
        piv = r;
      }
    }
  if (piv < 0 || amax == 0.0 || !std::isfinite(amax)) return 3;
  double pv = x[piv];
  pinv[piv] = k;
  prow[k] = piv;
  diag[k] = pv;
  if (amax < min_piv) min_piv = amax;
  for (int r : pattern)
    if (pinv[r] < 0 && x[r] != 0.0) {
      Lri.push_back(r);
      Lv.push_back(x[r] / pv);
    }
  Lcp.push_back((int)Lri.size());
  st.k = k + 1;
  return 0;
}

int lu_leading_follow(const CscMatrix &A, const OrderProgress &prog, LuLeading &st) {
  for (;;) {
    const int done = prog.done.load(std::memory_order_acquire);
    const int count = prog.count.load(std::memory_order_acquire);
    const int lead = prog.lead.load(std::memory_order_acquire);
    const int lim = (lead >= 0) ? std::min(count, lead) : count;
    if (st.k < lim) {
      while (st.k < lim)
        if (lu_leading_step(A, st, prog.order[st.k])) return 3;
      continue;
    }
    if (done) return 0;
    std::this_thread::yield();
  }
}

int sparse_lu_factor(const CscMatrix &A, const std::vector<int> &q, double pivot_threshold, LuFactors &F,
                     int dense, bool defer_dense, double *schur_buf) {
  (void)pivot_threshold;
  const int n = A.n;
  if (dense < 0 || dense > n) dense = 0;
  LuLeading st;
  lu_leading_init(st, n);
  for (int k = 0; k < n - dense; k++)
    if (lu_leading_step(A, st, q[k])) return 3;
  return sparse_lu_factor_rest(A, q, st, F, dense, defer_dense, schur_buf);
}

int sparse_lu_factor_rest(const CscMatrix &A, const std::vector<int> &q, LuLeading &st, LuFactors &F, int dense,
                          bool defer_dense, double *schur_buf) {
  const int n = A.n;
  if (dense < 0 || dense > n) dense = 0;
  const int m0 = n - dense;
  if (st.n != n || st.k != m0) return 3;
  F.n = n;
  F.q = q;
  F.dense = dense;
  F.pinv = std::move(st.pinv);
  std::vector<int> &prow = st.prow, &Lcp = st.Lcp, &Lri = st.Lri, &Ucp = st.Ucp, &Uri = st.Uri;
  std::vector<double> &Lv = st.Lv, &Uv = st.Uv, &diag = st.diag;
  double min_piv = st.min_piv;
  std::vector<int> tail_row;           // dense-block row of each original row (or -1)
  // Schur complement, column-major dense x dense (columns zeroed by the
  // thread that forms them)
  std::unique_ptr<double[]> S_own;
  double *S = nullptr;
  std::vector<int> tail_rows;          // original rows of the dense block, in block order
  if (dense > 0) {
    // The dense block: the rows not pivoted yet.  Its columns (the Schur
    // complement) depend only on the finished leading columns of L, so they
    // are formed in parallel, each with its own workspace, by the same steps
    // (and the same arithmetic order) as the leading columns.
    tail_row.assign(n, -1);
    for (int r = 0; r < n; r++)
      if (F.pinv[r] < 0) {
        tail_row[r] = (int)tail_rows.size();
        tail_rows.push_back(r);
      }
    if ((int)tail_rows.size() != dense) return 3;
    if (defer_dense && schur_buf) {
      S = schur_buf;
    } else {
      S_own.reset(new double[(size_t)dense * dense]);
      S = S_own.get();
    }
    std::vector<std::vector<int>> u_rows(dense);
    std::vector<std::vector<double>> u_vals(dense);
#pragma omp parallel
    {
      std::vector<double> xw(n, 0.0);
      std::vector<int> tw(n, -1), vw(n, -1), pat, tp, stk, cpos;
      pat.reserve(n);
      tp.reserve(n);
#pragma omp for schedule(dynamic, 4)
      for (int k = m0; k < n; k++) {
        const int col = q[k];
        pat.clear();
        tp.clear();
        for (int p = A.colptr[col]; p < A.colptr[col + 1]; p++) {
          int r = A.rowind[p];
          if (tw[r] != k) {
            tw[r] = k;
            pat.push_back(r);
            xw[r] = 0.0;
          }
          xw[r] += A.val[p];
          int j = F.pinv[r];
          if (j >= 0 && vw[j] != k) {
            stk.clear();
            cpos.clear();
            stk.push_back(j);
            cpos.push_back(Lcp[j]);
            vw[j] = k;
            while (!stk.empty()) {
              int jj = stk.back();
              int &cp = cpos.back();
              bool pushed = false;
              while (cp < Lcp[jj + 1]) {
                int rr = Lri[cp++];
                int j2 = F.pinv[rr];
                if (j2 >= 0 && vw[j2] != k) {
                  vw[j2] = k;
                  stk.push_back(j2);
                  cpos.push_back(Lcp[j2]);
                  pushed = true;
                  break;
                }
              }
              if (!pushed) {
                tp.push_back(jj);
                stk.pop_back();
                cpos.pop_back();
              }
            }
          }
        }
        for (int t = (int)tp.size() - 1; t >= 0; t--) {
          int j = tp[t];
          const int rj = prow[j];
          double xj = (tw[rj] == k) ? xw[rj] : 0.0;
          if (xj == 0.0) continue;
          for (int p = Lcp[j]; p < Lcp[j + 1]; p++) {
            int r = Lri[p];
            if (tw[r] != k) {
              tw[r] = k;
              pat.push_back(r);
              xw[r] = 0.0;
            }
            xw[r] -= Lv[p] * xj;
          }
        }
        std::vector<int> &ur = u_rows[k - m0];
        std::vector<double> &uv = u_vals[k - m0];
        for (int t = (int)tp.size() - 1; t >= 0; t--) {
          int j = tp[t];
          const int rj = prow[j];
          double v = (tw[rj] == k) ? xw[rj] : 0.0;
          if (v != 0.0) {
            ur.push_back(j);
            uv.push_back(v);
          }
        }
        double *sc = S + (size_t)(k - m0) * dense;
        std::fill(sc, sc + dense, 0.0);
        for (int r : pat)
          if (F.pinv[r] < 0) sc[tail_row[r]] = xw[r];
      }
    }
    for (int k = m0; k < n; k++) {
      Uri.insert(Uri.end(), u_rows[k - m0].begin(), u_rows[k - m0].end());
      Uv.insert(Uv.end(), u_vals[k - m0].begin(), u_vals[k - m0].end());
      Ucp.push_back((int)Uri.size());
      Lcp.push_back((int)Lri.size());
    }
  }
  LuPending W;
  W.Lcp = std::move(Lcp);
  W.Lri = std::move(Lri);
  W.Lv = std::move(Lv);
  W.Ucp = std::move(Ucp);
  W.Uri = std::move(Uri);
  W.Uv = std::move(Uv);
  W.diag = std::move(diag);
  W.prow = std::move(prow);
  W.tail_rows = std::move(tail_rows);
  W.min_piv = min_piv;
  if (dense > 0 && defer_dense) {
    F.schur = S;
    F.schur_own = std::move(S_own);
    F.pending = std::move(W);
    return 0;
  }
  std::vector<int> dpiv;
  if (dense > 0 && dense_lu(S, dense, dpiv, W.min_piv)) return 3;
  return finish_factors(F, W, dpiv, dense > 0 ? S : nullptr, nullptr);
}

int sparse_lu_finish(LuFactors &F, const std::vector<int> &dpiv, const std::vector<double> &tail_diag) {
  if ((int)dpiv.size() != F.dense || (int)tail_diag.size() != F.dense) return 3;
  for (double d : tail_diag) {
    if (!(d != 0.0) || !std::isfinite(d)) return 3;
    F.pending.min_piv = std::min(F.pending.min_piv, std::fabs(d));
  }
  const int rc = finish_factors(F, F.pending, dpiv, nullptr, tail_diag.data());
  F.pending = LuPending();
  F.schur = nullptr;
  F.schur_own.reset();
  return rc;
}

// The row permutation of the dense block from its pivots, the dense block's
// triangles (when factorised here) and the row-oriented factors.
static int finish_factors(LuFactors &F, LuPending &W, const std::vector<int> &dpiv, const double *S,
                          const double *tail_diag) {
  const int n = F.n, dense = F.dense, m0 = n - dense;
  std::vector<int> &Lcp = W.Lcp, &Lri = W.Lri, &Ucp = W.Ucp, &Uri = W.Uri, &prow = W.prow;
  std::vector<double> &Lv = W.Lv, &Uv = W.Uv, &diag = W.diag;
  if (dense > 0) {
    // block row order after the dense pivoting
    std::vector<int> order(dense);
    for (int i = 0; i < dense; i++) order[i] = i;
    for (int j = 0; j < dense; j++) std::swap(order[j], order[dpiv[j]]);
    for (int i = 0; i < dense; i++) {
      const int r = W.tail_rows[order[i]];
      F.pinv[r] = m0 + i;
      prow[m0 + i] = r;
    }
    if (S) {
      F.l22.assign((size_t)dense * dense, 0.0);
      F.u22.assign((size_t)dense * dense, 0.0);
      for (int c = 0; c < dense; c++)
        for (int i = 0; i < dense; i++) {
          const double v = S[(size_t)c * dense + i];
          if (i > c)
            F.l22[(size_t)c * dense + i] = v;
          else if (i < c)
            F.u22[(size_t)c * dense + i] = v;
          else
            diag[m0 + i] = v;
        }
    } else {
      for (int i = 0; i < dense; i++) diag[m0 + i] = tail_diag[i];
    }
  }
  F.min_abs_pivot = W.min_piv;
  // Row-oriented factors in pivot-step indices (entries inside the dense
  // block are kept only in the dense block).
  F.l_ptr.assign(n + 1, 0);
  for (int k = 0; k < m0; k++)
    for (int p = Lcp[k]; p < Lcp[k + 1]; p++) F.l_ptr[F.pinv[Lri[p]] + 1]++;
  for (int i = 0; i < n; i++) F.l_ptr[i + 1] += F.l_ptr[i];
  F.l_col.assign(F.l_ptr[n], 0);
  F.l_val.assign(F.l_ptr[n], 0.0);
  {
    std::vector<int> fill(F.l_ptr.begin(), F.l_ptr.end() - 1);
    for (int k = 0; k < m0; k++)
      for (int p = Lcp[k]; p < Lcp[k + 1]; p++) {
        int i = F.pinv[Lri[p]];
        F.l_col[fill[i]] = k;
        F.l_val[fill[i]++] = Lv[p];
      }
  }
  F.u_ptr.assign(n + 1, 0);
  for (int k = 0; k < n; k++)
    for (int p = Ucp[k]; p < Ucp[k + 1]; p++) F.u_ptr[Uri[p] + 1]++;
  for (int i = 0; i < n; i++) F.u_ptr[i + 1] += F.u_ptr[i];
  F.u_col.assign(F.u_ptr[n], 0);
  F.u_val.assign(F.u_ptr[n], 0.0);
  {
    std::vector<int> fill(F.u_ptr.begin(), F.u_ptr.end() - 1);
    for (int k = 0; k < n; k++)
      for (int p = Ucp[k]; p < Ucp[k + 1]; p++) {
        int i = Uri[p];
        F.u_col[fill[i]] = k;
        F.u_val[fill[i]++] = Uv[p];
      }
  }
  F.u_inv_diag.resize(n);
  for (int k = 0; k < n; k++) F.u_inv_diag[k] = 1.0 / diag[k];
  return 0;
}

void sparse_lu_solve_host(const LuFactors &F, const double *b, double *xout) {
  const int n = F.n, K = F.dense, m0 = n - K;
  std::vector<double> y(n);
  // y = P b
  for (int r = 0; r < n; r++) y[F.pinv[r]] = b[r];
  for (int i = 0; i < n; i++) {
    double s = y[i];
    for (int p = F.l_ptr[i]; p < F.l_ptr[i + 1]; p++) s -= F.l_val[p] * y[F.l_col[p]];
    if (i >= m0)
      for (int c = m0; c < i; c++) s -= F.l22[(size_t)(c - m0) * K + (i - m0)] * y[c];
    y[i] = s;
  }
  for (int i = n - 1; i >= 0; i--) {
    double s = y[i];
    for (int p = F.u_ptr[i]; p < F.u_ptr[i + 1]; p++) s -= F.u_val[p] * y[F.u_col[p]];
    if (i >= m0)
      for (int c = i + 1; c < n; c++) s -= F.u22[(size_t)(c - m0) * K + (i - m0)] * y[c];
    y[i] = s * F.u_inv_diag[i];
  }
  for (int k = 0; k < n; k++) xout[F.q[k]] = y[k];
}

}  // namespace andfn
