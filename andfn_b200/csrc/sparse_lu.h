// Sparse LU of the discharge system (host side).
//
// Replaces scipy.sparse.linalg.splu (SuperLU) as called at
// andfn/hpc/hpc_solve.py:121 (factor once per solve) and :651 (solve every
// iteration).  The factorisation here is
//     P A Q = L U     (L unit lower, U upper, P from partial pivoting,
//                      Q a fill-reducing column order)
// and the device solves x = Q U^-1 L^-1 P b every iteration with a
// dependency-driven kernel (see solver.cu).
#pragma once
#include <atomic>
#include <cmath>
#include <cstdint>
#include <memory>
#include <vector>

namespace andfn {

struct CscMatrix {
  int n = 0;
  std::vector<int> colptr, rowind;
  std::vector<double> val;
};

// State of a factorisation whose dense block is factorised elsewhere
// (sparse_lu_factor(..., defer_dense = true) then sparse_lu_finish).
struct LuPending {
  std::vector<int> Lcp, Lri, Ucp, Uri, prow, tail_rows;
  std::vector<double> Lv, Uv, diag;
  double min_piv = 0.0;
};

struct LuFactors {
  int n = 0;
  // Dense trailing block: the last `dense` pivot steps are factorised as a
  // dense matrix (column-major dense x dense, strictly lower part of L and
  // strictly upper part of U; the CSR arrays below then hold only entries
  // outside that block).
  int dense = 0;
  std::vector<double> l22, u22;
  std::vector<int> q;       // column order: pivot step k eliminates column q[k]
  std::vector<int> pinv;    // row -> pivot step (P as inverse permutation)
  // Row-oriented (CSR) factors in pivot-step indices, for the device solve:
  std::vector<int> l_ptr, l_col;  // strictly lower part of L (unit diagonal)
  std::vector<double> l_val;
  std::vector<int> u_ptr, u_col;  // strictly upper part of U
  std::vector<double> u_val;
  std::vector<double> u_inv_diag; // 1 / U(k,k)
  int64_t nnz() const { return (int64_t)l_val.size() + (int64_t)u_val.size() + n; }
  double min_abs_pivot = 0.0;
  // deferred dense block: the Schur complement (column-major dense x dense,
  // row order = block order) and the state sparse_lu_finish needs
  double *schur = nullptr;            // dense x dense, in schur_own or a caller's buffer
  std::unique_ptr<double[]> schur_own;
  const double *schur_data() const { return schur; }
  LuPending pending;
};

// Column ordering: minimum degree on the column-intersection graph of A,
// computed on a quotient graph whose initial elements are the rows of A
// (each row is a clique of its columns), with approximate external degrees.
// *dense_tail (optional) receives the number of trailing columns that remain
// once the minimum degree reaches dense_frac of the remaining columns (the
// graph is then nearly complete; 0 if that never happens with >= 64 left).
//
// With prog, the order is also published while it is computed, for a
// factorisation that runs beside it (see OrderProgress).
struct OrderProgress;
std::vector<int> column_min_degree_order(const CscMatrix &A, int *dense_tail = nullptr, double dense_frac = 0.15,
                                         int max_dense = 3072, OrderProgress *prog = nullptr);

// A column order published while it is computed: order[0 .. count) are
// final; lead >= 0 once the number of leading (sparse) columns is known,
// and then no entry below lead changes; done once all n entries are there.
// Stores are release, loads acquire.
struct OrderProgress {
  std::vector<int> order;  // n entries
  std::atomic<int> count{0};
  std::atomic<int> lead{-1};
  std::atomic<int> done{0};
  void reset(int n) {
    order.assign(n, -1);
    count.store(0);
    lead.store(-1);
    done.store(0);
  }
};

// The left-looking sparse pivot steps of sparse_lu_factor, kept between
// calls so that they can be taken while the column order is still being
// computed (lu_leading_follow) and finished by sparse_lu_factor_rest.
struct LuLeading {
  int n = 0, k = 0;  // pivot steps taken
  std::vector<int> pinv, prow, Lcp, Lri, Ucp, Uri;
  std::vector<double> Lv, Uv, diag, x;
  std::vector<int> touched, visited, pattern, topo, stack, childpos;
  double min_piv = INFINITY;
};
void lu_leading_init(LuLeading &st, int n);
// One pivot step on column col; 0, or 3 if it has no nonzero pivot.
int lu_leading_step(const CscMatrix &A, LuLeading &st, int col);
// Takes the pivot steps of the leading columns as the ordering publishes
// them; returns once the ordering is done and every leading column is
// factorised (0), or 3 on a zero pivot (the ordering is still waited for).
int lu_leading_follow(const CscMatrix &A, const OrderProgress &prog, LuLeading &st);

// LU with partial pivoting: left-looking sparse (Gilbert-Peierls) for the
// first n - dense pivot steps, then the Schur complement of the last `dense`
// columns as a dense matrix, factorised by a blocked right-looking dense LU
// with partial pivoting (OpenMP).  Returns 0 on success, 3 (singular) if a
// column has no nonzero pivot.
int sparse_lu_factor(const CscMatrix &A, const std::vector<int> &q, double pivot_threshold, LuFactors &out,
                     int dense = 0, bool defer_dense = false, double *schur_buf = nullptr);
// sparse_lu_factor after its leading pivot steps (st.k == n - dense) were
// taken by lu_leading_step / lu_leading_follow; the same factors.
int sparse_lu_factor_rest(const CscMatrix &A, const std::vector<int> &q, LuLeading &st, LuFactors &out, int dense,
                          bool defer_dense, double *schur_buf);

// With defer_dense, sparse_lu_factor stops after forming the Schur complement
// (out.schur: schur_buf when given, dense x dense doubles, e.g. page-locked
// memory for the upload, else memory of its own); once it is factorised in
// place elsewhere (partial pivoting,
// dpiv[j] = block row swapped with row j, unit lower L below the diagonal, U
// on and above it), sparse_lu_finish completes the row order and the
// row-oriented factors from the pivots and U's diagonal (l22 / u22 stay
// empty: the factorised block lives where it was factorised).
int sparse_lu_finish(LuFactors &F, const std::vector<int> &dpiv, const std::vector<double> &tail_diag);

// Reference triangular solve on the host (used for checks): x = A^-1 b.
void sparse_lu_solve_host(const LuFactors &F, const double *b, double *x);

}  // namespace andfn
