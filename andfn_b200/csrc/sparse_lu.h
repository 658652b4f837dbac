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
std::vector<int> column_min_degree_order(const CscMatrix &A, int *dense_tail = nullptr, double dense_frac = 0.15,
                                         int max_dense = 3072);

// LU with partial pivoting: left-looking sparse (Gilbert-Peierls) for the
// first n - dense pivot steps, then the Schur complement of the last `dense`
// columns as a dense matrix, factorised by a blocked right-looking dense LU
// with partial pivoting (OpenMP).  Returns 0 on success, 3 (singular) if a
// column has no nonzero pivot.
int sparse_lu_factor(const CscMatrix &A, const std::vector<int> &q, double pivot_threshold, LuFactors &out,
                     int dense = 0, bool defer_dense = false, double *schur_buf = nullptr);

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
