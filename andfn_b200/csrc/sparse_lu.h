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
#include <vector>

namespace andfn {

struct CscMatrix {
  int n = 0;
  std::vector<int> colptr, rowind;
  std::vector<double> val;
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
};

// Column ordering: minimum degree on the column-intersection graph of A,
// computed on a quotient graph whose initial elements are the rows of A
// (each row is a clique of its columns), with approximate external degrees.
// *dense_tail (optional) receives the number of trailing columns that remain
// once the minimum degree reaches dense_frac of the remaining columns (the
// graph is then nearly complete; 0 if that never happens with >= 64 left).
std::vector<int> column_min_degree_order(const CscMatrix &A, int *dense_tail = nullptr, double dense_frac = 0.4,
                                         int max_dense = 3072);

// LU with partial pivoting: left-looking sparse (Gilbert-Peierls) for the
// first n - dense pivot steps, then the Schur complement of the last `dense`
// columns as a dense matrix, factorised by a blocked right-looking dense LU
// with partial pivoting (OpenMP).  Returns 0 on success, 3 (singular) if a
// column has no nonzero pivot.
int sparse_lu_factor(const CscMatrix &A, const std::vector<int> &q, double pivot_threshold, LuFactors &out,
                     int dense = 0);

// Reference triangular solve on the host (used for checks): x = A^-1 b.
void sparse_lu_solve_host(const LuFactors &F, const double *b, double *x);

}  // namespace andfn
