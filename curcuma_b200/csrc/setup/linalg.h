// Small dense linear-algebra kernels for the host setup (no external BLAS/LAPACK).
#pragma once
#include <vector>

namespace gfnff {
namespace linalg {

// In-place Cholesky A = L L^T of a row-major n x n SPD matrix (lower triangle written).
// Blocked right-looking algorithm, OpenMP-parallel trailing update.  Returns false if a
// non-positive pivot is met.
bool cholesky(double* A, int n);

// Solves L L^T X = B for nrhs right-hand sides stored row-major as n x nrhs.
void cholesky_solve(const double* L, int n, double* B, int nrhs);

// The same factorisation and solve with cache-blocked, register-tiled kernels (packed
// panels, an 8 x 4 AVX2 micro-kernel): the EEQ of large systems in the CPU oracle, the way
// curcuma's EEQSolver runs it through Eigen's blocked LLT.  Different summation order from
// cholesky/cholesky_solve (agreement to rounding).
bool cholesky_blocked(double* A, int n);
void cholesky_solve_blocked(const double* L, int n, double* B, int nrhs);

// Dense LU with partial pivoting; solves A x = b in place (A destroyed). Returns false
// when singular.
bool lu_solve(double* A, int n, double* b);

// Constrained EEQ solve  [A C^T; C 0][q; lambda] = [x; qf]  with C the 0/1 fragment
// membership matrix (frag[i] in [0, nfrag)).  Follows the Schur-complement Cholesky
// route of curcuma's EEQSolver::solveWithSchurCholesky (eeq_solver.cpp:2087-2256):
// z1 = A^-1 x, Z2 = A^-1 C^T, S = C Z2, S lambda = C z1 - qf, q = z1 - Z2 lambda.
// A (n x n, row-major) is overwritten by its factor.  Falls back to an LU of the
// augmented system when A is not positive definite.  Returns false on failure.
// blocked: the cache-blocked kernels (the oracle's per-geometry EEQ); the set-up keeps the
// simple ones.
bool eeq_schur_solve(double* A, int n, const double* x, const int* frag, int nfrag,
                     const double* qf, double* q, bool blocked = false);

// Symmetric eigen-decomposition (cyclic Jacobi).  A is row-major n x n; on return
// eval is ascending and evec (row-major, column k = eigenvector k).
void sym_eig(const std::vector<double>& A, int n, std::vector<double>& eval,
             std::vector<double>& evec);

}  // namespace linalg
}  // namespace gfnff
