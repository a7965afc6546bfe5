// Dense host linear algebra used by the design setup (column-major storage).
// Small, self-contained routines: Householder QR, cyclic Jacobi eigen for
// small symmetric matrices, symmetric tridiagonal QL, and a Lanczos solver
// for the eigenpairs of largest magnitude of a larger symmetric matrix.
#pragma once
#include <vector>

namespace fkpc {

// A = Q R for A (rows x cols, rows >= cols): Q is rows x cols with
// orthonormal columns, R cols x cols upper triangular.
void householder_qr(const double* A, int rows, int cols, std::vector<double>* Q,
                    std::vector<double>* R);

// Eigen-decomposition of a small symmetric matrix (n x n) by cyclic Jacobi
// rotations.  values ascending, vectors column-major (column j <-> values[j]).
void jacobi_eigen(const double* A, int n, std::vector<double>* values,
                  std::vector<double>* vectors);

// Symmetric tridiagonal eigenproblem by implicit QL with Wilkinson shifts.
// d (n) diagonal, e (n) sub-diagonal in e[0..n-2].  On return d holds the
// eigenvalues (unsorted) and z (n x n, initialised to identity by the
// caller or to a basis to rotate) the eigenvectors.  Returns false when an
// eigenvalue fails to converge in 60 sweeps.
bool tridiagonal_ql(int n, double* d, double* e, double* z);

// The k eigenpairs of largest |value| of the symmetric n x n matrix A,
// ordered by descending value (algebraic).  Lanczos with full
// re-orthogonalisation, then one Rayleigh-Ritz refinement within the span of
// the converged Ritz vectors.  Each eigenvector is signed so that its
// largest-magnitude entry is positive.  Returns the Lanczos steps used.
int top_magnitude_eigen(const double* A, int n, int k, std::vector<double>* values,
                        std::vector<double>* vectors);

}  // namespace fkpc
