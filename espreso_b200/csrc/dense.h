// Host dense linear algebra for the subdomain preprocessing (factorisation and
// Schur-complement assembly stay on the host, timed separately from the GPU
// dual iteration).  All matrices are column-major doubles.
#pragma once

#include <cstddef>
#include <vector>

namespace feti {
namespace dense {

// C(m x n) -= A(m x k) * B(n x k)^T
void gemm_nt_sub(int m, int n, int k, const double *A, int lda, const double *B, int ldb, double *C, int ldc);

// Blocked right-looking Cholesky (lower) of the leading `ncols` columns of the
// n x n matrix A; the trailing (n-ncols) block is left holding the Schur
// complement.  Returns 0, or j+1 for a non-positive pivot in column j.
int potrf_lower(double *A, int n, int lda, int ncols);

// B(m x k) := B * L^{-T}, L k x k lower triangular.
void trsm_rlt(int m, int k, const double *L, int ldl, double *B, int ldb);

// In place inverse of a lower-triangular n x n matrix.
void trtri_lower(double *L, int n, int ld);

// C(n x n, full symmetric) := W^T W for lower-triangular W.
void lauum_lower(const double *W, int n, int ldw, double *C, int ldc);

// Packed lower-triangular column-major storage: column j holds rows j..n-1.
inline size_t packed_index(int n, int i, int j) {  // i >= j
    return (size_t)j * n - (size_t)j * (j - 1) / 2 + (size_t)(i - j);
}
void pack_lower(const double *A, int n, int lda, double *P);
// x := L^{-1} x and x := L^{-T} x for packed lower L.
void trsv_packed_lower(const double *P, int n, double *x);
void trsv_packed_lower_t(const double *P, int n, double *x);

// Cyclic Jacobi eigen-decomposition of a small symmetric matrix: eigenvalues
// ascending in w, eigenvectors in the columns of V (n x n).
void jacobi_eigen(const double *A, int n, double *w, double *V);

}  // namespace dense
}  // namespace feti
