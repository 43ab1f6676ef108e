// Dense FP64 linear algebra of the block GMRES solve (block.cu): the block Gram-Schmidt
// products with the basis, the Gram matrices and triangular factors of CholQR2, and the
// triangular solve of the block least-squares problem.  All matrices are column-major.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fftsvd {
namespace dense {

// Doubles of split-K partial products gemm_tn needs for these sizes.
int64_t gemm_tn_work(int M, int N, int64_t K);

// C (M x N, ld ldc) = alpha A^T B + beta C with A (K x M, ld lda) and B (K x N, ld ldb): the
// long inner dimension K is split into slices whose partial products are summed in a
// fixed order (the result does not depend on timing).  work holds gemm_tn_work(M, N, K)
// doubles.  K, lda and ldb even; A and B 16-byte aligned.
void gemm_tn(int M, int N, int64_t K, double alpha, const double* A, int64_t lda, const double* B, int64_t ldb,
             double beta, double* C, int64_t ldc, double* work, cudaStream_t s);

// C (M x N, ld ldc) = alpha A B + beta C with A (M x K, ld lda) and B (K x N, ld ldb).  C must
// not overlap A or B.  M, K, lda and ldb even; A and B 16-byte aligned.
void gemm_nn(int64_t M, int N, int K, double alpha, const double* A, int64_t lda, const double* B, int64_t ldb,
             double beta, double* C, int64_t ldc, cudaStream_t s);

// X_b = R_b^-1 for `count` upper-triangular n x n matrices R_b = R + b * r_step (ld ldr),
// X_b = X + b * x_step (ld ldx, zeros below the diagonal).  n <= 1024.
void trinv_upper(int n, int count, const double* R, int64_t ldr, int64_t r_step, double* X, int64_t ldx,
                 int64_t x_step, cudaStream_t s);

// Out (rows x N, ld rows) = R^-1 Y for the upper-triangular R (rows x rows, ld ldr) whose
// diagonal blocks of bs rows are inverted first (dinv: rows / bs blocks of bs x bs); Y is
// overwritten by the block back substitution.  rows a multiple of bs, bs even.
void trsm_upper_left(int rows, int N, int bs, const double* R, int64_t ldr, double* Y, double* dinv, double* Out,
                     cudaStream_t s);

// C = A + B elementwise (M x N; C may be A or B).
void add(int M, int N, const double* A, int64_t lda, const double* B, int64_t ldb, double* C, int64_t ldc,
         cudaStream_t s);

}  // namespace dense
}  // namespace fftsvd
