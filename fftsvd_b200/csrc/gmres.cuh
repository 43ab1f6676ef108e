// Device kernels of the GMRES solve (GMRES.c:446-539) and the block-diagonal
// preconditioner (Preconditioner.c:272-294).  FP64 throughout.
//
// Every kernel also runs a batch of independent columns: column c = blockIdx.z
// (blockIdx.x for givens_kernel) shifts each vector argument by c times its
// column stride (col for vectors and basis columns, pcol for partial sums, hcol
// for Gram-Schmidt coefficients, fcol for scale factors, ycol for combination
// weights).  Strides of zero and a one-column grid give the single solve.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fftsvd {

constexpr int kVecThreads = 256;
constexpr int kRowsPerThread = 4;  // rows per thread in row-wise kernels, kVecThreads apart
constexpr int kRowsPerBlock = kVecThreads * kRowsPerThread;
constexpr int kUpdateGroup = 4;    // basis vectors per load group of the update
constexpr int kDotChunk = 4096;             // rows per block of the multi-dot

// z[idx] = inv * r[idx] for every preconditioner block (blocks of size <= 8).
__global__ void precond_kernel(int nblocks, const int32_t* __restrict__ blk_ptr, const int32_t* __restrict__ blk_idx,
                               const int64_t* __restrict__ inv_off, const double* __restrict__ inv,
                               const double* __restrict__ r, double* __restrict__ z, int64_t col);

// grid (dot_blocks(n), nvec): partial[j * dot_blocks + b] = sum over rows of chunk b of V[j][k] * w[k]
__global__ void dots_partial_kernel(int64_t n, int nvec, const double* __restrict__ V, int64_t ldv,
                                    const double* __restrict__ w, double* __restrict__ partial, int64_t col,
                                    int64_t pcol);
// out[j] = (accumulate ? out[j] : 0) + sum_b partial[j * nblk + b]; one block per j
__global__ void reduce_partial_kernel(int nvec, int nblk, const double* __restrict__ partial, double* __restrict__ out,
                                      int accumulate, int64_t pcol, int64_t hcol);
// grid (vec_blocks(n)): h[j] = sum over b < nblk of partial[j * nblk + b] (the multi-dot's
// chunk partials, column stride dcol; block 0 stores h in h_out), then out = w - V h (out
// may alias w), with nvec doubles of dynamic shared memory; if norm_partial is given,
// norm_partial[b] = sum of squares of out over block b (column stride pcol)
__global__ void update_kernel(int64_t n, int nvec, const double* __restrict__ V, int64_t ldv,
                              const double* __restrict__ partial, int nblk, double* __restrict__ h_out,
                              const double* __restrict__ w, double* __restrict__ out,
                              double* __restrict__ norm_partial, int64_t col, int64_t dcol, int64_t pcol,
                              int64_t hcol);
// partial[b] = sum of squares of w over block b
__global__ void norm_partial_kernel(int64_t n, const double* __restrict__ w, double* __restrict__ partial, int64_t col,
                                    int64_t pcol);

struct GivensState {
   double normr;      // preconditioned rhs norm
   double residual;   // |g[i+1]| / normr after the last step
   double inv_beta;   // 1 / H[i][i+1]
   int32_t flag;      // 0 ok, 1 breakdown (beta == 0), 2 non-finite
   int32_t pad;
};

// Completes Arnoldi step i: H column from the two Gram-Schmidt passes and the
// norm partials, applies the previous rotations, forms the new one, updates g
// (GMRES.c:485-503).  One block per column with givens_smem(i) bytes of dynamic shared
// memory; a column whose active flag is 0 (active may be null: all active) only zeroes
// its inv_beta.  With hist (single column), hist[i] = {residual, flag} as well: the
// residual history the host reads after several steps.
__global__ void givens_kernel(int i, int ldh, double* __restrict__ H, const double* __restrict__ h1,
                              const double* __restrict__ h2, const double* __restrict__ norm_partial, int nblk,
                              double* __restrict__ cs, double* __restrict__ sn, double* __restrict__ g,
                              GivensState* __restrict__ st, int64_t hcol, int64_t pcol,
                              const int32_t* __restrict__ active, double2* __restrict__ hist = nullptr);

// dst = src * (factor_ptr ? *factor_ptr : factor); dst2, if given (single column), receives
// the same values.
__global__ void scale_kernel(int64_t n, const double* __restrict__ src, const double* __restrict__ factor_ptr,
                             double factor, double* __restrict__ dst, int64_t col, int64_t fcol,
                             double* __restrict__ dst2 = nullptr);

// x += V y  (y on device)
__global__ void combine_kernel(int64_t n, int nvec, const double* __restrict__ V, int64_t ldv,
                               const double* __restrict__ y, double* __restrict__ x, int64_t col, int64_t ycol);

// dst = a - b
__global__ void sub_kernel(int64_t n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ dst,
                           int64_t col);
// dst += a
__global__ void add_kernel(int64_t n, const double* __restrict__ a, double* __restrict__ dst, int64_t col);

inline size_t givens_smem(int i) { return sizeof(double) * (3 * (size_t)i + 2); }
inline int vec_blocks(int64_t n) { return (int)((n + kRowsPerBlock - 1) / kRowsPerBlock); }
inline int dot_blocks(int64_t n) { return (int)((n + kDotChunk - 1) / kDotChunk); }

}  // namespace fftsvd
