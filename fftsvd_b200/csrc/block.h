// Workspace of the block GMRES solve; see block.cu.
#pragma once

#include <cuda_runtime.h>

#include "common.h"

namespace fftsvd {

constexpr int kBlockMax = 256;  // right-hand sides per block Krylov space

struct BlockWorkspace {
   int64_t n = 0;
   int K = 0;     // columns of a block (a multiple of 8)
   int mmax = 0;  // block steps the basis holds
   DevBuf<double> V;                    // mmax + 1 blocks of K x n
   DevBuf<double> W, R0, T;             // K x n
   DevBuf<double> Bc, Xc, Rc, Tc;       // K x n: right-hand sides, iterate, residual, scratch
   DevBuf<double> Qs;                   // K x n: the block between the two CholQR passes
   DevBuf<double> H, H2;                // (mmax + 1) K x K Gram-Schmidt coefficients
   DevBuf<double> G, R1, R2, R, Rinv;   // K x K
   DevBuf<double> Y, Yo;                // mmax K x K least-squares right-hand side and solution
   DevBuf<double> Dinv;                 // mmax blocks K x K: inverted diagonal blocks of Rd
   DevBuf<double> gwork;                // split-K partial products (dense::gemm_tn)
   DevBuf<double> Rd;                   // (mmax K)^2: dense triangular factor of the least squares
   // least squares (block_ls.h): reflectors, their scalars, the transformed right-hand side
   // ((mmax + 1) K x K), two slots of the block column being transformed and of its statistics
   DevBuf<double> Lv, Ltau, Lg, Lcol[2], Lstat[2];
   DevBuf<double> scal, part, fac;      // column norms and partial sums, column factors
   DevBuf<int32_t> idx, flag;
   cudaStream_t ls_stream = nullptr;        // the least-squares updates, overlapped with the next step
   cudaEvent_t done[2] = {nullptr, nullptr};     // step j's column gathered (slot j & 1)
   cudaEvent_t ls_done[2] = {nullptr, nullptr};  // step j's least-squares update and statistics copied
   double* stat_h[2] = {nullptr, nullptr};  // pinned: statistics of the last two steps (3K + 1)
   int* flag_h = nullptr;                   // pinned: rank flag of the first block
   BlockWorkspace() = default;
   BlockWorkspace(const BlockWorkspace&) = delete;
   BlockWorkspace& operator=(const BlockWorkspace&) = delete;
   ~BlockWorkspace();
   void ensure(int64_t n, int K, int mmax, cudaStream_t stream);
};

}  // namespace fftsvd
