// Least-squares update of block GMRES on the device: the problem min || E1 S - Hbar Y || of
// the block upper Hessenberg matrix Hbar ((m+1)K x mK) is updated one block column per block
// Arnoldi step by block Householder transformations, as GMRES.c:485-503 updates its
// Hessenberg column with Givens rotations.  Each step applies the earlier blocks' reflectors
// to the new block column (block i acts on rows iK .. iK + 2K), factors the 2K x K panel of
// its last two blocks, and applies the new reflectors to the transformed right-hand side g;
// the residual norm of column c is then the norm of rows (m)K .. (m+1)K of column c of g.
//
// Storage (device, column-major, K <= 256):
//   col   the block column being transformed, at least (j+2)K rows, ld ldc
//   V     per block i: 2K x K reflector vectors at V + 2 i K^2 (ld 2K; v_r[r] = 1 and zeros
//         above r are stored)
//   tau   per block i: K scalars at tau + i K
//   g     the transformed right-hand side, ld ldg >= (m+1)K rows, zero below row K at first
//   stat  3K + 1 doubles per step: the residual norms (K), the squared norms of the new
//         column's projection coefficients (K) and of its subdiagonal block (K), the rank flag
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace fftsvd {
namespace lsq {

// g (ldg rows x K) = the upper triangle of S0 (K x K, ld K) in rows 0 .. K, zero below.
void init(int K, const double* S0, double* g, int64_t ldg, cudaStream_t s);

// Block column j of Hbar into col: rows 0 .. (j+1)K from h (ld ldh), rows (j+1)K .. (j+2)K
// the upper triangle of sub (K x K, ld ldsub).  stat[K + c] and stat[2K + c] receive the
// squared norms of the two parts of column c, stat[3K] the rank flag *flag (0 when flag is
// null).  h, sub and flag are read by this launch only, so the caller may overwrite them
// once it is ordered after it.
void gather(int j, int K, const double* h, int64_t ldh, const double* sub, int64_t ldsub, const int32_t* flag,
            double* col, int64_t ldc, double* stat, cudaStream_t s);

// Step j on the gathered column: the reflectors of blocks 0 .. j-1, the Householder QR of
// rows jK .. (j+2)K (block j's reflectors into V and tau), the new block column of the
// triangular factor (rows 0 .. (j+1)K of col) into Rd + j K ldr when Rd is set, block j's
// reflectors on g and the residual norms into stat[0 .. K).
void step(int j, int K, double* col, int64_t ldc, double* V, double* tau, double* g, int64_t ldg, double* Rd,
          int64_t ldr, double* stat, cudaStream_t s);

}  // namespace lsq
}  // namespace fftsvd
