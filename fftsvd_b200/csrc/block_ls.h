// Host side of block GMRES: the least-squares problem min || E1 S - Hbar Y || of the
// block upper Hessenberg matrix Hbar ((m+1)K x mK), updated one block column per block
// Arnoldi step by block Householder transformations, as GMRES.c:485-503 updates its
// Hessenberg column with Givens rotations.  Each step applies the earlier blocks'
// reflectors to the new block column (block i acts on rows iK .. iK + 2K), factors the
// 2K x K panel of its last two blocks, and applies the new reflectors to the transformed
// right-hand side g; the residual norm of column c is then the norm of rows (m)K .. (m+1)K
// of column c of g.  All matrices are column-major; work is spread over the columns with
// OpenMP.
#pragma once

#include <vector>

namespace fftsvd {

class BlockLeastSquares {
 public:
   // K columns per block, at most mmax block columns.
   void init(int K, int mmax, const double* S0 /* K x K, upper triangular, column-major */);
   // Block column j (0-based, j = number of columns added so far): h holds Hbar rows
   // 0 .. (j+1)K of the column (ld (j+1)K), sub the K x K upper-triangular block below it.
   // Afterwards res[c] = residual norm of right-hand side c (K entries).
   void add_column(const double* h, const double* sub, double* res);
   int columns() const { return m_; }
   // The triangular factor, block column j: rows 0 .. (j+1)K of its K columns (ld (j+1)K).
   // The solution's coefficients in the first m blocks of the basis are Y = R^-1 g_top,
   // g_top rows 0 .. mK of the transformed right-hand side (ld ldg()); the solve runs on
   // the device.
   const double* rcol(int j) const { return Rcol_[j].data(); }
   const double* g() const { return g_.data(); }
   int ldg() const { return (mmax_ + 1) * K_; }

 private:
   int K_ = 0, mmax_ = 0, m_ = 0;
   std::vector<std::vector<double>> V_;    // per block: 2K x K reflector vectors (v_r[r] = 1 implicit)
   std::vector<std::vector<double>> tau_;  // per block: K scalars
   std::vector<std::vector<double>> Rcol_; // per block column j: rows 0 .. (j+1)K of the transformed Hbar
   std::vector<double> g_;                 // transformed E1 S, ((mmax+1) K) x K
   void apply_block(int i, double* C, int ldc, int ncols) const;  // rows iK .. iK + 2K of C
};

}  // namespace fftsvd
