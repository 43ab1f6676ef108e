// Host least-squares update of block GMRES (the class is described in block_ls.h).
#include "block_ls.h"

#include <cmath>
#include <stdexcept>

namespace fftsvd {

void BlockLeastSquares::init(int K, int mmax, const double* S0) {
   if (K <= 0 || mmax <= 0) throw std::invalid_argument("block least squares: empty problem");
   K_ = K;
   mmax_ = mmax;
   m_ = 0;
   V_.assign(mmax, {});
   tau_.assign(mmax, {});
   Rcol_.assign(mmax, {});
   g_.assign((size_t)(mmax + 1) * K * K, 0.0);
   const int ldg = (mmax + 1) * K;
   for (int c = 0; c < K; c++)
      for (int r = 0; r <= c; r++) g_[(size_t)c * ldg + r] = S0[(size_t)c * K + r];
}

// Reflectors r = 0 .. K-1 of block i (H_r = I - tau_r v_r v_r^T, v_r[r] = 1, zero above r)
// applied in order to rows iK .. iK + 2K of every column of C.
void BlockLeastSquares::apply_block(int i, double* C, int ldc, int ncols) const {
   const int K = K_, L = 2 * K;
   const double* V = V_[i].data();
   const double* tau = tau_[i].data();
   double* base = C + (size_t)i * K;
#pragma omp parallel for schedule(static)
   for (int c = 0; c < ncols; c++) {
      double* x = base + (size_t)c * ldc;
      for (int r = 0; r < K; r++) {
         if (tau[r] == 0.0) continue;
         const double* v = V + (size_t)r * L;
         double s = x[r];
         for (int t = r + 1; t < L; t++) s += v[t] * x[t];
         s *= tau[r];
         x[r] -= s;
         for (int t = r + 1; t < L; t++) x[t] -= s * v[t];
      }
   }
}

void BlockLeastSquares::add_column(const double* h, const double* sub, double* res) {
   if (m_ >= mmax_) throw std::logic_error("block least squares: too many columns");
   const int K = K_, j = m_, L = 2 * K;
   const int ld = (j + 2) * K;  // rows of the new block column
   std::vector<double> col((size_t)ld * K, 0.0);
   const int ldh = (j + 1) * K;
   for (int c = 0; c < K; c++) {
      for (int r = 0; r < ldh; r++) col[(size_t)c * ld + r] = h[(size_t)c * ldh + r];
      for (int r = 0; r <= c; r++) col[(size_t)c * ld + ldh + r] = sub[(size_t)c * K + r];
   }
   // earlier blocks' reflectors
   for (int i = 0; i < j; i++) apply_block(i, col.data(), ld, K);
   // Householder QR of the 2K x K panel (rows jK .. jK + 2K), LAPACK dlarfg convention
   V_[j].assign((size_t)L * K, 0.0);
   tau_[j].assign(K, 0.0);
   double* P = col.data() + (size_t)j * K;
   for (int r = 0; r < K; r++) {
      double* x = P + (size_t)r * ld;
      const double alpha = x[r];
      double sigma = 0.0;
      for (int t = r + 1; t < L; t++) sigma += x[t] * x[t];
      double* v = V_[j].data() + (size_t)r * L;
      v[r] = 1.0;
      if (sigma == 0.0) {
         tau_[j][r] = 0.0;
         continue;
      }
      const double normx = std::sqrt(alpha * alpha + sigma);
      const double beta = alpha <= 0.0 ? normx : -normx;
      const double tau = (beta - alpha) / beta, scale = 1.0 / (alpha - beta);
      for (int t = r + 1; t < L; t++) {
         v[t] = x[t] * scale;
         x[t] = 0.0;
      }
      x[r] = beta;
      tau_[j][r] = tau;
#pragma omp parallel for schedule(static)
      for (int c = r + 1; c < K; c++) {
         double* y = P + (size_t)c * ld;
         double s = y[r];
         for (int t = r + 1; t < L; t++) s += v[t] * y[t];
         s *= tau;
         y[r] -= s;
         for (int t = r + 1; t < L; t++) y[t] -= s * v[t];
      }
   }
   // the new block column of R: rows 0 .. (j+1)K
   Rcol_[j].assign((size_t)ldh * K, 0.0);
   for (int c = 0; c < K; c++)
      for (int r = 0; r < ldh; r++) Rcol_[j][(size_t)c * ldh + r] = col[(size_t)c * ld + r];
   // right-hand side
   apply_block(j, g_.data(), ldg(), K);
   m_++;
   const int lg = ldg();
   for (int c = 0; c < K; c++) {
      double s = 0.0;
      const double* gc = g_.data() + (size_t)c * lg + (size_t)(j + 1) * K;
      for (int r = 0; r < K; r++) s += gc[r] * gc[r];
      res[c] = std::sqrt(s);
   }
}

}  // namespace fftsvd
