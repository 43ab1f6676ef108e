// Test driver for the host least-squares update of block GMRES (fftsvd_b200/csrc/block_ls.cpp):
// builds a seeded random block upper-Hessenberg problem, feeds it to BlockLeastSquares one
// block column at a time and writes everything a check needs to a binary file.
//
//   block_ls_driver K M seed out.bin
//
// out.bin (doubles): residuals after each step (M x K), then Hbar ((M+1)K x MK, column-major),
// S0 (K x K, column-major), the triangular factor R (MK x MK, column-major, upper) and g_top
// (MK x K, column-major).
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "../fftsvd_b200/csrc/block_ls.h"

int main(int argc, char** argv) {
   if (argc != 5) {
      std::fprintf(stderr, "usage: %s K M seed out.bin\n", argv[0]);
      return 2;
   }
   const int K = std::atoi(argv[1]), M = std::atoi(argv[2]);
   std::mt19937_64 gen(std::strtoull(argv[3], nullptr, 10));
   std::normal_distribution<double> N(0.0, 1.0);
   std::vector<double> S0((size_t)K * K, 0.0);
   for (int c = 0; c < K; c++)
      for (int r = 0; r <= c; r++) S0[(size_t)c * K + r] = N(gen) + (r == c ? 5.0 : 0.0);
   fftsvd::BlockLeastSquares ls;
   ls.init(K, M, S0.data());
   const int rows = (M + 1) * K, cols = M * K;
   std::vector<double> H((size_t)rows * cols, 0.0), res((size_t)M * K);
   for (int j = 0; j < M; j++) {
      const int ldh = (j + 1) * K;
      std::vector<double> h((size_t)ldh * K), sub((size_t)K * K, 0.0);
      for (double& v : h) v = N(gen);
      for (int c = 0; c < K; c++)
         for (int r = 0; r <= c; r++) sub[(size_t)c * K + r] = N(gen) + (r == c ? 2.0 : 0.0);
      for (int c = 0; c < K; c++) {
         for (int r = 0; r < ldh; r++) H[(size_t)(j * K + c) * rows + r] = h[(size_t)c * ldh + r];
         for (int r = 0; r <= c; r++) H[(size_t)(j * K + c) * rows + ldh + r] = sub[(size_t)c * K + r];
      }
      ls.add_column(h.data(), sub.data(), res.data() + (size_t)j * K);
   }
   std::vector<double> R((size_t)cols * cols, 0.0), gt((size_t)cols * K);
   for (int j = 0; j < M; j++) {
      const int ldr = (j + 1) * K;
      for (int c = 0; c < K; c++)
         for (int r = 0; r < ldr; r++) R[(size_t)(j * K + c) * cols + r] = ls.rcol(j)[(size_t)c * ldr + r];
   }
   for (int c = 0; c < K; c++)
      for (int r = 0; r < cols; r++) gt[(size_t)c * cols + r] = ls.g()[(size_t)c * ls.ldg() + r];
   FILE* f = std::fopen(argv[4], "wb");
   if (!f) return 1;
   std::fwrite(res.data(), sizeof(double), res.size(), f);
   std::fwrite(H.data(), sizeof(double), H.size(), f);
   std::fwrite(S0.data(), sizeof(double), S0.size(), f);
   std::fwrite(R.data(), sizeof(double), R.size(), f);
   std::fwrite(gt.data(), sizeof(double), gt.size(), f);
   std::fclose(f);
   return 0;
}
