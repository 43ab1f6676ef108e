// Batched solves: many right-hand sides of one surface at once.
//
// Lockstep GMRES: every column keeps its own Krylov basis, Hessenberg matrix,
// Givens rotations and convergence test, exactly as a single solve
// (GMRES.c:446-539), and all columns share each multi-vector matvec
// (DeviceOperator::apply_batch), which reads every operator element and
// translation table once per group of right-hand sides.  The vector kernels are
// the single-solve kernels run over a grid of columns, so a column of a batch
// takes the same arithmetic as the same right-hand side solved alone.
//
// Layout: a block of ncols vectors is column-major (column c at base + c * n);
// basis vector j of all columns is block j of V, so V_j is the input of one
// batched matvec.  ncols is padded to a multiple of kBatchGroup with inactive
// zero columns.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <string>
#include <thread>
#include <vector>

#include "batch.h"
#include "nbody.h"
#include "surface.h"

namespace fftsvd {

void BatchWorkspace::ensure(int n, int cols, int cap) {
   if (cols <= ncols && cap <= capacity) return;
   ncols = std::max(ncols, cols);
   capacity = std::max(capacity, cap);
   const int64_t nb = vec_blocks(n);
   V.alloc((size_t)capacity * ncols * n);
   H.alloc((size_t)ncols * capacity * capacity);
   cs.alloc((size_t)ncols * capacity);
   sn.alloc((size_t)ncols * capacity);
   g.alloc((size_t)ncols * capacity);
   h1.alloc((size_t)ncols * capacity);
   h2.alloc((size_t)ncols * capacity);
   y.alloc((size_t)ncols * capacity);
   partial.alloc((size_t)ncols * capacity * nb);
   normpart.alloc((size_t)ncols * nb);
   scal.alloc((size_t)ncols);
   factor.alloc((size_t)ncols);
   st.alloc((size_t)ncols);
   active.alloc((size_t)ncols);
   for (DevBuf<double>* b : {&w, &r, &b0, &x0, &xout, &t0, &t1, &t2}) b->alloc((size_t)ncols * n);
}

static int pad_cols(int k) { return (k + kBatchGroup - 1) / kBatchGroup * kBatchGroup; }

// Columns per batched matvec launch sequence: the batch buffers of one operator
// precision take at most a quarter of the free device memory.
int Surface::batch_chunk(int precision) {
   int& chunk = precision == FFTSVD_PREC_FP64 ? batch_chunk64 : batch_chunk32;
   if (chunk > 0) return chunk;
   size_t free_b = 0, total_b = 0;
   FFTSVD_CUDA(cudaMemGetInfo(&free_b, &total_b));
   const size_t per = precision == FFTSVD_PREC_FP64 ? op64.batch_bytes_per_rhs() : op32.batch_bytes_per_rhs();
   const size_t cols = std::max<size_t>(1, free_b / 4 / std::max<size_t>(per, 1));
   chunk = (int)std::min<size_t>(256, std::max<size_t>(kBatchGroup, cols / kBatchGroup * kBatchGroup));
   return chunk;
}

void Surface::apply_batch(int precision, const double* X, double* Y, int ncols) {
   FFTSVD_REQUIRE(ncols % kBatchGroup == 0, "batch width");
   const int chunk = batch_chunk(precision);
   for (int c0 = 0; c0 < ncols; c0 += chunk) {
      const int m = std::min(chunk, ncols - c0);
      if (precision == FFTSVD_PREC_FP64)
         op64.apply_batch(X + (int64_t)c0 * n, Y + (int64_t)c0 * n, m, stream);
      else
         op32.apply_batch(X + (int64_t)c0 * n, Y + (int64_t)c0 * n, m, stream);
   }
}

void Surface::precond_batch(const double* r_in, double* z, int ncols) {
   const int threads = 256;
   const int blocks = std::max(1, std::min((precond.nblocks + threads - 1) / threads, 148 * 8));
   precond_kernel<<<dim3(blocks, 1, ncols), threads, 0, stream>>>(precond.nblocks, precond.blk_ptr.get(),
                                                               precond.blk_idx.get(), precond.inv_off.get(),
                                                               precond.inv.get(), r_in, z, n);
   FFTSVD_CHECK_LAUNCH();
}

void Surface::pnorm_batch(const double* v, int ncols, std::vector<double>& out) {
   BatchWorkspace& B = *bw;
   const int nb = vec_blocks(n);
   norm_partial_kernel<<<dim3(nb, 1, ncols), kVecThreads, 0, stream>>>(n, v, B.normpart.get(), n, nb);
   FFTSVD_CHECK_LAUNCH();
   reduce_partial_kernel<<<dim3(1, 1, ncols), 256, 0, stream>>>(1, nb, B.normpart.get(), B.scal.get(), 0, nb, 1);
   FFTSVD_CHECK_LAUNCH();
   out.resize(ncols);
   FFTSVD_CUDA(cudaMemcpyAsync(out.data(), B.scal.get(), sizeof(double) * ncols, cudaMemcpyDeviceToHost, stream));
   FFTSVD_CUDA(cudaStreamSynchronize(stream));
   for (double& v2 : out) v2 = std::sqrt(v2);
}

int Surface::gmres_batch(int precision, int ncols, const double* rhs, double* x, const std::vector<double>& tol,
                         int maxit, const std::vector<char>& run, bool absolute_zero_check, std::vector<double>& res,
                         std::vector<int>& iters, std::vector<int>& status) {
   BatchWorkspace& B = *bw;
   FFTSVD_REQUIRE(ncols <= B.ncols && ncols % kBatchGroup == 0, "batch workspace too small");
   maxit = std::min(maxit, B.capacity - 1);
   const int cap = B.capacity;
   const int nb = vec_blocks(n), nd = dot_blocks(n);
   const int ew_blocks = std::max(1, std::min((n + 255) / 256, 148 * 8));
   const int64_t ldv = (int64_t)ncols * n;
   res.assign(ncols, 0.0);
   iters.assign(ncols, 0);
   status.assign(ncols, FFTSVD_OK);
   FFTSVD_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * ncols * n, stream));
   // r = P^-1 rhs (GMRES.c:457-465), per column
   precond_batch(rhs, B.r.get(), ncols);
   std::vector<double> normr;
   pnorm_batch(B.r.get(), ncols, normr);
   std::vector<int32_t> act(ncols, 0);
   std::vector<double> inv(ncols, 0.0), g0((size_t)ncols * cap, 0.0);
   std::vector<GivensState> sth(ncols);
   int running = 0;
   for (int c = 0; c < ncols; c++) {
      sth[c] = GivensState{normr[c], 1.0, 0.0, 0, 0};
      if (!run[c]) continue;
      if (!std::isfinite(normr[c])) {
         status[c] = FFTSVD_ERR_NONFINITE;
         res[c] = normr[c];
         continue;
      }
      if (absolute_zero_check && normr[c] < tol[c]) continue;  // zero solution (GMRES.c:461-465)
      if (normr[c] == 0.0) continue;
      act[c] = 1;
      inv[c] = 1.0 / normr[c];
      g0[(size_t)c * cap] = normr[c];
      res[c] = 1.0;
      running++;
   }
   std::vector<int> k_of(ncols, 0);
   if (running > 0) {
      double* Vp = B.V.get();
      FFTSVD_CUDA(cudaMemcpyAsync(B.factor.get(), inv.data(), sizeof(double) * ncols, cudaMemcpyHostToDevice, stream));
      scale_kernel<<<dim3(ew_blocks, 1, ncols), 256, 0, stream>>>(n, B.r.get(), B.factor.get(), 0.0, Vp, n, 1);
      FFTSVD_CHECK_LAUNCH();
      FFTSVD_CUDA(cudaMemcpyAsync(B.g.get(), g0.data(), sizeof(double) * g0.size(), cudaMemcpyHostToDevice, stream));
      FFTSVD_CUDA(cudaMemcpyAsync(B.st.get(), sth.data(), sizeof(GivensState) * ncols, cudaMemcpyHostToDevice, stream));
      FFTSVD_CUDA(cudaMemcpyAsync(B.active.get(), act.data(), sizeof(int32_t) * ncols, cudaMemcpyHostToDevice, stream));
      const int64_t pcol = (int64_t)cap * nb;
      const int64_t fcol = sizeof(GivensState) / sizeof(double);
      int i = 0;
      for (i = 0; i < maxit && running > 0; i++) {
         const int nvec = i + 1;
         const double* vi = Vp + (int64_t)i * ldv;
         double* vnext = Vp + (int64_t)(i + 1) * ldv;
         apply_batch(precision, vi, B.w.get(), ncols);
         precond_batch(B.w.get(), B.w.get(), ncols);
         // CGS2 per column (see Surface::gmres)
         const size_t sh = sizeof(double) * nvec;
         dots_partial_kernel<<<dim3(nd, nvec, ncols), kVecThreads, 0, stream>>>(n, nvec, Vp, ldv, B.w.get(),
                                                                                 B.partial.get(), n, pcol);
         FFTSVD_CHECK_LAUNCH();
         update_kernel<<<dim3(nb, 1, ncols), kVecThreads, sh, stream>>>(n, nvec, Vp, ldv, B.partial.get(), nd,
                                                                        B.h1.get(), B.w.get(), B.w.get(), nullptr, n,
                                                                        pcol, 0, cap);
         FFTSVD_CHECK_LAUNCH();
         dots_partial_kernel<<<dim3(nd, nvec, ncols), kVecThreads, 0, stream>>>(n, nvec, Vp, ldv, B.w.get(),
                                                                                 B.partial.get(), n, pcol);
         FFTSVD_CHECK_LAUNCH();
         update_kernel<<<dim3(nb, 1, ncols), kVecThreads, sh, stream>>>(n, nvec, Vp, ldv, B.partial.get(), nd,
                                                                        B.h2.get(), B.w.get(), vnext,
                                                                        B.normpart.get(), n, pcol, nb, cap);
         FFTSVD_CHECK_LAUNCH();
         givens_kernel<<<ncols, 256, givens_smem(i), stream>>>(i, cap, B.H.get(), B.h1.get(), B.h2.get(),
                                                               B.normpart.get(), nb, B.cs.get(), B.sn.get(), B.g.get(),
                                                               B.st.get(), cap, nb, B.active.get());
         FFTSVD_CHECK_LAUNCH();
         scale_kernel<<<dim3(ew_blocks, 1, ncols), 256, 0, stream>>>(n, vnext, &B.st.get()->inv_beta, 0.0, vnext, n,
                                                                  fcol);
         FFTSVD_CHECK_LAUNCH();
         FFTSVD_CUDA(cudaMemcpyAsync(sth.data(), B.st.get(), sizeof(GivensState) * ncols, cudaMemcpyDeviceToHost,
                                     stream));
         FFTSVD_CUDA(cudaStreamSynchronize(stream));
         bool changed = false;
         for (int c = 0; c < ncols; c++) {
            if (!act[c]) continue;
            res[c] = sth[c].residual;
            bool stop = false;
            if (sth[c].flag == 2) {
               status[c] = FFTSVD_ERR_NONFINITE;
               stop = true;
            } else if (sth[c].residual < tol[c] || sth[c].flag == 1) {
               stop = true;
            }
            if (stop) {
               k_of[c] = i + 1;
               act[c] = 0;
               running--;
               changed = true;
            }
         }
         if (changed && running > 0)
            FFTSVD_CUDA(cudaMemcpyAsync(B.active.get(), act.data(), sizeof(int32_t) * ncols, cudaMemcpyHostToDevice,
                                        stream));
      }
      for (int c = 0; c < ncols; c++)
         if (act[c]) {  // iteration cap reached (GMRES.c:505-510)
            k_of[c] = maxit;
            status[c] = FFTSVD_ERR_NOT_CONVERGED;
         }
      // back substitution per column on the host (GMRES.c:512-521)
      int kmax = 0;
      for (int c = 0; c < ncols; c++) kmax = std::max(kmax, k_of[c]);
      if (kmax > 0) {
         std::vector<double> Hh((size_t)ncols * cap * cap), gh((size_t)ncols * cap), yh((size_t)ncols * kmax, 0.0);
         FFTSVD_CUDA(cudaMemcpyAsync(Hh.data(), B.H.get(), sizeof(double) * Hh.size(), cudaMemcpyDeviceToHost, stream));
         FFTSVD_CUDA(cudaMemcpyAsync(gh.data(), B.g.get(), sizeof(double) * gh.size(), cudaMemcpyDeviceToHost, stream));
         FFTSVD_CUDA(cudaStreamSynchronize(stream));
         for (int c = 0; c < ncols; c++) {
            const int k = k_of[c];
            if (k == 0 || status[c] == FFTSVD_ERR_NONFINITE) continue;
            const double* Hc = Hh.data() + (size_t)c * cap * cap;
            double* yc = yh.data() + (size_t)c * kmax;
            for (int q = 0; q < k; q++) yc[q] = gh[(size_t)c * cap + q];
            for (int q = k - 1; q >= 0; q--) {
               yc[q] /= Hc[(size_t)q * cap + q];
               for (int j = q - 1; j >= 0; j--) yc[j] -= Hc[(size_t)q * cap + j] * yc[q];
            }
         }
         FFTSVD_CUDA(cudaMemcpyAsync(B.y.get(), yh.data(), sizeof(double) * yh.size(), cudaMemcpyHostToDevice, stream));
         combine_kernel<<<dim3(ew_blocks, 1, ncols), 256, sizeof(double) * kmax, stream>>>(n, kmax, Vp, ldv, B.y.get(), x,
                                                                                        n, kmax);
         FFTSVD_CHECK_LAUNCH();
      }
   }
   FFTSVD_CUDA(cudaStreamSynchronize(stream));
   int maxk = 0;
   for (int c = 0; c < ncols; c++) {
      iters[c] = k_of[c];
      maxk = std::max(maxk, k_of[c]);
   }
   return maxk;
}

int Surface::solve_batch(int precision, int k, const double* rhs, double* x, double tol, int maxit,
                         fftsvd_solve_info* info) {
   FFTSVD_REQUIRE(k > 0 && k <= kMaxBatch, "right-hand side count");
   FFTSVD_REQUIRE(tol > 0.0 && maxit > 0, "tolerance and iteration cap must be positive");
   const auto clock_start = std::chrono::steady_clock::now();
   const int ncols = pad_cols(k);
   if (!bw) bw = std::make_unique<BatchWorkspace>();
   // basis capacity: the iteration cap, or what a third of the free memory holds
   size_t free_b = 0, total_b = 0;
   FFTSVD_CUDA(cudaMemGetInfo(&free_b, &total_b));
   const size_t per_vec = sizeof(double) * (size_t)ncols * n;
   const size_t fixed = 8 * per_vec;
   const int cap_mem = (int)std::max<int64_t>(2, (int64_t)((free_b / 3 > fixed ? free_b / 3 - fixed : 0) / per_vec));
   bw->ensure(n, ncols, std::min(maxit + 1, std::max(bw->capacity, cap_mem)));
   BatchWorkspace& B = *bw;
   const size_t bytes = sizeof(double) * (size_t)k * n;
   FFTSVD_CUDA(cudaMemsetAsync(B.b0.get(), 0, sizeof(double) * ncols * n, stream));
   FFTSVD_CUDA(cudaMemcpyAsync(B.b0.get(), rhs, bytes, cudaMemcpyDeviceToDevice, stream));
   std::vector<char> run(ncols, 0);
   for (int c = 0; c < k; c++) run[c] = 1;
   std::vector<double> res(ncols, 0.0);
   std::vector<int> iters(ncols, 0), refinements(ncols, 0), status(ncols, FFTSVD_OK);
   if (precision == FFTSVD_PREC_FP64 || precision == FFTSVD_PREC_FP32) {
      gmres_batch(precision, ncols, B.b0.get(), B.x0.get(), std::vector<double>(ncols, tol), maxit, run, true, res,
                  iters, status);
   } else if (precision == FFTSVD_PREC_MIXED) {
      // FP64 iterative refinement around FP32-operator GMRES, column by column as in
      // the single solve: x += A32^-1 (b - A64 x), inner targets kInnerTarget tol / residual
      const int ew_blocks = std::max(1, std::min((n + 255) / 256, 148 * 8));
      precond_batch(B.b0.get(), B.t0.get(), ncols);
      std::vector<double> bn;
      pnorm_batch(B.t0.get(), ncols, bn);
      FFTSVD_CUDA(cudaMemsetAsync(B.x0.get(), 0, sizeof(double) * ncols * n, stream));
      FFTSVD_CUDA(cudaMemcpyAsync(B.t1.get(), B.b0.get(), sizeof(double) * ncols * n, cudaMemcpyDeviceToDevice, stream));
      for (int c = 0; c < ncols; c++) {
         if (!run[c]) continue;
         if (!std::isfinite(bn[c])) status[c] = FFTSVD_ERR_NONFINITE;
         else res[c] = bn[c] < tol ? 0.0 : 1.0;
      }
      for (int pass = 0; pass < 8; pass++) {
         std::vector<char> act(ncols, 0);
         std::vector<double> itol(ncols, 1.0);
         bool any = false;
         for (int c = 0; c < ncols; c++)
            if (run[c] && status[c] == FFTSVD_OK && res[c] >= tol) {
               act[c] = 1;
               itol[c] = std::min(0.1, std::max(kInnerTarget * tol / res[c], 1e-13));
               refinements[c]++;
               any = true;
            }
         if (!any) break;
         std::vector<double> ires;
         std::vector<int> iit, ist;
         gmres_batch(FFTSVD_PREC_FP32, ncols, B.t1.get(), B.xout.get(), itol, maxit, act, false, ires, iit, ist);
         for (int c = 0; c < ncols; c++)
            if (act[c]) {
               iters[c] += iit[c];
               if (ist[c] == FFTSVD_ERR_NONFINITE) status[c] = FFTSVD_ERR_NONFINITE;
            }
         add_kernel<<<dim3(ew_blocks, 1, ncols), 256, 0, stream>>>(n, B.xout.get(), B.x0.get(), n);
         FFTSVD_CHECK_LAUNCH();
         apply_batch(FFTSVD_PREC_FP64, B.x0.get(), B.t2.get(), ncols);
         sub_kernel<<<dim3(ew_blocks, 1, ncols), 256, 0, stream>>>(n, B.b0.get(), B.t2.get(), B.t1.get(), n);
         FFTSVD_CHECK_LAUNCH();
         precond_batch(B.t1.get(), B.t0.get(), ncols);
         std::vector<double> rn;
         pnorm_batch(B.t0.get(), ncols, rn);
         for (int c = 0; c < ncols; c++)
            if (act[c] && status[c] == FFTSVD_OK) {
               res[c] = rn[c] / bn[c];
               if (!std::isfinite(res[c])) status[c] = FFTSVD_ERR_NONFINITE;
            }
      }
      for (int c = 0; c < k; c++)
         if (status[c] == FFTSVD_OK && res[c] >= tol) status[c] = FFTSVD_ERR_NOT_CONVERGED;
   } else {
      throw Error(FFTSVD_ERR_ARGUMENT, "unknown precision mode");
   }
   FFTSVD_CUDA(cudaMemcpyAsync(x, B.x0.get(), bytes, cudaMemcpyDeviceToDevice, stream));
   FFTSVD_CUDA(cudaStreamSynchronize(stream));
   const auto clock_end = std::chrono::steady_clock::now();
   const double ms = std::chrono::duration<double, std::milli>(clock_end - clock_start).count();
   int first_bad = FFTSVD_OK;
   for (int c = 0; c < k; c++) {
      if (first_bad == FFTSVD_OK && status[c] != FFTSVD_OK) first_bad = status[c];
      if (info) {
         info[c].iterations = iters[c];
         info[c].refinements = refinements[c];
         info[c].status = status[c];
         info[c].residual = res[c];
         info[c].setup_ms = 0.0;
         info[c].solve_ms = ms;
      }
   }
   return first_bad;
}

}  // namespace fftsvd

using namespace fftsvd;

extern "C" {

int fftsvd_b200_solve_batch_device(fftsvd_surface* s, int32_t nrhs, int32_t precision, const double* rhs, double* sol,
                                   double tol, int32_t max_iterations, fftsvd_solve_info* info) {
   if (!s || !rhs || !sol || nrhs <= 0) return FFTSVD_ERR_ARGUMENT;
   int status = FFTSVD_OK;
   const int rc = guarded([&] { status = s->s.solve_batch(precision, nrhs, rhs, sol, tol, max_iterations, info); });
   return rc != FFTSVD_OK ? rc : status;
}

int fftsvd_b200_solve_batch(fftsvd_surface* s, int32_t nrhs, int32_t precision, const double* rhs, double* sol,
                            double tol, int32_t max_iterations, fftsvd_solve_info* info) {
   if (!s || !rhs || !sol || nrhs <= 0) return FFTSVD_ERR_ARGUMENT;
   int status = FFTSVD_OK;
   const int rc = guarded([&] {
      Surface& S = s->s;
      const size_t bytes = sizeof(double) * (size_t)nrhs * S.n;
      DevBuf<double> din((size_t)nrhs * S.n), dout((size_t)nrhs * S.n);
      FFTSVD_CUDA(cudaMemcpyAsync(din.get(), rhs, bytes, cudaMemcpyHostToDevice, S.stream));
      status = S.solve_batch(precision, nrhs, din.get(), dout.get(), tol, max_iterations, info);
      FFTSVD_CUDA(cudaMemcpyAsync(sol, dout.get(), bytes, cudaMemcpyDeviceToHost, S.stream));
      FFTSVD_CUDA(cudaStreamSynchronize(S.stream));
   });
   return rc != FFTSVD_OK ? rc : status;
}

int fftsvd_b200_matvec_batch_device(fftsvd_surface* s, int32_t precision, int32_t nrhs, const double* x, double* y) {
   if (!s || !x || !y || nrhs <= 0) return FFTSVD_ERR_ARGUMENT;
   return guarded([&] {
      Surface& S = s->s;
      const int ncols = pad_cols(nrhs);
      const int prec = precision == FFTSVD_PREC_FP64 ? FFTSVD_PREC_FP64 : FFTSVD_PREC_FP32;
      if (ncols == nrhs) {
         S.apply_batch(prec, x, y, ncols);
      } else {  // padded copy: the batched matvec works on whole groups of right-hand sides
         DevBuf<double> xin((size_t)ncols * S.n), yout((size_t)ncols * S.n);
         FFTSVD_CUDA(cudaMemsetAsync(xin.get(), 0, sizeof(double) * ncols * S.n, S.stream));
         FFTSVD_CUDA(cudaMemcpyAsync(xin.get(), x, sizeof(double) * nrhs * S.n, cudaMemcpyDeviceToDevice, S.stream));
         S.apply_batch(prec, xin.get(), yout.get(), ncols);
         FFTSVD_CUDA(cudaMemcpyAsync(y, yout.get(), sizeof(double) * nrhs * S.n, cudaMemcpyDeviceToDevice, S.stream));
         FFTSVD_CUDA(cudaStreamSynchronize(S.stream));
      }
   });
}

int fftsvd_b200_matvec_batch_tensor_device(fftsvd_surface* s, int32_t nrhs, const double* x, double* y) {
   if (!s || !x || !y || nrhs <= 0 || nrhs % kBatchGroup != 0) return FFTSVD_ERR_ARGUMENT;
   return guarded([&] {
      Surface& S = s->s;
      if (!S.op32.tensor_near_available())
         throw Error(FFTSVD_ERR_UNSUPPORTED, "a leaf has more rows than the tensor-core near field takes (256)");
      S.op32.set_tensor_near(true);
      try {
         S.apply_batch(FFTSVD_PREC_FP32, x, y, nrhs);
      } catch (...) {
         S.op32.set_tensor_near(false);
         throw;
      }
      S.op32.set_tensor_near(false);
      FFTSVD_CUDA(cudaStreamSynchronize(S.stream));
      if (S.op32.tensor_status(true)) throw Error(FFTSVD_ERR_TIMEOUT, "a tensor-core near-field wait gave up");
   });
}

}  // extern "C"

// ---- many surfaces at once
//
// Every surface owns its buffers, streams and events, so solves of different surfaces
// are independent: a pool of host threads runs them concurrently (largest surface
// first), each on its surface's device and streams, and the GPU overlaps their kernels.
extern "C" int fftsvd_b200_solve_many(int32_t count, fftsvd_surface* const* surfaces, const double* const* rhs,
                                      double* const* sol, int32_t precision, double tol, int32_t max_iterations,
                                      fftsvd_solve_info* info) {
   if (count <= 0 || !surfaces || !rhs || !sol) return FFTSVD_ERR_ARGUMENT;
   for (int i = 0; i < count; i++)
      if (!surfaces[i] || !rhs[i] || !sol[i]) return FFTSVD_ERR_ARGUMENT;
   std::vector<int> order(count);
   for (int i = 0; i < count; i++) order[i] = i;
   std::stable_sort(order.begin(), order.end(),
                    [&](int a, int b) { return surfaces[a]->s.n > surfaces[b]->s.n; });
   std::vector<int> status(count, FFTSVD_OK);
   std::vector<std::string> message(count);
   std::atomic<int> next{0};
   // up to two solver threads per host core (they spend most of their time waiting on their
   // streams): 64 blobs on 16 cores solved 1.2 % faster with 32 threads than with 16
   const int workers = std::max(1, std::min<int>(count, std::min(32u, 2 * std::max(1u, std::thread::hardware_concurrency()))));
   auto work = [&]() {
      for (;;) {
         const int k = next.fetch_add(1);
         if (k >= count) return;
         const int i = order[k];
         fftsvd::Surface& S = surfaces[i]->s;
         fftsvd_solve_info one{};
         int st = FFTSVD_OK;
         const int rc = guarded([&] {
            FFTSVD_CUDA(cudaSetDevice(S.device));
            st = S.solve(precision, rhs[i], sol[i], tol, max_iterations, &one);
         });
         status[i] = rc != FFTSVD_OK ? rc : st;
         if (rc != FFTSVD_OK) message[i] = fftsvd_b200_last_error();
         if (info) info[i] = one;
      }
   };
   std::vector<std::thread> pool;
   for (int w = 1; w < workers; w++) pool.emplace_back(work);
   work();
   for (auto& t : pool) t.join();
   for (int i = 0; i < count; i++)
      if (status[i] != FFTSVD_OK) {
         fftsvd::set_last_error(message[i].empty() ? "surface " + std::to_string(i) + " did not solve"
                                                   : "surface " + std::to_string(i) + ": " + message[i]);
         return status[i];
      }
   return FFTSVD_OK;
}
