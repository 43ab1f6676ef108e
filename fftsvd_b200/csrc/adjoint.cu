// Adjoint (derivatives of the solvation energy).  No counterpart in the reference,
// whose FFTSVDforce computes conductor capacitance forces (FFTSVDforce.c:111-156).
//
// With u = A^-1 B q the surface solution (B: charges -> right-hand side,
// SurfaceOperator.c:291-321) and L the collection (SurfaceOperator.c:364-396),
//   dG = 1/2 k q^T L A^-1 B q,            k = 332.112 / eps_in,
//   d dG / d q_j = 1/2 k (phi_reac_j + (B^T lambda)_j),   lambda = A^-T L^T q,
//   d dG / d x_j = 1/2 k q_j (grad phi_reac(x_j) + sum_i lambda_phi(i) grad_x 1/|x - c_i| at x_j),
// the exact gradient of the discrete energy: the operator A does not depend on the
// charges, and lambda comes from one transposed solve (DeviceOperator::apply_transpose
// with the transposed block preconditioner).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "nbody.h"
#include "surface.h"

namespace fftsvd {

constexpr int kAdjThreads = 128;
constexpr int kAdjChargeTile = 128;
constexpr int kAdjPanelTile = 16;
constexpr int kAdjChunks = 64;
constexpr int kAdjOut = 8;  // per charge: phi_reac, B^T lambda, grad phi_reac (3), grad of the B term (3)

// c = L^T q: per panel, over all charges (in order), c[dphi_row] = sum q_j SLP_i(x_j),
// c[phi_row] = -sum q_j DLP_i(x_j) - 4 pi q_j [x_j == c_i]
__global__ void __launch_bounds__(kAdjThreads) collection_t_kernel(int np, const FlatPanel* __restrict__ panels,
                                                                   const int32_t* __restrict__ phi_row,
                                                                   const int32_t* __restrict__ dphi_row, int nq,
                                                                   const double* __restrict__ qpos,
                                                                   const double* __restrict__ q,
                                                                   double* __restrict__ c) {
   __shared__ double4 tile[kAdjChargeTile];
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   FlatPanel P;
   if (i < np) P = panels[i];
   double cs = 0.0, cd = 0.0;
   for (int base = 0; base < nq; base += kAdjChargeTile) {
      const int cnt = min(kAdjChargeTile, nq - base);
      __syncthreads();
      for (int j = threadIdx.x; j < cnt; j += blockDim.x)
         tile[j] = make_double4(qpos[3 * (base + j)], qpos[3 * (base + j) + 1], qpos[3 * (base + j) + 2], q[base + j]);
      __syncthreads();
      if (i < np)
         for (int j = 0; j < cnt; j++) {
            const double4 t = tile[j];
            if (t.w == 0.0) continue;
            const double pt[3] = {t.x, t.y, t.z};
            double s, d;
            laplace_panel(pt, P, &s, &d);
            cs += t.w * s;
            cd -= t.w * d;
            if (P.centroid[0] == pt[0] && P.centroid[1] == pt[1] && P.centroid[2] == pt[2]) cd -= 4.0 * M_PI * t.w;
         }
   }
   if (i < np) {
      c[dphi_row[i]] = cs;
      c[phi_row[i]] = cd;
   }
}

// Block (charge chunk, panel chunk): each thread owns one charge and sums, over the
// panels of its chunk, the reaction potential and its gradient from the solution u and
// the transposed right-hand-side terms from lambda.
__global__ void __launch_bounds__(kAdjThreads) adjoint_charge_kernel(
    int np, const FlatPanel* __restrict__ panels, const int32_t* __restrict__ phi_row,
    const int32_t* __restrict__ dphi_row, const double* __restrict__ u, const double* __restrict__ lambda, int nq,
    const double* __restrict__ qpos, double* __restrict__ partial) {
   __shared__ FlatPanel tile[kAdjPanelTile];
   __shared__ double4 dens[kAdjPanelTile];  // {u_phi, u_dphi, lambda_phi, -}
   const int j = blockIdx.x * blockDim.x + threadIdx.x;
   const int per = (np + gridDim.y - 1) / gridDim.y;
   const int p0 = blockIdx.y * per, p1 = min(np, p0 + per);
   double pt[3] = {0, 0, 0};
   if (j < nq) { pt[0] = qpos[3 * j]; pt[1] = qpos[3 * j + 1]; pt[2] = qpos[3 * j + 2]; }
   double acc[kAdjOut] = {0, 0, 0, 0, 0, 0, 0, 0};
   for (int base = p0; base < p1; base += kAdjPanelTile) {
      const int cnt = min(kAdjPanelTile, p1 - base);
      __syncthreads();
      {
         const double* src = reinterpret_cast<const double*>(panels + base);
         double* dst = reinterpret_cast<double*>(tile);
         const int words = cnt * (int)(sizeof(FlatPanel) / sizeof(double));
         for (int w = threadIdx.x; w < words; w += blockDim.x) dst[w] = src[w];
         for (int k = threadIdx.x; k < cnt; k += blockDim.x)
            dens[k] = make_double4(u[phi_row[base + k]], u[dphi_row[base + k]], lambda[phi_row[base + k]], 0.0);
      }
      __syncthreads();
      if (j < nq)
         for (int k = 0; k < cnt; k++) {
            const FlatPanel& P = tile[k];
            const double4 dn = dens[k];
            double s, d, gs[3], gd[3];
            const int br = laplace_panel_branch(pt, P);
            if (br != 0) {  // moment expansion: value and exact gradient in one pass
               laplace_panel_far_grad(pt, P, br, &s, &d, gs, gd);
            } else {
               laplace_panel(pt, P, &s, &d);
               laplace_panel_grad(pt, P, gs, gd);
            }
            acc[0] += dn.y * s - dn.x * d;
            if (P.centroid[0] == pt[0] && P.centroid[1] == pt[1] && P.centroid[2] == pt[2]) acc[0] -= 4.0 * M_PI * dn.x;
            const double rx = pt[0] - P.centroid[0], ry = pt[1] - P.centroid[1], rz = pt[2] - P.centroid[2];
            const double r2 = rx * rx + ry * ry + rz * rz, rinv = 1.0 / sqrt(r2), r3 = rinv * rinv * rinv;
            acc[1] += dn.z * rinv;
            acc[2] += dn.y * gs[0] - dn.x * gd[0];
            acc[3] += dn.y * gs[1] - dn.x * gd[1];
            acc[4] += dn.y * gs[2] - dn.x * gd[2];
            acc[5] -= dn.z * rx * r3;
            acc[6] -= dn.z * ry * r3;
            acc[7] -= dn.z * rz * r3;
         }
   }
   if (j < nq)
      for (int o = 0; o < kAdjOut; o++) partial[((size_t)blockIdx.y * nq + j) * kAdjOut + o] = acc[o];
}

__global__ void adjoint_reduce_kernel(int nq, int chunks, const double* __restrict__ partial, double* __restrict__ out) {
   const int j = blockIdx.x * blockDim.x + threadIdx.x;
   if (j >= nq) return;
   for (int o = 0; o < kAdjOut; o++) {
      double s = 0.0;
      for (int c = 0; c < chunks; c++) s += partial[((size_t)c * nq + j) * kAdjOut + o];
      out[(size_t)j * kAdjOut + o] = s;
   }
}

int Surface::adjoint(int precision, double tol, int maxit, double* energy, double* dG_dq, double* dG_dx,
                     fftsvd_solve_info* info) {
   FFTSVD_REQUIRE(geom, "surface has no panel geometry");
   const int nq = num_charges, np = geom->num_panels;
   double* const b = work_buf(kWorkB, n);
   double* const u = work_buf(kWorkU, n);
   double* const c = work_buf(kWorkC, n);
   double* const lam = work_buf(kWorkLam, n);
   double* const phi = work_buf(kWorkPhi, nq);
   fftsvd_solve_info inf[2] = {};
   // forward: u = A^-1 B q
   rhs_device(*this, b);
   int st = solve(precision, b, u, tol, maxit, &inf[0]);
   if (st != FFTSVD_OK) {
      if (info) info[0] = inf[0];
      return st;
   }
   reaction_device(*this, u, phi);
   *energy = energy_device(*this, phi);
   if (nq == 0) {
      if (info) { info[0] = inf[0]; info[1] = inf[1]; }
      return FFTSVD_OK;
   }
   // adjoint: lambda = A^-T L^T q
   FFTSVD_CUDA(cudaMemsetAsync(c, 0, sizeof(double) * n, stream));
   collection_t_kernel<<<(np + kAdjThreads - 1) / kAdjThreads, kAdjThreads, 0, stream>>>(
       np, geom->panels.get(), geom->phi_row.get(), geom->dphi_row.get(), nq, charge_pos.get(), charge_q.get(), c);
   FFTSVD_CHECK_LAUNCH();
   transposed = true;
   try {
      st = solve(precision, c, lam, tol, maxit, &inf[1]);
   } catch (...) {
      transposed = false;
      throw;
   }
   transposed = false;
   if (info) { info[0] = inf[0]; info[1] = inf[1]; }
   if (st != FFTSVD_OK) return st;
   // per-charge sums
   const int chunks = std::max(1, std::min(kAdjChunks, (np + kAdjPanelTile - 1) / kAdjPanelTile));
   double* const partial = work_buf(kWorkPartial, (size_t)chunks * nq * kAdjOut);
   double* const out = work_buf(kWorkOut, (size_t)nq * kAdjOut);
   dim3 grid((nq + kAdjThreads - 1) / kAdjThreads, chunks);
   adjoint_charge_kernel<<<grid, kAdjThreads, 0, stream>>>(np, geom->panels.get(), geom->phi_row.get(),
                                                           geom->dphi_row.get(), u, lam, nq, charge_pos.get(),
                                                           partial);
   FFTSVD_CHECK_LAUNCH();
   adjoint_reduce_kernel<<<(nq + 127) / 128, 128, 0, stream>>>(nq, chunks, partial, out);
   FFTSVD_CHECK_LAUNCH();
   std::vector<double> h((size_t)nq * kAdjOut);
   FFTSVD_CUDA(cudaMemcpyAsync(h.data(), out, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, stream));
   FFTSVD_CUDA(cudaStreamSynchronize(stream));
   const double k = 332.112 / eps_in;
   for (int j = 0; j < nq; j++) {
      const double* o = &h[(size_t)j * kAdjOut];
      const double qj = charge_q_host[j];
      if (dG_dq) dG_dq[j] = 0.5 * k * (o[0] + o[1]);
      if (dG_dx)
         for (int a = 0; a < 3; a++) dG_dx[3 * j + a] = 0.5 * k * qj * (o[2 + a] + o[5 + a]);
   }
   return FFTSVD_OK;
}

}  // namespace fftsvd

using namespace fftsvd;

extern "C" {

int fftsvd_b200_set_charges(fftsvd_surface* s, int32_t num_charges, const double* charge_pos, const double* charge) {
   if (!s) return FFTSVD_ERR_ARGUMENT;
   return guarded([&] { set_charges(s->s, num_charges, charge_pos, charge); });
}

int fftsvd_b200_matvec_transpose_device(fftsvd_surface* s, int32_t precision, const double* x, double* y) {
   if (!s || !x || !y) return FFTSVD_ERR_ARGUMENT;
   return guarded([&] {
      Surface& S = s->s;
      if (precision == FFTSVD_PREC_FP64)
         S.op64.apply_transpose(x, y, S.stream);
      else
         S.op32.apply_transpose(x, y, S.stream);
   });
}

int fftsvd_b200_matvec_transpose(fftsvd_surface* s, int32_t precision, const double* x, double* y) {
   if (!s || !x || !y) return FFTSVD_ERR_ARGUMENT;
   return guarded([&] {
      Surface& S = s->s;
      FFTSVD_CUDA(cudaMemcpyAsync(S.xin.get(), x, sizeof(double) * S.n, cudaMemcpyHostToDevice, S.stream));
      if (precision == FFTSVD_PREC_FP64)
         S.op64.apply_transpose(S.xin.get(), S.w.get(), S.stream);
      else
         S.op32.apply_transpose(S.xin.get(), S.w.get(), S.stream);
      FFTSVD_CUDA(cudaMemcpyAsync(y, S.w.get(), sizeof(double) * S.n, cudaMemcpyDeviceToHost, S.stream));
      FFTSVD_CUDA(cudaStreamSynchronize(S.stream));
   });
}

int fftsvd_b200_adjoint(fftsvd_surface* s, int32_t precision, double tol, int32_t max_iterations, double* energy,
                        double* dG_dq, double* dG_dx, fftsvd_solve_info* info) {
   if (!s || !energy) return FFTSVD_ERR_ARGUMENT;
   int status = FFTSVD_OK;
   const int rc = guarded([&] { status = s->s.adjoint(precision, tol, max_iterations, energy, dG_dq, dG_dx, info); });
   return rc != FFTSVD_OK ? rc : status;
}

}  // extern "C"
