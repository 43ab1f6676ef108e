// Surface object, preconditioner, GMRES driver and the fftsvd_b200_* C-ABI.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>

#include "batch.h"
#include "nbody.h"
#include "block.h"
#include "block_ls.h"
#include "dense.h"
#include "surface.h"

namespace fftsvd {

std::atomic<long long> g_kernel_launches{0};
std::atomic<long long> g_device_allocs{0};
static thread_local std::string g_last_error;
void set_last_error(const std::string& msg) { g_last_error = msg; }

// ------------------------------------------------------------------ preconditioner

// Split the assembled sparse matrix into connected components of its pattern
// (one 2x2 block per panel for the PBE operator, SurfaceOperator.c:183-193)
// and store the dense inverse of each.  Entries given twice are summed.
void Preconditioner::build(const fftsvd_precond_csc& P, int n) {
   FFTSVD_REQUIRE(P.n == n, "preconditioner size does not match the operator");
   std::vector<int> parent(n);
   std::iota(parent.begin(), parent.end(), 0);
   auto find = [&](int a) {
      while (parent[a] != a) a = parent[a] = parent[parent[a]];
      return a;
   };
   for (int c = 0; c < n; c++)
      for (int k = P.col_ptr[c]; k < P.col_ptr[c + 1]; k++) {
         const int r = P.row_index[k];
         FFTSVD_REQUIRE(r >= 0 && r < n, "preconditioner row out of range");
         const int a = find(r), b = find(c);
         if (a != b) parent[a] = b;
      }
   std::vector<int> root_block(n, -1), local(n), size;
   std::vector<std::vector<int>> members;
   for (int i = 0; i < n; i++) {
      const int rt = find(i);
      if (root_block[rt] < 0) {
         root_block[rt] = (int)members.size();
         members.emplace_back();
      }
      const int b = root_block[rt];
      local[i] = (int)members[b].size();
      members[b].push_back(i);
   }
   nblocks = (int)members.size();
   std::vector<int32_t> ptr(nblocks + 1, 0), idx;
   std::vector<int64_t> off(nblocks);
   std::vector<double> inv;
   std::vector<std::vector<double>> dense(nblocks);
   for (int b = 0; b < nblocks; b++) {
      const int k = (int)members[b].size();
      if (k > 8) throw Error(FFTSVD_ERR_UNSUPPORTED, "preconditioner block larger than 8 unknowns");
      dense[b].assign((size_t)k * k, 0.0);
   }
   for (int c = 0; c < n; c++)
      for (int k = P.col_ptr[c]; k < P.col_ptr[c + 1]; k++) {
         const int r = P.row_index[k];
         const int b = root_block[find(c)];
         const int kk = (int)members[b].size();
         dense[b][(size_t)local[r] * kk + local[c]] += P.value[k];
      }
   for (int b = 0; b < nblocks; b++) {
      const int k = (int)members[b].size();
      ptr[b + 1] = ptr[b] + k;
      for (int i : members[b]) idx.push_back(i);
      off[b] = (int64_t)inv.size();
      // Gauss-Jordan with partial pivoting
      std::vector<double> a = dense[b], e((size_t)k * k, 0.0);
      for (int i = 0; i < k; i++) e[(size_t)i * k + i] = 1.0;
      for (int col = 0; col < k; col++) {
         int piv = col;
         for (int i = col + 1; i < k; i++)
            if (std::fabs(a[(size_t)i * k + col]) > std::fabs(a[(size_t)piv * k + col])) piv = i;
         if (a[(size_t)piv * k + col] == 0.0 || !std::isfinite(a[(size_t)piv * k + col]))
            throw Error(FFTSVD_ERR_SINGULAR, "singular preconditioner block at unknown " + std::to_string(members[b][col]));
         if (piv != col)
            for (int j = 0; j < k; j++) {
               std::swap(a[(size_t)piv * k + j], a[(size_t)col * k + j]);
               std::swap(e[(size_t)piv * k + j], e[(size_t)col * k + j]);
            }
         const double d = a[(size_t)col * k + col];
         for (int j = 0; j < k; j++) { a[(size_t)col * k + j] /= d; e[(size_t)col * k + j] /= d; }
         for (int i = 0; i < k; i++) {
            if (i == col) continue;
            const double f = a[(size_t)i * k + col];
            if (f == 0.0) continue;
            for (int j = 0; j < k; j++) {
               a[(size_t)i * k + j] -= f * a[(size_t)col * k + j];
               e[(size_t)i * k + j] -= f * e[(size_t)col * k + j];
            }
         }
      }
      inv.insert(inv.end(), e.begin(), e.end());
   }
   blk_ptr.upload(ptr);
   blk_idx.upload(idx);
   inv_off.upload(off);
   this->inv.upload(inv);
   // inverse of the transposed block = transpose of the inverse (adjoint solves)
   std::vector<double> invt(inv.size());
   for (int b = 0; b < nblocks; b++) {
      const int k = ptr[b + 1] - ptr[b];
      for (int i = 0; i < k; i++)
         for (int j = 0; j < k; j++) invt[off[b] + (size_t)i * k + j] = inv[off[b] + (size_t)j * k + i];
   }
   this->inv_t.upload(invt);
}

void Preconditioner::apply(const double* r, double* z, cudaStream_t s, bool transpose) const {
   const int threads = 256;
   const int blocks = std::max(1, std::min((nblocks + threads - 1) / threads, 148 * 8));
   precond_kernel<<<blocks, threads, 0, s>>>(nblocks, blk_ptr.get(), blk_idx.get(), inv_off.get(),
                                             transpose ? inv_t.get() : inv.get(), r, z, 0);
   FFTSVD_CHECK_LAUNCH();
}

// ------------------------------------------------------------------ surface

Surface::~Surface() {
   blk.reset();  // its events and buffers go before the stream they were used on
   release_step_graphs();
   if (st_host) cudaFreeHost(st_host);
   if (hist_host) cudaFreeHost(hist_host);
   if (stream) cudaStreamDestroy(stream);
}

double* Surface::work_buf(WorkSlot slot, size_t elems) {
   DevBuf<double>& b = work[slot];
   elems = std::max<size_t>(elems, 1);
   if (b.size() < elems) b.alloc(elems);
   return b.get();
}

void Surface::release_step_graphs() {
   for (auto& byprec : step_graphs)
      for (StepGraph& g : byprec) {
         if (g.exec) cudaGraphExecDestroy(g.exec);
         g.exec = nullptr;
         g.kernels = 0;
      }
}

void Surface::step_apply(int precision) {
   StepGraph& g = step_graphs[precision == FFTSVD_PREC_FP64 ? 1 : 0][transposed ? 1 : 0];
   if (!g.exec) {
      // capture on the surface's stream: the operator's chain and near-field streams fork
      // from it and join back into it, so the graph holds the whole concurrent matvec
      FFTSVD_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
      cudaGraph_t graph = nullptr;
      try {
         apply(precision, krylov_in.get(), w.get());
         pinv(w.get(), w.get());
      } catch (...) {
         cudaStreamEndCapture(stream, &graph);
         if (graph) cudaGraphDestroy(graph);
         throw;
      }
      FFTSVD_CUDA(cudaStreamEndCapture(stream, &graph));
      // kernel nodes of the graph: the launch count is charged when the graph runs
      size_t nodes = 0;
      cudaError_t e = cudaGraphGetNodes(graph, nullptr, &nodes);
      std::vector<cudaGraphNode_t> list(nodes);
      if (e == cudaSuccess && nodes) e = cudaGraphGetNodes(graph, list.data(), &nodes);
      long long kernels = 0;
      for (size_t k = 0; e == cudaSuccess && k < nodes; k++) {
         cudaGraphNodeType type;
         e = cudaGraphNodeGetType(list[k], &type);
         if (type == cudaGraphNodeTypeKernel) kernels++;
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&g.exec, graph, 0);
      cudaGraphDestroy(graph);
      FFTSVD_CUDA(e);
      g.kernels = kernels;
      g_kernel_launches.fetch_sub(kernels);  // the captured launches did not run
   }
   FFTSVD_CUDA(cudaGraphLaunch(g.exec, stream));
   g_kernel_launches.fetch_add(g.kernels);
}

void Surface::ensure_capacity(int nvec) {
   if (nvec <= capacity) return;
   const int64_t nb = vec_blocks(n);
   V.alloc((size_t)nvec * n);
   H.alloc((size_t)nvec * nvec);
   cs.alloc(nvec);
   sn.alloc(nvec);
   g.alloc(nvec);
   h1.alloc(nvec);
   h2.alloc(nvec);
   y.alloc(nvec);
   partial.alloc((size_t)nvec * nb);
   hist.alloc(nvec);
   if (hist_host) cudaFreeHost(hist_host);
   hist_host = nullptr;
   FFTSVD_CUDA(cudaMallocHost(&hist_host, sizeof(double2) * nvec));
   capacity = nvec;
}

void Surface::apply(int precision, const double* x, double* yv) {
   if (transposed) {
      if (precision == FFTSVD_PREC_FP64)
         op64.apply_transpose(x, yv, stream);
      else
         op32.apply_transpose(x, yv, stream);
   } else if (precision == FFTSVD_PREC_FP64) {
      op64.apply(x, yv, stream);
   } else {
      op32.apply(x, yv, stream);
   }
}

void Surface::pinv(const double* r_in, double* z) { precond.apply(r_in, z, stream, transposed); }

double Surface::pnorm(const double* v) {
   const int nb = vec_blocks(n);
   norm_partial_kernel<<<nb, kVecThreads, 0, stream>>>(n, v, normpart.get(), 0, 0);
   FFTSVD_CHECK_LAUNCH();
   reduce_partial_kernel<<<1, 256, 0, stream>>>(1, nb, normpart.get(), scal.get(), 0, 0, 0);
   FFTSVD_CHECK_LAUNCH();
   double s = 0.0;
   FFTSVD_CUDA(cudaMemcpyAsync(&s, scal.get(), sizeof(double), cudaMemcpyDeviceToHost, stream));
   FFTSVD_CUDA(cudaStreamSynchronize(stream));
   return std::sqrt(s);
}

int Surface::gmres(int precision, const double* rhs, double* x, double tol, int maxit, double* res, int* status,
                   bool absolute_zero_check) {
   const int nb = vec_blocks(n), nd = dot_blocks(n);
   const int ew_blocks = std::max(1, std::min((n + 255) / 256, 148 * 8));
   ensure_capacity(maxit + 1);
   *status = FFTSVD_OK;
   FFTSVD_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, stream));
   // r = P^-1 rhs (GMRES.c:457-465)
   pinv(rhs, r.get());
   const double normr = pnorm(r.get());
   if (!std::isfinite(normr)) {
      *status = FFTSVD_ERR_NONFINITE;
      *res = normr;
      return 0;
   }
   if (absolute_zero_check && normr < tol) {  // hand back zero solution (GMRES.c:461-465)
      *res = 0.0;
      return 0;
   }
   double* Vp = V.get();
   const int64_t ldv = n;
   // v0 = r / |r|, also into the operator's input buffer
   scale_kernel<<<ew_blocks, 256, 0, stream>>>(n, r.get(), nullptr, 1.0 / normr, Vp, 0, 0, krylov_in.get());
   FFTSVD_CHECK_LAUNCH();
   FFTSVD_CUDA(cudaMemsetAsync(g.get(), 0, sizeof(double) * capacity, stream));
   FFTSVD_CUDA(cudaMemcpyAsync(g.get(), &normr, sizeof(double), cudaMemcpyHostToDevice, stream));
   st_host->normr = normr;
   st_host->residual = 1.0;
   st_host->flag = 0;
   FFTSVD_CUDA(cudaMemcpyAsync(st.get(), st_host, sizeof(GivensState), cudaMemcpyHostToDevice, stream));

   // Arnoldi step i (GMRES.c:470-503): w = P^-1 A v_i (one graph launch), CGS2 against
   // v_0..v_i, the Givens update on the device, v_{i+1} = w / beta (also into the
   // operator's input buffer for step i + 1).  The residual of every step lands in hist.
   auto step = [&](int i) {
      const int nvec = i + 1;
      double* vnext = Vp + (int64_t)(i + 1) * ldv;
      step_apply(precision);
      // CGS2: h1 = V^T w, w -= V h1, h2 = V^T w, vnext = w - V h2 with its norm partials
      const size_t sh = sizeof(double) * nvec;
      dots_partial_kernel<<<dim3(nd, nvec), kVecThreads, 0, stream>>>(n, nvec, Vp, ldv, w.get(), partial.get(), 0, 0);
      FFTSVD_CHECK_LAUNCH();
      update_kernel<<<nb, kVecThreads, sh, stream>>>(n, nvec, Vp, ldv, partial.get(), nd, h1.get(), w.get(), w.get(),
                                                     nullptr, 0, 0, 0, 0);
      FFTSVD_CHECK_LAUNCH();
      dots_partial_kernel<<<dim3(nd, nvec), kVecThreads, 0, stream>>>(n, nvec, Vp, ldv, w.get(), partial.get(), 0, 0);
      FFTSVD_CHECK_LAUNCH();
      update_kernel<<<nb, kVecThreads, sh, stream>>>(n, nvec, Vp, ldv, partial.get(), nd, h2.get(), w.get(), vnext,
                                                     normpart.get(), 0, 0, 0, 0);
      FFTSVD_CHECK_LAUNCH();
      givens_kernel<<<1, 256, givens_smem(i), stream>>>(i, capacity, H.get(), h1.get(), h2.get(), normpart.get(), nb,
                                                        cs.get(), sn.get(), g.get(), st.get(), 0, 0, nullptr,
                                                        hist.get());
      FFTSVD_CHECK_LAUNCH();
      scale_kernel<<<ew_blocks, 256, 0, stream>>>(n, vnext, &st.get()->inv_beta, 0.0, vnext, 0, 0, krylov_in.get());
      FFTSVD_CHECK_LAUNCH();
   };

   // Steps are issued in runs without waiting in between: the host reads the residual
   // history only after each run.  A run is as long as the residual's recent rate of decrease
   // predicts the solve to stay above tol (at most kMaxRun steps, one step near the end).
   // Steps issued past the converged one add basis vectors and Hessenberg columns that the
   // solution never uses: GMRES's least-squares problem of the first k steps does not
   // depend on later ones.
   constexpr int kMaxRun = 8;
   int i = 0, last = -1;
   double resid = 1.0;
   while (i < maxit && last < 0) {
      int run = 1;
      if (i >= 4) {
         const double r_now = hist_host[i - 1].x, r_past = hist_host[i - 4].x;
         if (r_now > 0.0 && r_past > r_now) {
            const double per_step = std::log(r_now / r_past) / 3.0;  // < 0
            const double left = std::log(tol / r_now) / per_step;     // steps still predicted above tol
            run = (int)std::max(1.0, std::min((double)kMaxRun, std::floor(0.6 * left)));
         }
      }
      run = std::min(run, maxit - i);
      for (int j = 0; j < run; j++) step(i + j);
      FFTSVD_CUDA(cudaMemcpyAsync(hist_host + i, hist.get() + i, sizeof(double2) * run, cudaMemcpyDeviceToHost,
                                  stream));
      FFTSVD_CUDA(cudaStreamSynchronize(stream));
      for (int j = 0; j < run; j++) {
         const int flag = (int)hist_host[i + j].y;
         resid = hist_host[i + j].x;
         if (flag == 2) {
            *status = FFTSVD_ERR_NONFINITE;
            last = i + j;
            break;
         }
         if (resid < tol || flag == 1) {
            last = i + j;
            break;
         }
      }
      i += run;
   }
   if (last < 0) {
      last = maxit - 1;
      *status = FFTSVD_ERR_NOT_CONVERGED;
   }
   // back substitution on the host (GMRES.c:512-521): k <= 1000 unknowns
   const int k = last + 1;
   std::vector<double> Hh((size_t)k * capacity), gh(k), yh(k);
   FFTSVD_CUDA(cudaMemcpyAsync(Hh.data(), H.get(), sizeof(double) * (size_t)k * capacity, cudaMemcpyDeviceToHost, stream));
   FFTSVD_CUDA(cudaMemcpyAsync(gh.data(), g.get(), sizeof(double) * k, cudaMemcpyDeviceToHost, stream));
   FFTSVD_CUDA(cudaStreamSynchronize(stream));
   for (int q = 0; q < k; q++) yh[q] = gh[q];
   for (int q = k - 1; q >= 0; q--) {
      yh[q] /= Hh[(size_t)q * capacity + q];
      for (int j = q - 1; j >= 0; j--) yh[j] -= Hh[(size_t)q * capacity + j] * yh[q];
   }
   FFTSVD_CUDA(cudaMemcpyAsync(y.get(), yh.data(), sizeof(double) * k, cudaMemcpyHostToDevice, stream));
   combine_kernel<<<ew_blocks, 256, sizeof(double) * k, stream>>>(n, k, Vp, ldv, y.get(), x, 0, 0);
   FFTSVD_CHECK_LAUNCH();
   FFTSVD_CUDA(cudaStreamSynchronize(stream));
   *res = resid;
   return k;
}

int Surface::solve(int precision, const double* rhs, double* x, double tol, int maxit, fftsvd_solve_info* info) {
   FFTSVD_REQUIRE(tol > 0.0 && maxit > 0, "tolerance and iteration cap must be positive");
   const auto clock_start = std::chrono::steady_clock::now();
   int status = FFTSVD_OK, iters = 0, refinements = 0;
   double res = 0.0;
   if (precision == FFTSVD_PREC_FP64 || precision == FFTSVD_PREC_FP32) {
      iters = gmres(precision, rhs, x, tol, maxit, &res, &status);
   } else if (precision == FFTSVD_PREC_MIXED) {
      // FP64 iterative refinement around FP32-operator GMRES: x += A32^-1 (b - A64 x)
      const int ew_blocks = std::max(1, std::min((n + 255) / 256, 148 * 8));
      pinv(rhs, t0.get());
      const double bn = pnorm(t0.get());
      FFTSVD_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, stream));
      FFTSVD_CUDA(cudaMemcpyAsync(t1.get(), rhs, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
      res = 1.0;
      if (!std::isfinite(bn)) status = FFTSVD_ERR_NONFINITE;
      else if (bn < tol) res = 0.0;
      // Each inner solve targets an absolute preconditioned error of kInnerTarget tol
      // ||P^-1 b||: the first one therefore runs to kInnerTarget tol, a correction to
      // kInnerTarget tol / (current residual).  The FP32 operator differs from the FP64 one
      // by ~1e-7 relative, far below the remaining 1 - kInnerTarget of the tolerance, so
      // one correction is rarely needed and the FP64 operator is applied once per
      // refinement only.
      for (refinements = 0; status == FFTSVD_OK && res >= tol && refinements < 8; refinements++) {
         double inner_res = 0.0;
         int st2 = FFTSVD_OK;
         const double inner_tol = std::min(0.1, std::max(kInnerTarget * tol / res, 1e-13));
         iters += gmres(FFTSVD_PREC_FP32, t1.get(), xout.get(), inner_tol, maxit, &inner_res, &st2, false);
         if (st2 == FFTSVD_ERR_NONFINITE) { status = st2; break; }
         add_kernel<<<ew_blocks, 256, 0, stream>>>(n, xout.get(), x, 0);
         FFTSVD_CHECK_LAUNCH();
         apply(FFTSVD_PREC_FP64, x, t2.get());
         sub_kernel<<<ew_blocks, 256, 0, stream>>>(n, rhs, t2.get(), t1.get(), 0);
         FFTSVD_CHECK_LAUNCH();
         pinv(t1.get(), t0.get());
         res = pnorm(t0.get()) / bn;
         if (!std::isfinite(res)) status = FFTSVD_ERR_NONFINITE;
      }
      if (status == FFTSVD_OK && res >= tol) status = FFTSVD_ERR_NOT_CONVERGED;
   } else {
      throw Error(FFTSVD_ERR_ARGUMENT, "unknown precision mode");
   }
   FFTSVD_CUDA(cudaStreamSynchronize(stream));
   if (op32.tensor_status(true) | op64.tensor_status(true))
      throw Error(FFTSVD_ERR_TIMEOUT, "a bounded device wait of the matvec gave up (results discarded)");
   const auto clock_end = std::chrono::steady_clock::now();
   if (info) {
      info->iterations = iters;
      info->refinements = refinements;
      info->status = status;
      info->residual = res;
      info->solve_ms = std::chrono::duration<double, std::milli>(clock_end - clock_start).count();
   }
   return status;
}

void init_surface(Surface& S, int num_unknowns, int num_trees, const fftsvd_tree_flat* trees,
                         const fftsvd_region_map* maps, const fftsvd_precond_csc* P) {
   int ndev = 0;
   if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      throw Error(FFTSVD_ERR_NO_DEVICE, "no CUDA device visible");
   FFTSVD_REQUIRE(trees && maps && P, "null operator description");
   S.n = num_unknowns;
   FFTSVD_CUDA(cudaGetDevice(&S.device));
   FFTSVD_CUDA(cudaStreamCreateWithFlags(&S.stream, cudaStreamNonBlocking));
   OperatorLayout L = build_layout(num_unknowns, num_trees, trees, maps);
   S.operator_elems = L.operator_elems;
   S.t_elems = L.t_elems;
   S.kernel_bytes = L.kernel_bytes;
   S.tile_problems = L.problems;
   S.op64.upload(L);
   S.op32.upload(L);
   S.precond.build(*P, num_unknowns);
   const int nb = vec_blocks(num_unknowns);
   S.w.alloc(num_unknowns);
   S.r.alloc(num_unknowns);
   S.t0.alloc(num_unknowns);
   S.t1.alloc(num_unknowns);
   S.t2.alloc(num_unknowns);
   S.xin.alloc(num_unknowns);
   S.xout.alloc(num_unknowns);
   S.sold.alloc(num_unknowns);
   S.krylov_in.alloc(num_unknowns);
   S.scal.alloc(8);
   S.normpart.alloc(nb);
   S.st.alloc(1);
   FFTSVD_CUDA(cudaMallocHost(&S.st_host, sizeof(GivensState)));
   FFTSVD_CUDA(cudaDeviceSynchronize());
}

}  // namespace fftsvd

using namespace fftsvd;

extern "C" {

const char* fftsvd_b200_last_error(void) { return g_last_error.c_str(); }
int fftsvd_b200_version(void) { return 100; }

int fftsvd_b200_surface_create_flat(int32_t num_unknowns, int32_t num_trees, const fftsvd_tree_flat* trees,
                                    const fftsvd_region_map* maps, const fftsvd_precond_csc* precond,
                                    int32_t num_charges, const double* charge_pos, const double* charge,
                                    double eps_in, fftsvd_surface** out) {
   if (!out) return FFTSVD_ERR_ARGUMENT;
   *out = nullptr;
   fftsvd_surface* s = new (std::nothrow) fftsvd_surface();
   if (!s) return FFTSVD_ERR_ARGUMENT;
   int rc = guarded([&] {
      init_surface(s->s, num_unknowns, num_trees, trees, maps, precond);
      s->s.eps_in = eps_in;
      set_charges(s->s, num_charges, charge_pos, charge);
   });
   if (rc != FFTSVD_OK) {
      delete s;
      return rc;
   }
   *out = s;
   return FFTSVD_OK;
}

void fftsvd_b200_surface_free(fftsvd_surface* s) { delete s; }

int32_t fftsvd_b200_surface_num_unknowns(const fftsvd_surface* s) { return s ? s->s.n : 0; }

int fftsvd_b200_matvec_device(fftsvd_surface* s, int32_t precision, const double* x, double* y) {
   if (!s || !x || !y) return FFTSVD_ERR_ARGUMENT;
   return guarded([&] { s->s.apply(precision == FFTSVD_PREC_FP64 ? FFTSVD_PREC_FP64 : FFTSVD_PREC_FP32, x, y); });
}

int fftsvd_b200_matvec(fftsvd_surface* s, int32_t precision, const double* x, double* y) {
   if (!s || !x || !y) return FFTSVD_ERR_ARGUMENT;
   return guarded([&] {
      Surface& S = s->s;
      FFTSVD_CUDA(cudaMemcpyAsync(S.xin.get(), x, sizeof(double) * S.n, cudaMemcpyHostToDevice, S.stream));
      S.apply(precision == FFTSVD_PREC_FP64 ? FFTSVD_PREC_FP64 : FFTSVD_PREC_FP32, S.xin.get(), S.w.get());
      FFTSVD_CUDA(cudaMemcpyAsync(y, S.w.get(), sizeof(double) * S.n, cudaMemcpyDeviceToHost, S.stream));
      FFTSVD_CUDA(cudaStreamSynchronize(S.stream));
      if (S.op32.tensor_status(true) | S.op64.tensor_status(true))
         throw Error(FFTSVD_ERR_TIMEOUT, "a bounded device wait of the matvec gave up (results discarded)");
   });
}

int fftsvd_b200_precond_solve(fftsvd_surface* s, const double* r, double* z) {
   if (!s || !r || !z) return FFTSVD_ERR_ARGUMENT;
   return guarded([&] {
      Surface& S = s->s;
      FFTSVD_CUDA(cudaMemcpyAsync(S.xin.get(), r, sizeof(double) * S.n, cudaMemcpyHostToDevice, S.stream));
      S.precond.apply(S.xin.get(), S.w.get(), S.stream);
      FFTSVD_CUDA(cudaMemcpyAsync(z, S.w.get(), sizeof(double) * S.n, cudaMemcpyDeviceToHost, S.stream));
      FFTSVD_CUDA(cudaStreamSynchronize(S.stream));
   });
}

int fftsvd_b200_solve_device(fftsvd_surface* s, int32_t precision, const double* rhs, double* sol, double tol,
                             int32_t max_iterations, fftsvd_solve_info* info) {
   if (!s || !rhs || !sol) return FFTSVD_ERR_ARGUMENT;
   int status = FFTSVD_OK;
   int rc = guarded([&] { status = s->s.solve(precision, rhs, sol, tol, max_iterations, info); });
   if (rc != FFTSVD_OK) return rc;
   if (status != FFTSVD_OK)
      set_last_error(status == FFTSVD_ERR_NOT_CONVERGED ? "GMRES reached the iteration cap above tolerance"
                                                        : "non-finite value in the right-hand side or an iterate");
   return status;
}

int fftsvd_b200_solve(fftsvd_surface* s, int32_t precision, const double* rhs, double* sol, double tol,
                      int32_t max_iterations, fftsvd_solve_info* info) {
   if (!s || !rhs || !sol) return FFTSVD_ERR_ARGUMENT;
   int status = FFTSVD_OK;
   int rc = guarded([&] {
      Surface& S = s->s;
      FFTSVD_CUDA(cudaMemcpyAsync(S.xin.get(), rhs, sizeof(double) * S.n, cudaMemcpyHostToDevice, S.stream));
      status = S.solve(precision, S.xin.get(), S.sold.get(), tol, max_iterations, info);
      FFTSVD_CUDA(cudaMemcpyAsync(sol, S.sold.get(), sizeof(double) * S.n, cudaMemcpyDeviceToHost, S.stream));
      FFTSVD_CUDA(cudaStreamSynchronize(S.stream));
   });
   if (rc != FFTSVD_OK) return rc;
   return status;
}

long long fftsvd_b200_launch_count(void) { return g_kernel_launches.load(); }

int fftsvd_b200_bounded_wait_selftest(int32_t polls) {
   if (polls <= 0) return FFTSVD_ERR_ARGUMENT;
   int result = 0;
   const int rc = guarded([&] { result = bounded_wait_selftest(polls); });
   if (rc != FFTSVD_OK) return rc;
   if (result == 1) {
      set_last_error("bounded device wait gave up as expected");
      return FFTSVD_ERR_TIMEOUT;
   }
   set_last_error("bounded device wait completed without an arrival");
   return FFTSVD_ERR_CUDA;
}
long long fftsvd_b200_device_alloc_count(void) { return g_device_allocs.load(); }

int fftsvd_b200_dense_gemm_device(int transpose_a, int64_t m, int32_t n, int64_t k, double alpha, const double* a,
                                  int64_t lda, const double* b, int64_t ldb, double beta, double* c, int64_t ldc) {
   if (m < 0 || n < 0 || k < 0 || !a || !b || !c) return FFTSVD_ERR_ARGUMENT;
   return guarded([&] {
      FFTSVD_REQUIRE(ldc >= m && ldb >= k && lda >= (transpose_a ? k : m), "leading dimensions");
      if (transpose_a) {
         FFTSVD_REQUIRE(m <= INT32_MAX, "rows");
         DevBuf<double> work((size_t)std::max<int64_t>(1, dense::gemm_tn_work((int)m, n, k)));
         dense::gemm_tn((int)m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, work.get(), nullptr);
         FFTSVD_CUDA(cudaStreamSynchronize(nullptr));
      } else {
         FFTSVD_REQUIRE(k <= INT32_MAX, "inner dimension");
         dense::gemm_nn(m, n, (int)k, alpha, a, lda, b, ldb, beta, c, ldc, nullptr);
         FFTSVD_CUDA(cudaStreamSynchronize(nullptr));
      }
   });
}

int fftsvd_b200_dense_trsm_device(int32_t rows, int32_t n, int32_t bs, const double* r, int64_t ldr, double* y,
                                  double* out) {
   if (rows < 0 || n < 0 || bs <= 0 || !r || !y || !out || ldr < rows) return FFTSVD_ERR_ARGUMENT;
   return guarded([&] {
      DevBuf<double> dinv((size_t)std::max(1, rows) * bs);
      dense::trsm_upper_left(rows, n, bs, r, ldr, y, dinv.get(), out, nullptr);
      FFTSVD_CUDA(cudaStreamSynchronize(nullptr));
   });
}

int fftsvd_b200_block_ls_device(int32_t k, int32_t m, const double* s0, const double* hbar, double* res, double* r,
                                double* gtop) {
   if (k <= 0 || k > kBlockMax || m <= 0 || !s0 || !hbar || !res || !r || !gtop) return FFTSVD_ERR_ARGUMENT;
   return guarded([&] {
      const int64_t K = k, ldh = (int64_t)(m + 1) * K, cols = (int64_t)m * K;
      DevBuf<double> V((size_t)m * 2 * K * K), tau((size_t)m * K), g((size_t)ldh * K), col((size_t)ldh * K),
          stat((size_t)3 * K + 1);
      lsq::init(k, s0, g.get(), ldh, nullptr);
      for (int j = 0; j < m; j++) {
         const double* h = hbar + (int64_t)j * K * ldh;
         lsq::gather(j, k, h, ldh, h + (int64_t)(j + 1) * K, ldh, nullptr, col.get(), ldh, stat.get(), nullptr);
         lsq::step(j, k, col.get(), ldh, V.get(), tau.get(), g.get(), ldh, r, cols, stat.get(), nullptr);
         FFTSVD_CUDA(cudaMemcpyAsync(res + (int64_t)j * K, stat.get(), sizeof(double) * K, cudaMemcpyDeviceToDevice,
                                     nullptr));
      }
      FFTSVD_CUDA(cudaMemcpy2DAsync(gtop, sizeof(double) * cols, g.get(), sizeof(double) * ldh, sizeof(double) * cols,
                                    K, cudaMemcpyDeviceToDevice, nullptr));
      FFTSVD_CUDA(cudaStreamSynchronize(nullptr));
   });
}

void* fftsvd_b200_surface_stream(const fftsvd_surface* s) { return s ? (void*)s->s.stream : nullptr; }

int fftsvd_b200_matvec_kernel_bytes(const fftsvd_surface* s, int32_t precision, double* bytes5) {
   if (!s || !bytes5) return FFTSVD_ERR_ARGUMENT;
   const KernelBytes& kb = s->s.kernel_bytes;
   const double es = precision == FFTSVD_PREC_FP64 ? 8.0 : 4.0;
   for (int k = 0; k < kNumKernels; k++) bytes5[k] = kb.elems[k] * es + kb.fixed[k];
   return FFTSVD_OK;
}

int fftsvd_b200_profile_matvec(fftsvd_surface* s, int32_t precision, const double* x, double* y, int32_t reps,
                               double* ms5) {
   if (!s || !x || !y || !ms5 || reps <= 0) return FFTSVD_ERR_ARGUMENT;
   return guarded([&] {
      Surface& S = s->s;
      double acc[kNumKernels] = {0, 0, 0, 0, 0};
      for (int r = 0; r < reps; r++) {
         float t[kNumKernels];
         if (precision == FFTSVD_PREC_FP64) {
            S.op64.enable_timing(true);
            S.op64.apply(x, y, S.stream);
            S.op64.stage_ms(t);
            S.op64.enable_timing(false);
         } else {
            S.op32.enable_timing(true);
            S.op32.apply(x, y, S.stream);
            S.op32.stage_ms(t);
            S.op32.enable_timing(false);
         }
         for (int k = 0; k < kNumKernels; k++) acc[k] += t[k];
      }
      for (int k = 0; k < kNumKernels; k++) ms5[k] = acc[k] / reps;
   });
}

int fftsvd_b200_translate_smem_bytes(const fftsvd_surface* s, int32_t precision, double* bytes) {
   if (!s || !bytes) return FFTSVD_ERR_ARGUMENT;
   *bytes = precision == FFTSVD_PREC_FP64 ? s->s.op64.translate_smem_bytes() : s->s.op32.translate_smem_bytes();
   return FFTSVD_OK;
}

int fftsvd_b200_matvec_bytes(const fftsvd_surface* s, int32_t precision, double* bytes) {
   if (!s || !bytes) return FFTSVD_ERR_ARGUMENT;
   const double es = precision == FFTSVD_PREC_FP64 ? 8.0 : 4.0;
   *bytes = (double)s->s.operator_elems * es + (double)s->s.t_elems * es + 2.0 * s->s.n * 8.0;
   return FFTSVD_OK;
}

}  // extern "C"
