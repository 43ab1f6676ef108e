// The surface object behind the C-ABI: both operator precisions, the
// block-diagonal preconditioner, the GMRES workspace and (optionally) the
// panel geometry and point charges used by the right-hand side and the
// reaction-potential collection.
#pragma once

#include <cuda_runtime.h>

#include <memory>
#include <vector>

#include "batch.h"
#include "block.h"
#include "common.h"
#include "gmres.cuh"
#include "operator.h"

namespace fftsvd {

struct PanelGeometry;  // nbody.h

// Share of the tolerance the FP32-operator inner solves of the mixed mode aim at (single
// and lockstep-batch solves): the FP64 refinement residual then stays below the tolerance
// by the FP32 operator's ~1e-7 relative error.
constexpr double kInnerTarget = 0.8;

struct Preconditioner {
   int nblocks = 0;
   DevBuf<int32_t> blk_ptr, blk_idx;
   DevBuf<int64_t> inv_off;
   DevBuf<double> inv, inv_t;  // block inverses and their transposes
   void build(const fftsvd_precond_csc& P, int n);  // host factorisation into dense block inverses
   // z = P^-1 r, or P^-T r for the transposed system
   void apply(const double* r, double* z, cudaStream_t s, bool transpose = false) const;
};

struct Surface {
   int n = 0;  // unknowns
   int device = 0;  // CUDA device ordinal the surface lives on
   cudaStream_t stream = nullptr;
   DeviceOperator<double> op64;
   DeviceOperator<float> op32;
   Preconditioner precond;
   int64_t operator_elems = 0, t_elems = 0;
   KernelBytes kernel_bytes;
   double eps_in = 1.0;
   // inner region (interior, Laplace) tree panel -> unknown rows, for RHS and collection
   std::vector<int32_t> inner_phi_row, inner_dphi_row;
   std::shared_ptr<PanelGeometry> geom;
   int num_charges = 0;
   DevBuf<double> charge_pos, charge_q;
   std::vector<double> charge_q_host;

   // setup statistics (zero for surfaces built from a flat operator)
   fftsvd_surface_stats stats{};

   // Work arrays of the adjoint and of the reaction-potential collection, kept between calls
   // (grown when a call needs more, never shrunk): allocating and freeing them per call put
   // cudaMalloc/cudaFree, which synchronise the device, inside every adjoint.
   enum WorkSlot { kWorkB, kWorkU, kWorkC, kWorkLam, kWorkPhi, kWorkPartial, kWorkOut, kWorkReact, kWorkSlots };
   DevBuf<double> work[kWorkSlots];
   double* work_buf(WorkSlot slot, size_t elems);

   // GMRES workspace
   int capacity = 0;  // basis vectors
   DevBuf<double> V, H, cs, sn, g, h1, h2, partial, normpart, y;
   DevBuf<double> w, r, t0, t1, t2, xin, xout, sold, scal, krylov_in;
   DevBuf<GivensState> st;
   GivensState* st_host = nullptr;
   DevBuf<double2> hist;           // per Arnoldi step {residual, flag}
   double2* hist_host = nullptr;   // pinned copy, capacity entries

   // One Arnoldi step's operator application, krylov_in -> w = P^-1 A krylov_in, captured
   // once per (operator precision, direction) as a CUDA graph: one launch replays the
   // join, the concurrent grid-size chains and near field, the far-field add and the
   // preconditioner.  Rebuilt after the translation tiles change.
   struct StepGraph {
      cudaGraphExec_t exec = nullptr;
      long long kernels = 0;  // kernel nodes, for fftsvd_b200_launch_count
   };
   StepGraph step_graphs[2][2];   // [FP64 operator][transposed]
   void step_apply(int precision);
   void release_step_graphs();

   ~Surface();
   void ensure_capacity(int nvec);
   // While `transposed` is set, apply, pinv, gmres and solve work on A^T and P^T (adjoint solves).
   bool transposed = false;
   void apply(int precision, const double* x, double* y);
   void pinv(const double* r, double* z);
   double pnorm(const double* v);  // ||v|| on device, synchronous
   // Left-preconditioned un-restarted GMRES (GMRES.c:446-539) with operator `precision`;
   // x overwritten.  Returns iterations; residual via *res.
   int gmres(int precision, const double* rhs, double* x, double tol, int maxit, double* res, int* status,
             bool absolute_zero_check = true);
   int solve(int precision, const double* rhs, double* x, double tol, int maxit, fftsvd_solve_info* info);
   // Translation tile shapes: each candidate timed on both operators, the fastest kept (tune.cu).
   std::shared_ptr<TileProblems> tile_problems;
   void autotune(fftsvd_tune_info* info);
   void set_tile_limits(int max_groups, int max_src, int max_entries);
   // Solvation energy and its derivatives with respect to the charges and their positions
   // (adjoint.cu); dG_dq holds num_charges entries, dG_dx 3 * num_charges; info[0] is the
   // forward solve, info[1] the adjoint (transposed) solve.
   int adjoint(int precision, double tol, int maxit, double* energy, double* dG_dq, double* dG_dx,
               fftsvd_solve_info* info);

   // ---- many right-hand sides (batch.cu); blocks of ncols vectors, column c at base + c * n
   std::unique_ptr<BatchWorkspace> bw;
   int batch_chunk32 = 0, batch_chunk64 = 0;  // columns per batched matvec launch sequence
   int batch_chunk(int precision);
   void apply_batch(int precision, const double* X, double* Y, int ncols);
   void precond_batch(const double* r, double* z, int ncols);
   void pnorm_batch(const double* v, int ncols, std::vector<double>& out);
   // Lockstep GMRES over ncols columns; columns with run[c] == 0 stay zero.
   int gmres_batch(int precision, int ncols, const double* rhs, double* x, const std::vector<double>& tol, int maxit,
                   const std::vector<char>& run, bool absolute_zero_check, std::vector<double>& res,
                   std::vector<int>& iters, std::vector<int>& status);
   // k right-hand sides; info may be null or hold k entries.  Returns the first non-OK status.
   int solve_batch(int precision, int k, const double* rhs, double* x, double tol, int maxit,
                   fftsvd_solve_info* info);

   // ---- block GMRES over one shared Krylov space (block.cu)
   std::unique_ptr<BlockWorkspace> blk;
   void block_qr(const double* X, double* Q, int K);
   int gmres_block(int precision, int K, const double* R0, double* X, int nmon, const std::vector<double>& target,
                   int mmax, std::vector<double>& res);
   int solve_block(int precision, int k, const double* rhs, double* x, double tol, int maxit,
                   fftsvd_solve_info* info);
};

void init_surface(Surface& S, int num_unknowns, int num_trees, const fftsvd_tree_flat* trees,
                  const fftsvd_region_map* maps, const fftsvd_precond_csc* P);

}  // namespace fftsvd

struct fftsvd_surface {
   fftsvd::Surface s;
};
