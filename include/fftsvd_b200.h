/*
 * fftsvd_b200 — B200 (sm_100a) implementation of the FFTSVD boundary-element
 * matvec and GMRES solve for the linearised Poisson-Boltzmann equation.
 *
 * Two C-ABI surfaces live here:
 *
 * 1. Drop-in replacements for the reference entry points of FFTSVDpbeAPI.h
 *    (same names, signatures and ownership).  A program that builds its
 *    operator with the reference host code (generateSurfaceOperator and
 *    generateSurfaceOperatorPreconditioner) relinks against this library and
 *    the solve, the right-hand side and the potential collection run on the
 *    GPU.  The reference structures are read, never modified.
 *
 * 2. fftsvd_b200_* entry points over plain arrays: a surface built by this
 *    library's own host setup from a triangle mesh and point charges, matvec,
 *    solve (FP64 or FP32 operator with FP64 refinement), right-hand side,
 *    reaction potentials and energy.  All return an int status
 *    (FFTSVD_OK = 0) and never exit the process; fftsvd_b200_last_error()
 *    describes the last failure of the calling thread.
 *
 * Kernel and unit conventions follow the reference: Green's function 1/r
 * (Laplace) and exp(-kappa r)/r (Yukawa), no 1/(4 pi); unknowns are
 * x = [phi(0..N-1); dphi/dn(0..N-1)]; energies in kcal/mol.
 */
#ifndef FFTSVD_B200_H
#define FFTSVD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FFTSVD_MAX_DEPTH 16

/* status codes */
#define FFTSVD_OK 0
#define FFTSVD_ERR_ARGUMENT 1      /* invalid argument or size */
#define FFTSVD_ERR_CUDA 2          /* CUDA runtime or launch failure */
#define FFTSVD_ERR_NO_DEVICE 3     /* no CUDA device visible */
#define FFTSVD_ERR_SINGULAR 4      /* singular preconditioner block or GMRES breakdown */
#define FFTSVD_ERR_NOT_CONVERGED 5 /* iteration cap reached above tolerance */
#define FFTSVD_ERR_NONFINITE 6     /* NaN or Inf in input or iterate */
#define FFTSVD_ERR_TIMEOUT 7       /* a bounded device wait expired */
#define FFTSVD_ERR_UNSUPPORTED 8   /* operator topology this build does not handle */

/* solve precision modes */
#define FFTSVD_PREC_FP64 0         /* FP64 operator, FP64 Krylov vectors */
#define FFTSVD_PREC_MIXED 1        /* FP32 operator inside GMRES, FP64 residual refinement */
#define FFTSVD_PREC_FP32 2         /* FP32 operator, FP64 Krylov vectors, no refinement (reference as shipped) */

/*
 * Compressed FFTSVD operator of one region tree, flattened.  Mirrors the
 * content of the reference Tree/Cube objects (Tree.h:3-38, Cube.h:3-54) in
 * struct-of-arrays form.  All matrices are row-major.  Index arrays are
 * zero-based; *_ptr arrays have count+1 entries.
 */
typedef struct {
   int32_t num_panels;            /* source panels of the tree (columns) */
   int32_t num_points;            /* collocation points (rows) */
   int32_t depth;                 /* partitioning levels */
   int32_t grid[FFTSVD_MAX_DEPTH];/* equivalent-density grid edge n per level (Tree.c:158-170) */

   /* near field: every leaf with drows > 0 and dcolumns > 0 (Cube.c:715-793) */
   int32_t num_leaves;
   const int32_t* leaf_row_ptr;   /* [num_leaves+1] into leaf_rows */
   const int32_t* leaf_rows;      /* point indices of the leaf (D rows) */
   const int32_t* leaf_col_ptr;   /* [num_leaves+1] into leaf_cols */
   const int32_t* leaf_cols;      /* own panels, then each local cube's panels (D columns) */
   const int64_t* leaf_d_ptr;     /* [num_leaves+1] element offsets of each drows x dcolumns block */
   const double* d_single;        /* single-layer near-field blocks */
   const double* d_double;        /* double-layer near-field blocks */

   /* far field: every cube with a non-empty interaction list */
   int32_t num_cubes;
   const int32_t* cube_level;     /* [num_cubes] */
   const int32_t* cube_index;     /* [3*num_cubes] integer cube coordinates on its level */
   const int32_t* cube_panel_ptr; /* [num_cubes+1] into cube_panels */
   const int32_t* cube_panels;
   const int32_t* cube_point_ptr; /* [num_cubes+1] into cube_points */
   const int32_t* cube_points;
   const int32_t* cube_row_rank;  /* VTsrc rows; 0 when the cube has no panels */
   const int32_t* cube_col_rank;  /* Udest columns; 0 when the cube has no points */
   const int64_t* cube_vt_ptr;    /* [num_cubes+1]; VT is row_rank x numpanels */
   const double* vt;
   const int64_t* cube_pv_ptr;    /* [num_cubes+1]; PV is n^3 x row_rank */
   const double* pv_single;
   const double* pv_double;
   const int64_t* cube_uti_ptr;   /* [num_cubes+1]; UTI is col_rank x n^3 */
   const double* uti;
   const int64_t* cube_u_ptr;     /* [num_cubes+1]; U is numpoints x col_rank */
   const double* u;
   const int32_t* inter_ptr;      /* [num_cubes+1] into inter_cubes */
   const int32_t* inter_cubes;    /* interacting cubes, as indices into the cube arrays */

   /* translation operators (Tree.c:387-445): per level, 7*7*7 offset slots of
      (2n-1)*(2n-1)*((2n-1)/2+1) complex values (re, im interleaved); slot
      ((dx+3)*7+(dy+3))*7+(dz+3) for dx = dest.index - source.index; slots of
      local offsets are unused */
   const int64_t* t_level_ptr;    /* [depth+1] complex-element offsets */
   const double* t_ops;
} fftsvd_tree_flat;

/*
 * How one region tree reads and writes the global unknown vector
 * (SurfaceOperator.c:51-158).  For tree panel k:
 *   xs[k] = dphi_scale[k] * x[dphi_index[k]]   (single-layer density)
 *   xd[k] = phi_scale[k]  * x[phi_index[k]]    (double-layer density)
 *   y[out_index[k]] = (S xs + D xd)[k] + jump[k] * xd[k]
 */
typedef struct {
   const int32_t* phi_index;
   const double* phi_scale;
   const int32_t* dphi_index;
   const double* dphi_scale;
   const int32_t* out_index;
   const double* jump;
} fftsvd_region_map;

/* Preconditioner entries in compressed-column form (Preconditioner.c:201-225). */
typedef struct {
   int32_t n;
   const int32_t* col_ptr;        /* [n+1] */
   const int32_t* row_index;
   const double* value;
} fftsvd_precond_csc;

/* Problem description for the library's own host setup. */
typedef struct {
   int32_t num_panels;
   const double* vertices;        /* [9*num_panels] v1,v2,v3 per flat triangle, normal = (v3-v1)x(v2-v1) outward */
   int32_t num_charges;
   const double* charge_pos;      /* [3*num_charges] */
   const double* charge;          /* [num_charges] in e */
   double eps_in, eps_out;        /* dielectric constants inside / outside */
   double kappa;                  /* inverse Debye length outside (1/A); 0 selects Laplace outside */
   double svd_tol;                /* FFTSVD sampling tolerance (reference default 1e-5) */
   int32_t max_panels_per_leaf;   /* octree leaf criterion (reference 32) */
   int32_t grid_points;           /* equivalent-density grid edge (reference 4) */
   int32_t num_threads;           /* host threads for setup; 0 = all */
} fftsvd_problem;

typedef struct fftsvd_surface fftsvd_surface;

typedef struct {
   int32_t depth[2];              /* partitioning levels of the exterior and interior trees */
   int32_t num_leaves[2];
   int32_t num_cubes[2];          /* cubes with a non-empty interaction list */
   double setup_ms[8];            /* wall ms of the setup stages: [0] partition + lists, [1] near field,
                                     [2] pinv + translation operators, [3] bases, [4] flattening,
                                     [5] panel integrals in batches (device; inside [1] and [3]),
                                     [6] device layout and upload, [7] the whole surface creation */
   double device_bytes;           /* resident operator bytes, both precisions */
   double matvec_bytes_fp32;      /* algorithmic bytes of one matvec, FP32 operator */
   double matvec_bytes_fp64;      /* algorithmic bytes of one matvec, FP64 operator */
} fftsvd_surface_stats;

typedef struct {
   int32_t iterations;            /* total inner GMRES iterations */
   int32_t refinements;           /* outer FP64 refinement steps (mixed mode) */
   int32_t status;
   double residual;               /* final preconditioned relative residual */
   double setup_ms, solve_ms;
} fftsvd_solve_info;

/* ---- library entry points (no counterpart in the reference unless stated) ---- */

const char* fftsvd_b200_last_error(void);
int fftsvd_b200_version(void);

/* Build a two-region PBE surface (interior Laplace eps_in; exterior Laplace or
   Yukawa eps_out) with this library's host setup and upload it to the current
   CUDA device.  Replaces generateSurfaceOperator + Tree_fill +
   generateSurfaceOperatorPreconditioner (FFTSVDpbeAPI.c:1053-1739,1853-1861). */
int fftsvd_b200_surface_create(const fftsvd_problem* problem, fftsvd_surface** out);

/* The same host setup without any device work: the two region trees in flat
   form (tree 0 exterior, tree 1 interior) and the preconditioner entries.
   The views stay valid until fftsvd_b200_host_operator_free. */
typedef struct fftsvd_host_operator fftsvd_host_operator;
int fftsvd_b200_host_setup(const fftsvd_problem* problem, fftsvd_host_operator** out);
int fftsvd_b200_host_operator_tree(const fftsvd_host_operator* op, int32_t tree, fftsvd_tree_flat* view);
/* The same setup with its panel integrals on the current CUDA device: the near-field
   blocks (Cube.c:715-793), the first sampling pass of every cube's row and column bases
   and the 49-point sphere fits (Cube.c:1104-1281, 795-1002) are integrated in FP64 in one
   batched launch per tree; the rank-revealing factorisations, projections and
   translation operators stay on the host.  The integrals agree with the host ones to
   rounding (the device's FP64 sqrt, log, exp and atan2 against the host's).
   fftsvd_b200_surface_create uses this path. */
int fftsvd_b200_device_setup(const fftsvd_problem* problem, fftsvd_host_operator** out);
/* The device setup's batches of panel integrals evaluated on the host instead: the
   same operator as fftsvd_b200_host_setup, bit for bit (a check of the batch layout
   that needs no GPU). */
int fftsvd_b200_host_setup_batched(const fftsvd_problem* problem, fftsvd_host_operator** out);
int fftsvd_b200_host_operator_precond(const fftsvd_host_operator* op, fftsvd_precond_csc* out);
/* Wall milliseconds of the setup stages, as the first six entries of
   fftsvd_surface_stats.setup_ms. */
int fftsvd_b200_host_operator_timings(const fftsvd_host_operator* op, double* ms6);
void fftsvd_b200_host_operator_free(fftsvd_host_operator* op);

/* Upload an operator given in flat form (one tree per region). */
int fftsvd_b200_surface_create_flat(int32_t num_unknowns, int32_t num_trees, const fftsvd_tree_flat* trees,
                                    const fftsvd_region_map* maps, const fftsvd_precond_csc* precond,
                                    int32_t num_charges, const double* charge_pos, const double* charge,
                                    double eps_in, fftsvd_surface** out);

void fftsvd_b200_surface_free(fftsvd_surface* s);
int32_t fftsvd_b200_surface_num_unknowns(const fftsvd_surface* s);
int fftsvd_b200_surface_stats(const fftsvd_surface* s, fftsvd_surface_stats* out);

/* y = A x.  SurfaceOperator_topmultiply (SurfaceOperator.c:90-97).  Host pointers. */
int fftsvd_b200_matvec(fftsvd_surface* s, int32_t precision, const double* x, double* y);
/* Same with device pointers, asynchronous on the library stream. */
int fftsvd_b200_matvec_device(fftsvd_surface* s, int32_t precision, const double* x, double* y);

/* z = P^-1 r.  Preconditioner_solve (Preconditioner.c:272-294).  Host pointers. */
int fftsvd_b200_precond_solve(fftsvd_surface* s, const double* r, double* z);

/* GMRES solve of A x = rhs (GMRES.c:446-539).  Host pointers. */
int fftsvd_b200_solve(fftsvd_surface* s, int32_t precision, const double* rhs, double* sol, double tol,
                      int32_t max_iterations, fftsvd_solve_info* info);
/* Same with device pointers (rhs, sol resident in HBM). */
int fftsvd_b200_solve_device(fftsvd_surface* s, int32_t precision, const double* rhs, double* sol, double tol,
                             int32_t max_iterations, fftsvd_solve_info* info);

/* Attach the panel geometry of the charge-bearing region to a surface built
   with fftsvd_b200_surface_create_flat: vertices as in fftsvd_problem, and for
   each panel the unknown rows of its phi and dphi/dn. */
int fftsvd_b200_set_geometry(fftsvd_surface* s, int32_t num_panels, const double* vertices, const int32_t* phi_row,
                             const int32_t* dphi_row);

/* rhs[i] = sum_j q_j / |x_j - c_i| on the interior rows (SurfaceOperator.c:291-321). */
int fftsvd_b200_rhs(fftsvd_surface* s, double* rhs);
int fftsvd_b200_rhs_device(fftsvd_surface* s, double* rhs);
/* Reaction potential at every charge from a surface solution
   (SurfaceOperator.c:364-396, direct analytic panel integrals). */
int fftsvd_b200_reaction_potentials(fftsvd_surface* s, const double* sol, double* phi);
int fftsvd_b200_reaction_potentials_device(fftsvd_surface* s, const double* sol, double* phi);

/* The same reaction potentials without any device allocation (no counterpart
   in the reference).  For callers that cannot call cudaMalloc: programs whose
   device memory is owned by another allocator (a framework's caching
   allocator or a pool reserved at start-up, where a stray cudaMalloc fails or
   fragments the pool) and latency-sensitive callers for whom the implicit
   device synchronisation of cudaMalloc/cudaFree is not acceptable.  sol
   (2N doubles) and phi (one double per charge) are device pointers the caller
   allocated; the surface itself was allocated when it was created.
   The call reads sol on the surface's own stream (fftsvd_b200_surface_stream)
   without waiting for any other stream: every write to sol must have finished
   before the call, for example by making the surface's stream wait on an event
   recorded after the writes, or by synchronising the writing stream.
   The per-chunk partial sums live in one file-scope device array of
   524288 doubles (4 MiB), which every GPU that loads this library holds until
   the process exits; surfaces with more than 524288 charges are rejected with
   FFTSVD_ERR_ARGUMENT before any launch.  Up to 8192 charges the panels are
   split into the same 64 chunks as in fftsvd_b200_reaction_potentials; above
   that into 524288 / charges chunks, so the sums are grouped differently and
   agree with the allocating call to rounding, not bit for bit.  The first call
   on a device looks up that array's device address with the surface's device
   current; that first call should come before any stream capture.  All calls
   share the one array and every call overwrites the entries it reads, so
   nothing carries over between calls; calls that overlap on the GPU
   (different threads or streams) race on it.  The call returns after its work
   on the surface's stream has finished. */
int fftsvd_b200_reaction_potentials_noalloc(fftsvd_surface* s, const double* sol, double* phi);
/* 0.5 * sum q phi * 332.112 / eps_in (FFTSVDsalt.c:167-170). */
int fftsvd_b200_energy(fftsvd_surface* s, const double* phi, double* energy);

/* Algorithmic bytes of one matvec at the given precision: compressed operator
   (D, VT, PV, UTI, U) at the stored element size, unique translation tables,
   and the FP64 input and output vectors. */
int fftsvd_b200_matvec_bytes(const fftsvd_surface* s, int32_t precision, double* bytes);

/* Shared-memory bytes one matvec's translation stage moves (staged table and halo rows
   written, source and table rows read): the translation is bound by the SMs' shared-memory
   bandwidth rather than by HBM. */
int fftsvd_b200_translate_smem_bytes(const fftsvd_surface* s, int32_t precision, double* bytes);
/* Algorithmic bytes of each matvec kernel: [join, far_forward, translate, far_backward, near]. */
int fftsvd_b200_matvec_kernel_bytes(const fftsvd_surface* s, int32_t precision, double* bytes5);
/* Run `reps` matvecs on device vectors with CUDA events around each kernel on
   the library stream; average milliseconds per kernel in ms5 (same order). */
int fftsvd_b200_profile_matvec(fftsvd_surface* s, int32_t precision, const double* x, double* y, int32_t reps,
                               double* ms5);
/* The CUDA stream all work of this surface is issued on (cudaStream_t). */
void* fftsvd_b200_surface_stream(const fftsvd_surface* s);

/* ---- tile-shape autotuner (no counterpart in the reference) ---- */

#define FFTSVD_TUNE_MAX_CANDIDATES 8
typedef struct {
   int32_t candidates;                        /* candidate tile limits tried */
   int32_t chosen[2];                         /* index kept for the FP32 and the FP64 operator */
   int32_t max_groups[FFTSVD_TUNE_MAX_CANDIDATES];   /* per candidate: member groups per tile */
   int32_t max_src[FFTSVD_TUNE_MAX_CANDIDATES];      /* halo source spectra per tile */
   int32_t max_entries[FFTSVD_TUNE_MAX_CANDIDATES];  /* (group, source) entries per tile */
   double matvec_ms[2][FFTSVD_TUNE_MAX_CANDIDATES];  /* concurrent matvec time, FP32 and FP64 */
} fftsvd_tune_info;

/* Rebuild the surface's translation tiles under each candidate limit set, time 10
   matvecs of each operator precision with each (after 3 warm-up matvecs) and keep the
   fastest per precision.  The tiles only change launch shapes: every sum keeps its
   order, so later results are bit-for-bit those of the untuned surface.  Synchronises
   the device; do not call it while other work of this surface is in flight.  info may
   be null. */
int fftsvd_b200_surface_autotune(fftsvd_surface* s, fftsvd_tune_info* info);

/* Rebuild the translation tiles of both operators under explicit limits: member groups
   per tile (1..32), halo source spectra per tile (1..320), entries per tile (4..3072).
   The default surface uses 32, 320, 3072.  Like the autotuner this changes launch
   shapes only.  Synchronises the device. */
int fftsvd_b200_surface_set_tile_limits(fftsvd_surface* s, int32_t max_groups, int32_t max_src, int32_t max_entries);

/* ---- adjoint: derivatives of the solvation energy (no counterpart in the
   reference; its FFTSVDforce computes conductor forces, FFTSVDforce.c:111-156) ---- */

/* Replace the surface's point charges (positions [3*num_charges] in A, values in e). */
int fftsvd_b200_set_charges(fftsvd_surface* s, int32_t num_charges, const double* charge_pos, const double* charge);
/* y = A^T x, the transposed surface operator (near blocks and the far field run
   backwards, the translation with the opposite-offset tables).  Column sums use
   FP64 atomics, so results are not bitwise reproducible run to run. */
int fftsvd_b200_matvec_transpose(fftsvd_surface* s, int32_t precision, const double* x, double* y);
int fftsvd_b200_matvec_transpose_device(fftsvd_surface* s, int32_t precision, const double* x, double* y);
/* Solvation energy dG = 1/2 k q^T L A^-1 B q (k = 332.112 / eps_in, B the right-hand
   side of the charges, L the reaction-potential collection) and its exact derivatives
   with respect to every charge (dG_dq, num_charges entries, kcal/mol/e) and every
   charge position (dG_dx, 3 * num_charges entries, kcal/mol/A), from one forward and
   one transposed solve (lambda = A^-T L^T q) at `precision` and `tol`.  dG_dq and
   dG_dx may be NULL; info is NULL or two entries (forward, adjoint solve). */
int fftsvd_b200_adjoint(fftsvd_surface* s, int32_t precision, double tol, int32_t max_iterations, double* energy,
                        double* dG_dq, double* dG_dx, fftsvd_solve_info* info);

/* ---- many right-hand sides of one surface (no counterpart in the reference;
   the batched solve named by the port's plan, fftsvd_b200_solve_batch) ----
   Blocks of k vectors of fftsvd_b200_num_unknowns doubles are stored one vector
   after the other (vector c at base + c * num_unknowns). */

/* Y = A X for nrhs vectors, device pointers.  The multi-vector matvec reads every
   operator element and translation table once per group of 8 right-hand sides;
   each column goes through the same arithmetic as fftsvd_b200_matvec_device.
   Like that call it is issued on the surface's stream and returns before it
   finishes (when nrhs is not a multiple of 8 it waits for a padded copy). */
int fftsvd_b200_matvec_batch_device(fftsvd_surface* s, int32_t precision, int32_t nrhs, const double* x, double* y);
/* Y = A X with the FP32 operator for nrhs vectors (a multiple of 8), device pointers, the
   near field on the tensor cores: per leaf and 128 right-hand sides one kind::tf32 GEMM with
   three-product splitting (FP32-level accuracy; the columns differ from
   fftsvd_b200_matvec_batch_device at FP32 rounding level).  The block solve's inner
   matvecs take this path.  Synchronous.  No counterpart in the reference. */
int fftsvd_b200_matvec_batch_tensor_device(fftsvd_surface* s, int32_t nrhs, const double* x, double* y);
/* Solves A x_c = rhs_c for nrhs columns at once: lockstep GMRES in which every
   column keeps its own Krylov basis, Hessenberg matrix, Givens rotations and
   stopping test (as fftsvd_b200_solve), over the multi-vector matvec.  For
   FFTSVD_PREC_MIXED each column is refined in FP64 as in fftsvd_b200_solve.
   info is NULL or holds nrhs entries (solve_ms is the whole batch).  The basis
   of all columns stays on the device: max_iterations + 1 vectors per column,
   fewer if a third of the free device memory cannot hold them (columns that
   reach that bound report FFTSVD_ERR_NOT_CONVERGED).  Returns the first
   column's non-OK status, else FFTSVD_OK. */
int fftsvd_b200_solve_batch_device(fftsvd_surface* s, int32_t nrhs, int32_t precision, const double* rhs, double* sol,
                                   double tol, int32_t max_iterations, fftsvd_solve_info* info);
/* Same with host pointers. */
int fftsvd_b200_solve_batch(fftsvd_surface* s, int32_t nrhs, int32_t precision, const double* rhs, double* sol,
                            double tol, int32_t max_iterations, fftsvd_solve_info* info);
/* Solves A x_c = rhs_c for nrhs columns by block GMRES (no counterpart in the
   reference): the columns, in blocks of at most 256, share one Krylov space that
   grows by one block of vectors per multi-vector matvec, so each column's solution
   is sought in the span of every column's Krylov vectors and the block needs far
   fewer steps than a column alone.  Stopping test per column as fftsvd_b200_solve:
   preconditioned residual below tol relative to the preconditioned right-hand side,
   the residual recomputed in FP64 for FFTSVD_PREC_MIXED (FP32-operator block
   GMRES inside FP64 refinement; only unconverged columns take part in a refinement
   pass).  Results agree with the single solves to the tolerance, not bit for bit.
   max_iterations caps the block steps of each block of columns; iterations in info
   counts the block steps a column took part in, refinements the refinement passes.
   Zero columns get the zero solution; non-finite columns report
   FFTSVD_ERR_NONFINITE and the others solve.  If the right-hand sides of a block
   are linearly dependent the block falls back to fftsvd_b200_solve_batch_device.
   Returns the first column's non-OK status, else FFTSVD_OK. */
int fftsvd_b200_solve_block_device(fftsvd_surface* s, int32_t nrhs, int32_t precision, const double* rhs, double* sol,
                                   double tol, int32_t max_iterations, fftsvd_solve_info* info);
/* Same with host pointers. */
int fftsvd_b200_solve_block(fftsvd_surface* s, int32_t nrhs, int32_t precision, const double* rhs, double* sol,
                            double tol, int32_t max_iterations, fftsvd_solve_info* info);
/* Solves `count` surfaces concurrently: rhs[i] and sol[i] are device vectors of
   surface i (fftsvd_b200_solve_device semantics per surface), info is NULL or count
   entries.  A pool of host threads drives the solves, each on its surface's device and
   streams, largest surface first, so the surfaces' kernels overlap on the GPU.  Returns
   the first non-OK status (by surface index), else FFTSVD_OK. */
int fftsvd_b200_solve_many(int32_t count, fftsvd_surface* const* surfaces, const double* const* rhs,
                           double* const* sol, int32_t precision, double tol, int32_t max_iterations,
                           fftsvd_solve_info* info);
/* Right-hand sides of charge groups: group g is the surface's charges
   [group_ptr[g], group_ptr[g+1]) (host array of ngroups + 1 non-decreasing
   offsets); rhs (device) receives ngroups vectors (SurfaceOperator.c:291-321
   restricted to the group). */
int fftsvd_b200_rhs_groups_device(fftsvd_surface* s, int32_t ngroups, const int32_t* group_ptr, double* rhs);
/* Solvation energy of each charge group from its own solution column (device
   sol, ngroups vectors): 0.5 sum over the group of q phi_reac * 332.112 / eps_in,
   phi_reac from that column only.  energies is a host array of ngroups. */
int fftsvd_b200_group_energies_device(fftsvd_surface* s, int32_t ngroups, const int32_t* group_ptr, const double* sol,
                                      double* energies);
/* Failure-detection self-test (no counterpart in the reference): one device wait on an
   mbarrier that nothing arrives at, bounded by `polls` polls exactly as the library's
   tensor-core kernels bound their waits.  Returns FFTSVD_ERR_TIMEOUT when the wait gave
   up (the expected outcome; the context stays usable), FFTSVD_ERR_CUDA when it completed. */
int fftsvd_b200_bounded_wait_selftest(int32_t polls);
/* The block solve's dense FP64 kernels on device arrays (column-major), synchronous on the
   legacy default stream.  transpose_a = 0: C (m x n) = alpha A B + beta C with A (m x k);
   transpose_a = 1: C = alpha A^T B + beta C with A (k x m); B is k x n.  Leading dimensions,
   m (transpose_a = 0) and k even, A and B 16-byte aligned; C must not overlap A or B. */
int fftsvd_b200_dense_gemm_device(int transpose_a, int64_t m, int32_t n, int64_t k, double alpha, const double* a,
                                  int64_t lda, const double* b, int64_t ldb, double beta, double* c, int64_t ldc);
/* out (rows x n, ld rows) = R^-1 y for the upper-triangular R (rows x rows, ld ldr), by
   blocks of bs rows (rows a multiple of an even bs); y is overwritten. */
int fftsvd_b200_dense_trsm_device(int32_t rows, int32_t n, int32_t bs, const double* r, int64_t ldr, double* y,
                                  double* out);
/* The block solve's least-squares update on device arrays (column-major), synchronous on
   the legacy default stream: s0 (k x k, upper triangle read) is the first block's factor,
   hbar ((m+1)k x mk) the block upper Hessenberg matrix, whose block columns are fed one at
   a time (rows 0 .. (j+2)k of block column j are read; the k x k block below the diagonal
   block is upper triangular).  After block column j, res[j k + c] is the residual norm of
   min || E1 s0 - Hbar_j Y || in column c; r (mk x mk) receives the triangular factor's
   upper triangle and gtop (mk x k) the transformed right-hand side, so Y = r^-1 gtop.
   k <= 256. */
int fftsvd_b200_block_ls_device(int32_t k, int32_t m, const double* s0, const double* hbar, double* res, double* r,
                                double* gtop);
/* Kernel launches issued by this library since it was loaded. */
long long fftsvd_b200_launch_count(void);
/* Device allocations (cudaMalloc calls) made by this library since it was loaded. */
long long fftsvd_b200_device_alloc_count(void);

/* ---- drop-in replacements for FFTSVDpbeAPI.h (reference types are opaque here) ----
   The declarations in FFTSVDpbeAPI.h are ABI-identical.  PDBentry is an
   unnamed struct there, so the two declarations of collectPotentials are not
   the same C type: a file that includes FFTSVDpbeAPI.h before this header
   gets the reference's declaration only (guarded by its include guard). */

struct _SurfaceOperator;
struct _Preconditioner;
struct PDBentry_s;

/* FFTSVDpbeAPI.h:153 — solution is allocated with calloc (2*numtotalpanels
   doubles) and owned by the caller, as in FFTSVDpbeAPI.c:1884-1888. */
void solveSurfaceOperator(double** solution, struct _SurfaceOperator* pbesurfaceoperator,
                          struct _Preconditioner* preconditioner, double* rhs, unsigned int numtotalpanels);
/* FFTSVDpbeAPI.h:150 — rhs is allocated with calloc (2*numtotalpanels doubles). */
void generateRHS(double** rhs, struct _SurfaceOperator* pbesurfaceoperator, unsigned int numtotalpanels);
/* FFTSVDpbeAPI.h:156 — FFTSVDpbeAPI.c:1896-1922.  Writes
   PDBcollectentries[a].potential = 561 * phi_reac[a] / innerdielectric (kT/e),
   phi_reac[charges->globalindexstart + j] being the reaction potential of
   charge j of every region that holds charges (SurfaceOperator.c:364-401,
   evaluated on the GPU from the host vector solution); when the reference
   global addcoulombic is set, adds 561 q_a / (innerdielectric d) over the input
   entries whose chain is not 'X'.  innerdielectric and addcoulombic are the
   reference's process globals; without an innerdielectric the dielectric
   constant of the charged regions is used.  Regions with an M3 tree are
   rejected.  Errors go to stderr and leave every entry unchanged. */
#ifndef FFTSVDpbeAPI_H
void collectPotentials(struct PDBentry_s* PDBcollectentries, unsigned int numPDBcollectentries,
                       struct PDBentry_s* PDBinputentries, unsigned int numPDBinputentries,
                       struct _SurfaceOperator* pbesurfaceoperator, double* solution);
#endif

#ifdef __cplusplus
}
#endif

#endif
