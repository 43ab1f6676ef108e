/*
 * ORACLE — test infrastructure only.  Never linked into the product.
 *
 * A small C driver over the reference FFTSVD sources (compiled unchanged from
 * the reference tree by oracle/Makefile into oracle/_ref/).  It builds the PBE
 * SurfaceOperator from plain arrays the way the reference drivers do
 * (FFTSVDsalt.c:93-147 for the two-region salt case; FFTSVDpbeAPI.c:1381-1730
 * for the same topology with and without salt), then exposes the operations
 * that tests compare against:
 *
 *   matvec            SurfaceOperator_topmultiply        (SurfaceOperator.c:90-97)
 *   tree matvec       Tree_multiplyboth                  (Tree.c:597-683)
 *   preconditioner    generatePreconditioner + factor/solve (SurfaceOperator.c:170-197,
 *                                                         Preconditioner.c:201-294)
 *   rhs               SurfaceOperator_makeRHS            (SurfaceOperator.c:291-321)
 *   solve             GMRES_SurfaceOperator              (GMRES.c:446-539)
 *   reaction          SurfaceOperator_calculateReactionPotentials (SurfaceOperator.c:323-401)
 *   energy            0.5 * sum q phi * 332.112 / eps_in (FFTSVDsalt.c:167-170)
 *   export            walks Tree/Cube and copies the compressed operator into the
 *                     flat layout declared in include/fftsvd_b200.h, so that the
 *                     product's device kernels can be checked on the reference's
 *                     own operator.
 *
 * It also builds the operator through the reference API entry point
 * generateSurfaceOperator (FFTSVDpbeAPI.c:1053) so that the drop-in symbols of the
 * product can be exercised against reference-built structures.
 */
#include "FFTSVDpbeAPI.h"
#include <string.h>
#include "../include/fftsvd_b200.h"

unsigned int num_GMRES_iter;

typedef struct {
   unsigned int numpanels;
   Panel* panels;
   Vector3D* centroids;
   Charge charge;
   SurfaceOperator outer;     /* root region: outside the dielectric, no own panels */
   SurfaceOperator inner;     /* child region: inside the dielectric, owns the panels */
   Preconditioner precond;
   double kappa;              /* storage the outer tree's parameter pointer refers to */
   double eps_in, eps_out;
   int from_api;
   PDBentry* pdb;
   unsigned int numpdb;
} oref_system;

static void make_panels(oref_system* s, unsigned int numpanels, const double* verts) {
   unsigned int i;
   Vector3D v1 = Vector3D_allocate(), v2 = Vector3D_allocate(), v3 = Vector3D_allocate();
   s->numpanels = numpanels;
   s->panels = (Panel*)calloc(numpanels, sizeof(Panel));
   s->centroids = (Vector3D*)calloc(numpanels, sizeof(Vector3D));
   for (i = 0; i < numpanels; i++) {
      const double* p = verts + 9 * (size_t)i;
      v1->x = p[0]; v1->y = p[1]; v1->z = p[2];
      v2->x = p[3]; v2->y = p[4]; v2->z = p[5];
      v3->x = p[6]; v3->y = p[7]; v3->z = p[8];
      s->panels[i] = Panel_allocate();
      Panel_FlatPanel(s->panels[i], FlatPanel_allocate(v1, v2, v3));
      s->centroids[i] = Vector3D_allocate();
      Vector3D_copy(s->centroids[i], s->panels[i]->centroid);
   }
   Vector3D_free(v1); Vector3D_free(v2); Vector3D_free(v3);
}

static Charge make_charges(unsigned int numcharges, const double* pos, const double* q) {
   unsigned int i;
   Charge c = Charge_allocate();
   c->numcharges = numcharges;
   c->globalindexstart = 0;
   c->points = (Vector3D*)calloc(numcharges, sizeof(Vector3D));
   c->charges = Vector_allocate(numcharges);
   for (i = 0; i < numcharges; i++) {
      c->points[i] = Vector3D_allocate();
      c->points[i]->x = pos[3 * i]; c->points[i]->y = pos[3 * i + 1]; c->points[i]->z = pos[3 * i + 2];
      c->charges[i] = q[i];
   }
   return c;
}

/* Two-region PBE operator with an explicit FFTSVD tolerance (FFTSVDsalt.c:93-147). */
oref_system* oref_create(unsigned int numpanels, const double* verts, unsigned int numcharges, const double* qpos,
                         const double* q, double eps_in, double eps_out, double kappa, double svdtol,
                         unsigned int maxpanels, unsigned int gridpoints) {
   oref_system* s = (oref_system*)calloc(1, sizeof(oref_system));
   unsigned int index = 0;
   BEMKernelType outerkernel = (kappa > 0.0) ? HELMHOLTZ_KERNEL : POISSON_KERNEL;

   make_panels(s, numpanels, verts);
   s->charge = make_charges(numcharges, qpos, q);
   s->kappa = kappa;
   s->eps_in = eps_in;
   s->eps_out = eps_out;

   s->outer = SurfaceOperator_allocate();
   s->outer->kernel = outerkernel;
   s->outer->epsilon = eps_out;
   s->outer->kappa = kappa;
   s->outer->mynumpanels = 0;
   s->outer->tree = Tree_allocate(s->panels, numpanels, s->centroids, numpanels, maxpanels, outerkernel,
                                  (kappa > 0.0) ? (void*)&s->kappa : NULL, gridpoints, svdtol,
                                  SINGLE_AND_DOUBLE_LAYER_INT, 0.0);
   s->outer->numchildren = 1;
   s->outer->children = (SurfaceOperator*)calloc(1, sizeof(SurfaceOperator));
   s->outer->resultInternal = Vector_allocate(numpanels);
   s->outer->resultExternal = Vector_allocate(numpanels);
   s->outer->parent = NULL;
   s->outer->charges = NULL;

   s->inner = SurfaceOperator_allocate();
   s->inner->kernel = POISSON_KERNEL;
   s->inner->epsilon = eps_in;
   s->inner->kappa = 0.0;
   s->inner->mynumpanels = numpanels;
   s->inner->tree = Tree_allocate(s->panels, numpanels, s->centroids, numpanels, maxpanels, POISSON_KERNEL, NULL,
                                  gridpoints, svdtol, SINGLE_AND_DOUBLE_LAYER_INT, 0.0);
   s->inner->numchildren = 0;
   s->inner->children = NULL;
   s->inner->resultInternal = Vector_allocate(numpanels);
   s->inner->resultExternal = Vector_allocate(numpanels);
   s->inner->parent = s->outer;
   s->inner->charges = s->charge;
   s->outer->children[0] = s->inner;

   SurfaceOperator_initStartIndices(s->outer, &index);
   Tree_lists(s->outer->tree);
   Tree_lists(s->inner->tree);
   Tree_fill(s->outer->tree);
   Tree_fill(s->inner->tree);

   s->precond = Preconditioner_allocate(2 * numpanels, 2 * numpanels);
   SurfaceOperator_generatePreconditioner(s->outer, s->precond);
   Preconditioner_factor(s->precond);
   return s;
}

/* The same system built through the reference API entry point
   generateSurfaceOperator (FFTSVDpbeAPI.c:1053), which fixes the FFTSVD
   tolerance at SVD_ERROR, the grid at GRID_SIZE and the leaf size at
   MAX_PANELS_PER_FINEST_CUBE (FFTSVDpbeAPI.h:16-19). */
oref_system* oref_create_api(unsigned int numpanels, const double* verts, unsigned int numcharges,
                             const double* qpos, const double* q, double eps_in, double eps_out,
                             double ionic_strength, double gmres_tol) {
   oref_system* s = (oref_system*)calloc(1, sizeof(oref_system));
   unsigned int i, numpanelsarr[1];
   Panel* dielectric[1];

   make_panels(s, numpanels, verts);
   s->from_api = 1;
   s->eps_in = eps_in;
   s->eps_out = eps_out;
   innerdielectric = eps_in;
   outerdielectric = eps_out;
   ionicstrength = ionic_strength;
   ionexclusionradius = 0.0;
   errortolerance = gmres_tol;

   s->numpdb = numcharges;
   s->pdb = (PDBentry*)calloc(numcharges, sizeof(PDBentry));
   for (i = 0; i < numcharges; i++) {
      s->pdb[i].x = qpos[3 * i]; s->pdb[i].y = qpos[3 * i + 1]; s->pdb[i].z = qpos[3 * i + 2];
      s->pdb[i].charge = q[i];
      s->pdb[i].chain = 'A';
   }
   dielectric[0] = s->panels;
   numpanelsarr[0] = numpanels;
   generateSurfaceOperator(&s->outer, s->pdb, numcharges, NULL, NULL, 0, dielectric, numpanelsarr, 1, NULL,
                           NULL, NULL, 0, NULL, NULL, NULL, 0, NULL, numpanels);
   s->inner = s->outer->children[0];
   s->charge = s->inner->charges;
   generateSurfaceOperatorPreconditioner(&s->precond, s->outer, numpanels);
   return s;
}

void oref_free(oref_system* s) {
   unsigned int i;
   if (!s) return;
   Preconditioner_free(s->precond);
   Tree_free(s->outer->tree);
   Tree_free(s->inner->tree);
   Charge_free(s->charge);
   free(s->outer->children);
   Vector_free(s->outer->resultInternal); Vector_free(s->outer->resultExternal);
   Vector_free(s->inner->resultInternal); Vector_free(s->inner->resultExternal);
   free(s->inner); free(s->outer);
   if (!s->from_api)
      for (i = 0; i < s->numpanels; i++) Vector3D_free(s->centroids[i]);
   free(s->centroids);
   free(s->panels);
   free(s->pdb);
   free(s);
}

/* Opaque reference handles for the drop-in tests. */
void* oref_surface_operator(oref_system* s) { return s->outer; }
void* oref_preconditioner(oref_system* s) { return s->precond; }
unsigned int oref_num_panels(oref_system* s) { return s->numpanels; }
unsigned int oref_depth(oref_system* s, int which) {
   return (which == 0 ? s->outer->tree : s->inner->tree)->partitioningdepth;
}

void oref_matvec(oref_system* s, const double* x, double* y) {
   SurfaceOperator_topmultiply(s->outer, y, (Vector)x);
}

void oref_tree_multiplyboth(oref_system* s, int which, const double* xs, const double* xd, double* b) {
   Tree t = (which == 0) ? s->outer->tree : s->inner->tree;
   Tree_multiplyboth(b, t, (Vector)xs, (Vector)xd);
}

void oref_precond_solve(oref_system* s, const double* b, double* x) {
   Preconditioner_solve(x, s->precond, (Vector)b);
}

void oref_rhs(oref_system* s, double* rhs) {
   memset(rhs, 0, sizeof(double) * 2 * s->numpanels);
   SurfaceOperator_makeRHS(s->outer, rhs);
}

int oref_gmres(oref_system* s, const double* rhs, double* sol, double tol) {
   GMRES_SurfaceOperator(s->outer, s->precond, (Vector)rhs, sol, 2 * s->numpanels, tol);
   return (int)num_GMRES_iter + 1;
}

void oref_reaction(oref_system* s, const double* sol, double* phi) {
   memset(phi, 0, sizeof(double) * s->charge->numcharges);
   SurfaceOperator_calculateReactionPotentials(s->outer, (Vector)sol, phi);
}

double oref_energy(oref_system* s, const double* phi) {
   unsigned int c;
   double e = 0.0;
   for (c = 0; c < s->charge->numcharges; c++) e += 0.5 * s->charge->charges[c] * phi[c];
   return e * 332.112 / s->eps_in;
}

/* Panel integrals straight from the reference (Integration.c:32), for
   checking the product's own integral kernels point by point. */
void oref_panel_integrals(oref_system* s, int kernel, double kappa, unsigned int npts, const double* pts,
                          const unsigned int* panel_of_point, double* slp, double* dlp) {
   unsigned int i;
   Vector3D p = Vector3D_allocate();
   double k = kappa;
   for (i = 0; i < npts; i++) {
      Panel pan = s->panels[panel_of_point[i]];
      p->x = pts[3 * i]; p->y = pts[3 * i + 1]; p->z = pts[3 * i + 2];
      slp[i] = Integration(p, pan, kernel ? HELMHOLTZ_KERNEL : POISSON_KERNEL, kernel ? (void*)&k : NULL,
                           SINGLE_LAYER_INT);
      dlp[i] = Integration(p, pan, kernel ? HELMHOLTZ_KERNEL : POISSON_KERNEL, kernel ? (void*)&k : NULL,
                           DOUBLE_LAYER_INT);
   }
   Vector3D_free(p);
}

/* ---------------- export of the compressed operator ---------------- */

typedef struct {
   /* growable arrays */
   int32_t *leaf_row_ptr, *leaf_rows, *leaf_col_ptr, *leaf_cols;
   int64_t* leaf_d_ptr;
   double *d_single, *d_double;
   int32_t *cube_level, *cube_index, *cube_panel_ptr, *cube_panels, *cube_point_ptr, *cube_points;
   int32_t *cube_row_rank, *cube_col_rank;
   int64_t *cube_vt_ptr, *cube_pv_ptr, *cube_uti_ptr, *cube_u_ptr;
   double *vt, *pv_single, *pv_double, *uti, *u;
   int32_t *inter_ptr, *inter_cubes;
   int64_t* t_level_ptr;
   double* t_ops;
   /* counters */
   int nleaf, ncube;
   long nrows, ncols, nd, npan, npts, nvt, npv, nuti, nu, ninter;
   Cube* cubes;  /* cube pointer per exported cube, for interaction lookups */
} exporter;

static void count_cubes(Cube c, exporter* e, int pass) {
   unsigned int cx, cy, cz;
   if (c->leaf && c->drows > 0 && c->dcolumns > 0) e->nleaf++;
   if (c->numinteractingcubes > 0) {
      if (pass == 1) e->cubes[e->ncube] = c;
      e->ncube++;
   }
   if (!c->leaf)
      for (cx = 0; cx <= 1; cx++)
         for (cy = 0; cy <= 1; cy++)
            for (cz = 0; cz <= 1; cz++)
               if (c->children[cx][cy][cz]) count_cubes(c->children[cx][cy][cz], e, pass);
}

static void export_leaves(Cube c, exporter* e) {
   unsigned int cx, cy, cz, i, j, k;
   if (c->leaf && c->drows > 0 && c->dcolumns > 0) {
      int L = e->nleaf++;
      e->leaf_row_ptr[L] = (int32_t)e->nrows;
      e->leaf_col_ptr[L] = (int32_t)e->ncols;
      e->leaf_d_ptr[L] = e->nd;
      for (i = 0; i < c->numpointindices; i++) e->leaf_rows[e->nrows++] = (int32_t)c->pointindices[i];
      for (i = 0; i < c->numpanelindices; i++) e->leaf_cols[e->ncols++] = (int32_t)c->panelindices[i];
      for (i = 0; i < c->numlocalcubes; i++)
         for (j = 0; j < c->localcubes[i]->numpanelindices; j++)
            e->leaf_cols[e->ncols++] = (int32_t)c->localcubes[i]->panelindices[j];
      for (i = 0; i < c->drows; i++)
         for (k = 0; k < c->dcolumns; k++) {
            e->d_single[e->nd] = c->D_single[i][k];
            e->d_double[e->nd] = c->D_double[i][k];
            e->nd++;
         }
      e->leaf_row_ptr[L + 1] = (int32_t)e->nrows;
      e->leaf_col_ptr[L + 1] = (int32_t)e->ncols;
      e->leaf_d_ptr[L + 1] = e->nd;
   }
   if (!c->leaf)
      for (cx = 0; cx <= 1; cx++)
         for (cy = 0; cy <= 1; cy++)
            for (cz = 0; cz <= 1; cz++)
               if (c->children[cx][cy][cz]) export_leaves(c->children[cx][cy][cz], e);
}

static long leaf_sizes(Cube c, long* rows, long* cols) {
   unsigned int cx, cy, cz;
   long d = 0;
   if (c->leaf && c->drows > 0 && c->dcolumns > 0) {
      *rows += c->drows;
      *cols += c->dcolumns;
      d += (long)c->drows * c->dcolumns;
   }
   if (!c->leaf)
      for (cx = 0; cx <= 1; cx++)
         for (cy = 0; cy <= 1; cy++)
            for (cz = 0; cz <= 1; cz++)
               if (c->children[cx][cy][cz]) d += leaf_sizes(c->children[cx][cy][cz], rows, cols);
   return d;
}

static int find_cube(exporter* e, Cube c) {
   int i;
   for (i = 0; i < e->ncube; i++)
      if (e->cubes[i] == c) return i;
   return -1;
}

/* Fill an owned flat description of one tree (0 = outer region, 1 = inner region).
   All arrays are malloc'd by the driver and released by oref_export_free. */
int oref_export_tree(oref_system* s, int which, fftsvd_tree_flat* out) {
   Tree t = (which == 0) ? s->outer->tree : s->inner->tree;
   exporter e;
   long rows = 0, cols = 0, dsz;
   int c, d;
   long npan = 0, npts = 0, nvt = 0, npv = 0, nuti = 0, nu = 0, ninter = 0, ntop = 0;

   memset(&e, 0, sizeof(e));
   memset(out, 0, sizeof(*out));
   count_cubes(t->root, &e, 0);
   e.cubes = (Cube*)calloc(e.ncube > 0 ? e.ncube : 1, sizeof(Cube));
   e.ncube = 0;
   e.nleaf = 0;
   count_cubes(t->root, &e, 1);

   dsz = leaf_sizes(t->root, &rows, &cols);
   e.leaf_row_ptr = calloc(e.nleaf + 1, sizeof(int32_t));
   e.leaf_col_ptr = calloc(e.nleaf + 1, sizeof(int32_t));
   e.leaf_d_ptr = calloc(e.nleaf + 1, sizeof(int64_t));
   e.leaf_rows = calloc(rows + 1, sizeof(int32_t));
   e.leaf_cols = calloc(cols + 1, sizeof(int32_t));
   e.d_single = calloc(dsz + 1, sizeof(double));
   e.d_double = calloc(dsz + 1, sizeof(double));
   out->num_leaves = e.nleaf;
   e.nleaf = 0;
   export_leaves(t->root, &e);

   for (c = 0; c < e.ncube; c++) {
      Cube cb = e.cubes[c];
      unsigned int gp = t->gridpointsperlevel[cb->level], gp3 = gp * gp * gp, i;
      npan += cb->numpanelindices;
      npts += cb->numpointindices;
      if (cb->numpanelindices > 0 && cb->rowrank > 0) {
         nvt += (long)cb->rowrank * cb->numpanelindices;
         npv += (long)gp3 * cb->rowrank;
      }
      if (cb->numpointindices > 0 && cb->columnrank > 0) {
         nuti += (long)cb->columnrank * gp3;
         nu += (long)cb->numpointindices * cb->columnrank;
      }
      for (i = 0; i < cb->numinteractingcubes; i++) ninter++;
   }
   e.cube_level = calloc(e.ncube + 1, sizeof(int32_t));
   e.cube_index = calloc(3 * e.ncube + 1, sizeof(int32_t));
   e.cube_panel_ptr = calloc(e.ncube + 1, sizeof(int32_t));
   e.cube_point_ptr = calloc(e.ncube + 1, sizeof(int32_t));
   e.cube_panels = calloc(npan + 1, sizeof(int32_t));
   e.cube_points = calloc(npts + 1, sizeof(int32_t));
   e.cube_row_rank = calloc(e.ncube + 1, sizeof(int32_t));
   e.cube_col_rank = calloc(e.ncube + 1, sizeof(int32_t));
   e.cube_vt_ptr = calloc(e.ncube + 1, sizeof(int64_t));
   e.cube_pv_ptr = calloc(e.ncube + 1, sizeof(int64_t));
   e.cube_uti_ptr = calloc(e.ncube + 1, sizeof(int64_t));
   e.cube_u_ptr = calloc(e.ncube + 1, sizeof(int64_t));
   e.vt = calloc(nvt + 1, sizeof(double));
   e.pv_single = calloc(npv + 1, sizeof(double));
   e.pv_double = calloc(npv + 1, sizeof(double));
   e.uti = calloc(nuti + 1, sizeof(double));
   e.u = calloc(nu + 1, sizeof(double));
   e.inter_ptr = calloc(e.ncube + 1, sizeof(int32_t));
   e.inter_cubes = calloc(ninter + 1, sizeof(int32_t));

   for (c = 0; c < e.ncube; c++) {
      Cube cb = e.cubes[c];
      unsigned int gp = t->gridpointsperlevel[cb->level], gp3 = gp * gp * gp, i, j;
      e.cube_level[c] = (int32_t)cb->level;
      e.cube_index[3 * c] = (int32_t)cb->indices[0];
      e.cube_index[3 * c + 1] = (int32_t)cb->indices[1];
      e.cube_index[3 * c + 2] = (int32_t)cb->indices[2];
      e.cube_panel_ptr[c] = (int32_t)e.npan;
      for (i = 0; i < cb->numpanelindices; i++) e.cube_panels[e.npan++] = (int32_t)cb->panelindices[i];
      e.cube_point_ptr[c] = (int32_t)e.npts;
      for (i = 0; i < cb->numpointindices; i++) e.cube_points[e.npts++] = (int32_t)cb->pointindices[i];
      e.cube_vt_ptr[c] = e.nvt;
      e.cube_pv_ptr[c] = e.npv;
      e.cube_uti_ptr[c] = e.nuti;
      e.cube_u_ptr[c] = e.nu;
      if (cb->numpanelindices > 0 && cb->rowrank > 0) {
         e.cube_row_rank[c] = (int32_t)cb->rowrank;
         for (i = 0; i < cb->rowrank; i++)
            for (j = 0; j < cb->numpanelindices; j++) e.vt[e.nvt++] = cb->VTsrc[i][j];
         for (i = 0; i < gp3; i++)
            for (j = 0; j < cb->rowrank; j++) {
               e.pv_single[e.npv] = cb->PV_single[i][j];
               e.pv_double[e.npv] = cb->PV_double[i][j];
               e.npv++;
            }
      }
      if (cb->numpointindices > 0 && cb->columnrank > 0) {
         e.cube_col_rank[c] = (int32_t)cb->columnrank;
         for (i = 0; i < cb->columnrank; i++)
            for (j = 0; j < gp3; j++) e.uti[e.nuti++] = cb->UTI[i][j];
         for (i = 0; i < cb->numpointindices; i++)
            for (j = 0; j < cb->columnrank; j++) e.u[e.nu++] = cb->Udest[i][j];
      }
      e.inter_ptr[c] = (int32_t)e.ninter;
      for (i = 0; i < cb->numinteractingcubes; i++) e.inter_cubes[e.ninter++] = find_cube(&e, cb->interactingcubes[i]);
   }
   e.cube_panel_ptr[e.ncube] = (int32_t)e.npan;
   e.cube_point_ptr[e.ncube] = (int32_t)e.npts;
   e.cube_vt_ptr[e.ncube] = e.nvt;
   e.cube_pv_ptr[e.ncube] = e.npv;
   e.cube_uti_ptr[e.ncube] = e.nuti;
   e.cube_u_ptr[e.ncube] = e.nu;
   e.inter_ptr[e.ncube] = (int32_t)e.ninter;

   /* translation operators: 7x7x7 offsets per level, local offsets left zero */
   e.t_level_ptr = calloc(t->partitioningdepth + 1, sizeof(int64_t));
   for (d = 0; d < (int)t->partitioningdepth; d++) {
      unsigned int np = 2 * t->gridpointsperlevel[d] - 1;
      e.t_level_ptr[d] = ntop;
      ntop += 343L * np * np * (np / 2 + 1);
   }
   e.t_level_ptr[t->partitioningdepth] = ntop;
   e.t_ops = calloc(2 * ntop + 2, sizeof(double));
   for (d = 0; d < (int)t->partitioningdepth; d++) {
      unsigned int np = 2 * t->gridpointsperlevel[d] - 1, pg = np * np * (np / 2 + 1);
      int x, y, z;
      for (x = 0; x < 7; x++)
         for (y = 0; y < 7; y++)
            for (z = 0; z < 7; z++) {
               ComplexSVector tv = t->Tprecomputed[d][x][y][z];
               long base = e.t_level_ptr[d] + (long)((x * 7 + y) * 7 + z) * pg;
               unsigned int f;
               if (!tv) continue;
               for (f = 0; f < pg; f++) {
                  e.t_ops[2 * (base + f)] = creal(tv[f]);
                  e.t_ops[2 * (base + f) + 1] = cimag(tv[f]);
               }
            }
   }

   out->num_panels = (int32_t)t->numpanels;
   out->num_points = (int32_t)t->numpoints;
   out->depth = (int32_t)t->partitioningdepth;
   for (d = 0; d < (int)t->partitioningdepth && d < FFTSVD_MAX_DEPTH; d++) out->grid[d] = (int32_t)t->gridpointsperlevel[d];
   out->leaf_row_ptr = e.leaf_row_ptr; out->leaf_rows = e.leaf_rows;
   out->leaf_col_ptr = e.leaf_col_ptr; out->leaf_cols = e.leaf_cols;
   out->leaf_d_ptr = e.leaf_d_ptr; out->d_single = e.d_single; out->d_double = e.d_double;
   out->num_cubes = e.ncube;
   out->cube_level = e.cube_level; out->cube_index = e.cube_index;
   out->cube_panel_ptr = e.cube_panel_ptr; out->cube_panels = e.cube_panels;
   out->cube_point_ptr = e.cube_point_ptr; out->cube_points = e.cube_points;
   out->cube_row_rank = e.cube_row_rank; out->cube_col_rank = e.cube_col_rank;
   out->cube_vt_ptr = e.cube_vt_ptr; out->vt = e.vt;
   out->cube_pv_ptr = e.cube_pv_ptr; out->pv_single = e.pv_single; out->pv_double = e.pv_double;
   out->cube_uti_ptr = e.cube_uti_ptr; out->uti = e.uti;
   out->cube_u_ptr = e.cube_u_ptr; out->u = e.u;
   out->inter_ptr = e.inter_ptr; out->inter_cubes = e.inter_cubes;
   out->t_level_ptr = e.t_level_ptr; out->t_ops = e.t_ops;
   free(e.cubes);
   return 0;
}

void oref_export_free(fftsvd_tree_flat* f) {
   free((void*)f->leaf_row_ptr); free((void*)f->leaf_rows); free((void*)f->leaf_col_ptr); free((void*)f->leaf_cols);
   free((void*)f->leaf_d_ptr); free((void*)f->d_single); free((void*)f->d_double);
   free((void*)f->cube_level); free((void*)f->cube_index); free((void*)f->cube_panel_ptr); free((void*)f->cube_panels);
   free((void*)f->cube_point_ptr); free((void*)f->cube_points); free((void*)f->cube_row_rank); free((void*)f->cube_col_rank);
   free((void*)f->cube_vt_ptr); free((void*)f->vt); free((void*)f->cube_pv_ptr); free((void*)f->pv_single);
   free((void*)f->pv_double); free((void*)f->cube_uti_ptr); free((void*)f->uti); free((void*)f->cube_u_ptr);
   free((void*)f->u); free((void*)f->inter_ptr); free((void*)f->inter_cubes); free((void*)f->t_level_ptr);
   free((void*)f->t_ops);
   memset(f, 0, sizeof(*f));
}

/* ---- input front end (FFTSVDpbeAPI.c), for checking the product's readers ----
 * getFlatPanels (:676-712) and readSRF (:776-1032) return reference Panel objects; these
 * copy their corner coordinates (FlatPanel.vertex, in FlatPanel_allocate order) to plain
 * arrays.  The reference's own readers must only be given valid files: they exit on errors. */
static unsigned int copy_flat(Panel* panels, unsigned int n, double* verts, unsigned int room) {
   unsigned int i, k;
   for (i = 0; i < n && i < room; i++) {
      FlatPanel fp = (FlatPanel)panels[i]->realpanel;
      for (k = 0; k < 3; k++) {
         verts[9 * (size_t)i + 3 * k + 0] = fp->vertex[k]->x;
         verts[9 * (size_t)i + 3 * k + 1] = fp->vertex[k]->y;
         verts[9 * (size_t)i + 3 * k + 2] = fp->vertex[k]->z;
      }
   }
   return n < room ? n : room;
}

unsigned int oref_flat_panels(const char* basename, unsigned int accessible, unsigned int cavity,
                              unsigned int qualocation, double* verts, unsigned int maxpanels) {
   Panel* panels = NULL;
   unsigned int n = 0;
   usequalocation = qualocation;
   getFlatPanels(basename, &panels, &n, accessible, cavity);
   usequalocation = 0;
   copy_flat(panels, n, verts, maxpanels);
   return n;
}

/* counts: numsalts, numdielectrics, numdielectriccavities, numsaltcavities, numtotalpanels.
 * layer_n: panels per layer, salts then dielectrics, dielectric cavities, salt cavities.
 * parents: dielectricparent, dielectriccavityparent, saltcavityparent, in that order.
 * verts: the panels of all layers in the same order (at most maxpanels). */
void oref_read_srf(const char* filename, unsigned int* counts, unsigned int* layer_n, unsigned int* parents,
                   unsigned int maxlayers, double* verts, unsigned int maxpanels) {
   Panel **sp = NULL, **dp = NULL, **dcp = NULL, **scp = NULL;
   unsigned int *nsp = NULL, *ndp = NULL, *ndcp = NULL, *nscp = NULL;
   unsigned int ns = 0, nd = 0, ndc = 0, nsc = 0, total = 0;
   unsigned int *dpar = NULL, *dcpar = NULL, *scpar = NULL;
   unsigned int i, l = 0, p = 0, done = 0;
   readSRF(filename, &sp, &nsp, &ns, &dp, &ndp, &nd, &dpar, &dcp, &ndcp, &ndc, &dcpar, &scp, &nscp, &nsc, &scpar,
           &total);
   counts[0] = ns; counts[1] = nd; counts[2] = ndc; counts[3] = nsc; counts[4] = total;
   for (i = 0; i < ns && l < maxlayers; i++, l++) { layer_n[l] = nsp[i]; done += copy_flat(sp[i], nsp[i], verts + 9 * (size_t)done, maxpanels - done); }
   for (i = 0; i < nd && l < maxlayers; i++, l++) { layer_n[l] = ndp[i]; done += copy_flat(dp[i], ndp[i], verts + 9 * (size_t)done, maxpanels - done); }
   for (i = 0; i < ndc && l < maxlayers; i++, l++) { layer_n[l] = ndcp[i]; done += copy_flat(dcp[i], ndcp[i], verts + 9 * (size_t)done, maxpanels - done); }
   for (i = 0; i < nsc && l < maxlayers; i++, l++) { layer_n[l] = nscp[i]; done += copy_flat(scp[i], nscp[i], verts + 9 * (size_t)done, maxpanels - done); }
   for (i = 0; i < nd && p < maxlayers; i++) parents[p++] = dpar[i];
   for (i = 0; i < ndc && p < maxlayers; i++) parents[p++] = dcpar[i];
   for (i = 0; i < nsc && p < maxlayers; i++) parents[p++] = scpar[i];
}
