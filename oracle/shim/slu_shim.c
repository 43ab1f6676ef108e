/*
 * Test-infrastructure shim (oracle only): exact block LU behind the SuperLU
 * calls of the reference preconditioner.  See slu_ddefs.h.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "slu_ddefs.h"

/* One factored connected component: dense LU with row pivots. */
typedef struct {
   int size;
   int* index;     /* global row/column indices of the component */
   double* lu;     /* size x size, row-major, L unit-lower and U upper */
   int* piv;       /* row pivot order */
} oracle_block;

typedef struct {
   int n;
   int numblocks;
   oracle_block* blocks;
   long stored;
} oracle_factor;

void StatInit(SuperLUStat_t* stat) { stat->TinyPivots = 0; stat->RefineSteps = 0; }
void StatFree(SuperLUStat_t* stat) { (void)stat; }
void set_default_options(superlu_options_t* options) { options->Fact = 0; options->DiagPivotThresh = 1.0; }
int sp_ienv(int ispec) { return ispec == 1 ? 12 : 6; }

void get_perm_c(int ispec, SuperMatrix* A, int* perm_c) {
   int i;
   (void)ispec;
   for (i = 0; i < A->ncol; i++) perm_c[i] = i;
}

void sp_preorder(superlu_options_t* options, SuperMatrix* A, int* perm_c, int* etree, SuperMatrix* AC) {
   (void)options; (void)perm_c; (void)etree;
   *AC = *A;
}

void dCreate_CompCol_Matrix(SuperMatrix* A, int m, int n, int nnz, double* nzval, int* rowind, int* colptr,
                            Stype_t stype, Dtype_t dtype, Mtype_t mtype) {
   NCformat* s = (NCformat*)malloc(sizeof(NCformat));
   s->nnz = nnz; s->nzval = nzval; s->rowind = rowind; s->colptr = colptr;
   A->Stype = stype; A->Dtype = dtype; A->Mtype = mtype; A->nrow = m; A->ncol = n; A->Store = s;
}

void dCreate_Dense_Matrix(SuperMatrix* X, int m, int n, double* x, int ldx, Stype_t stype, Dtype_t dtype,
                          Mtype_t mtype) {
   DNformat* s = (DNformat*)malloc(sizeof(DNformat));
   s->lda = ldx; s->nzval = x;
   X->Stype = stype; X->Dtype = dtype; X->Mtype = mtype; X->nrow = m; X->ncol = n; X->Store = s;
}

static int uf_find(int* parent, int a) {
   while (parent[a] != a) {
      parent[a] = parent[parent[a]];
      a = parent[a];
   }
   return a;
}

void dgstrf(superlu_options_t* options, SuperMatrix* A, int relax, int panel_size, int* etree, void* work,
            int lwork, int* perm_c, int* perm_r, SuperMatrix* L, SuperMatrix* U, GlobalLU_t* Glu,
            SuperLUStat_t* stat, int* info) {
   NCformat* s = (NCformat*)A->Store;
   int n = A->ncol, c, k, i, j;
   int* parent = (int*)malloc(sizeof(int) * n);
   int* root_to_block = (int*)malloc(sizeof(int) * n);
   int* fill = (int*)calloc(n, sizeof(int));
   int* local = (int*)malloc(sizeof(int) * n);
   double* val = (double*)s->nzval;
   oracle_factor* f = (oracle_factor*)calloc(1, sizeof(oracle_factor));
   (void)options; (void)relax; (void)panel_size; (void)etree; (void)work; (void)lwork; (void)perm_c;
   (void)Glu; (void)stat;

   *info = 0;
   for (i = 0; i < n; i++) { parent[i] = i; perm_r[i] = i; }
   for (c = 0; c < n; c++)
      for (k = s->colptr[c]; k < s->colptr[c + 1]; k++) {
         int a = uf_find(parent, s->rowind[k]), b = uf_find(parent, c);
         if (a != b) parent[a] = b;
      }

   f->n = n;
   for (i = 0; i < n; i++) root_to_block[i] = -1;
   for (i = 0; i < n; i++) {
      int r = uf_find(parent, i);
      if (root_to_block[r] < 0) root_to_block[r] = f->numblocks++;
   }
   f->blocks = (oracle_block*)calloc(f->numblocks, sizeof(oracle_block));
   for (i = 0; i < n; i++) f->blocks[root_to_block[uf_find(parent, i)]].size++;
   for (i = 0; i < f->numblocks; i++) {
      int sz = f->blocks[i].size;
      f->blocks[i].index = (int*)malloc(sizeof(int) * sz);
      f->blocks[i].lu = (double*)calloc((size_t)sz * sz, sizeof(double));
      f->blocks[i].piv = (int*)malloc(sizeof(int) * sz);
      f->stored += (long)sz * sz;
   }
   for (i = 0; i < n; i++) {
      int b = root_to_block[uf_find(parent, i)];
      local[i] = fill[b];
      f->blocks[b].index[fill[b]++] = i;
   }
   /* scatter entries; duplicates add, as a sparse assembly would */
   for (c = 0; c < n; c++)
      for (k = s->colptr[c]; k < s->colptr[c + 1]; k++) {
         int r = s->rowind[k];
         oracle_block* blk = &f->blocks[root_to_block[uf_find(parent, c)]];
         blk->lu[local[r] * blk->size + local[c]] += val[k];
      }
   /* dense LU with partial pivoting per block */
   for (i = 0; i < f->numblocks && *info == 0; i++) {
      oracle_block* blk = &f->blocks[i];
      int sz = blk->size;
      double* a = blk->lu;
      for (j = 0; j < sz; j++) blk->piv[j] = j;
      for (k = 0; k < sz; k++) {
         int p = k;
         double best = fabs(a[k * sz + k]);
         for (j = k + 1; j < sz; j++)
            if (fabs(a[j * sz + k]) > best) { best = fabs(a[j * sz + k]); p = j; }
         if (best == 0.0) { *info = blk->index[k] + 1; break; }
         if (p != k) {
            int t = blk->piv[k]; blk->piv[k] = blk->piv[p]; blk->piv[p] = t;
            for (j = 0; j < sz; j++) { double tv = a[k * sz + j]; a[k * sz + j] = a[p * sz + j]; a[p * sz + j] = tv; }
         }
         for (j = k + 1; j < sz; j++) {
            int m;
            double l = a[j * sz + k] / a[k * sz + k];
            a[j * sz + k] = l;
            for (m = k + 1; m < sz; m++) a[j * sz + m] -= l * a[k * sz + m];
         }
      }
   }
   L->Stype = SLU_SC; L->Dtype = SLU_D; L->Mtype = SLU_TRLU; L->nrow = n; L->ncol = n; L->Store = f;
   U->Stype = SLU_NC; U->Dtype = SLU_D; U->Mtype = SLU_TRU; U->nrow = n; U->ncol = n; U->Store = NULL;
   free(parent); free(root_to_block); free(fill); free(local);
}

void dgstrs(trans_t trans, SuperMatrix* L, SuperMatrix* U, int* perm_c, int* perm_r, SuperMatrix* B,
            SuperLUStat_t* stat, int* info) {
   oracle_factor* f = (oracle_factor*)L->Store;
   DNformat* d = (DNformat*)B->Store;
   double* x = (double*)d->nzval;
   double work[64], y[64];
   int i, j, k;
   (void)U; (void)perm_c; (void)perm_r; (void)stat;
   *info = 0;
   if (trans != NOTRANS) { *info = -1; return; }
   for (i = 0; i < f->numblocks; i++) {
      oracle_block* blk = &f->blocks[i];
      int sz = blk->size;
      double* a = blk->lu;
      double *w = work, *yy = y;
      if (sz > 64) { w = (double*)malloc(sizeof(double) * sz); yy = (double*)malloc(sizeof(double) * sz); }
      for (j = 0; j < sz; j++) w[j] = x[blk->index[blk->piv[j]]];
      for (j = 0; j < sz; j++) {          /* forward: unit lower */
         double acc = w[j];
         for (k = 0; k < j; k++) acc -= a[j * sz + k] * yy[k];
         yy[j] = acc;
      }
      for (j = sz - 1; j >= 0; j--) {     /* backward: upper */
         double acc = yy[j];
         for (k = j + 1; k < sz; k++) acc -= a[j * sz + k] * yy[k];
         yy[j] = acc / a[j * sz + j];
      }
      for (j = 0; j < sz; j++) x[blk->index[j]] = yy[j];
      if (sz > 64) { free(w); free(yy); }
   }
}

int dQuerySpace(SuperMatrix* L, SuperMatrix* U, mem_usage_t* mem_usage) {
   oracle_factor* f = (oracle_factor*)L->Store;
   (void)U;
   mem_usage->for_lu = f ? (float)(f->stored * sizeof(double)) : 0.0f;
   mem_usage->total_needed = mem_usage->for_lu;
   return 0;
}

void Destroy_SuperMatrix_Store(SuperMatrix* A) { free(A->Store); A->Store = NULL; }
void Destroy_CompCol_Permuted(SuperMatrix* A) { (void)A; /* shares the store of the unpermuted matrix */ }
void Destroy_CompCol_Matrix(SuperMatrix* A) { (void)A; }
void Destroy_SuperNode_Matrix(SuperMatrix* A) {
   oracle_factor* f = (oracle_factor*)A->Store;
   int i;
   if (!f) return;
   for (i = 0; i < f->numblocks; i++) {
      free(f->blocks[i].index); free(f->blocks[i].lu); free(f->blocks[i].piv);
   }
   free(f->blocks); free(f);
   A->Store = NULL;
}
