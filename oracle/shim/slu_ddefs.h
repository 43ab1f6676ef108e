/*
 * Test-infrastructure shim (oracle only): the subset of the SuperLU API that
 * the reference preconditioner calls (Preconditioner.c:16,169-173,201-304).
 * SuperLU is absent from this image; the reference build files name only a
 * local library file (-lsuperlu_5.2.2 in make-ubuntu.inc), no vendored copy.
 *
 * The shim factors the assembled sparse matrix exactly: it splits the matrix
 * into connected components of its sparsity graph and computes a dense LU with
 * partial pivoting of each component (for the FFTSVD PBE operator every
 * component is one 2x2 panel block, SurfaceOperator.c:183-193).  Solving with
 * the factors gives the same vector as any exact LU of the same matrix, up to
 * rounding.  Never linked into the product.
 */
#ifndef FFTSVD_ORACLE_SLU_DDEFS_SHIM_H
#define FFTSVD_ORACLE_SLU_DDEFS_SHIM_H

#ifndef TRUE
#define TRUE 1
#endif
#ifndef FALSE
#define FALSE 0
#endif

typedef enum { SLU_NC, SLU_NCP, SLU_NR, SLU_SC, SLU_SCP, SLU_SR, SLU_DN, SLU_NR_loc } Stype_t;
typedef enum { SLU_S, SLU_D, SLU_C, SLU_Z } Dtype_t;
typedef enum { SLU_GE, SLU_TRLU, SLU_TRUU, SLU_TRL, SLU_TRU, SLU_SYL, SLU_SYU, SLU_HEL, SLU_HEU } Mtype_t;
typedef enum { NOTRANS, TRANS, CONJ } trans_t;

typedef struct {
   Stype_t Stype;
   Dtype_t Dtype;
   Mtype_t Mtype;
   int nrow;
   int ncol;
   void* Store;
} SuperMatrix;

typedef struct {
   int lda;
   void* nzval;
} DNformat;

typedef struct {
   int nnz;
   void* nzval;
   int* rowind;
   int* colptr;
} NCformat;

typedef struct {
   int Fact;
   double DiagPivotThresh;
} superlu_options_t;

typedef struct {
   int TinyPivots;
   int RefineSteps;
} SuperLUStat_t;

typedef struct {
   int unused;
} GlobalLU_t;

typedef struct {
   float for_lu;
   float total_needed;
} mem_usage_t;

void StatInit(SuperLUStat_t* stat);
void StatFree(SuperLUStat_t* stat);
void set_default_options(superlu_options_t* options);
int sp_ienv(int ispec);
void get_perm_c(int ispec, SuperMatrix* A, int* perm_c);
void sp_preorder(superlu_options_t* options, SuperMatrix* A, int* perm_c, int* etree, SuperMatrix* AC);
void dCreate_CompCol_Matrix(SuperMatrix* A, int m, int n, int nnz, double* nzval, int* rowind, int* colptr,
                            Stype_t stype, Dtype_t dtype, Mtype_t mtype);
void dCreate_Dense_Matrix(SuperMatrix* X, int m, int n, double* x, int ldx, Stype_t stype, Dtype_t dtype,
                          Mtype_t mtype);
void dgstrf(superlu_options_t* options, SuperMatrix* A, int relax, int panel_size, int* etree, void* work,
            int lwork, int* perm_c, int* perm_r, SuperMatrix* L, SuperMatrix* U, GlobalLU_t* Glu,
            SuperLUStat_t* stat, int* info);
void dgstrs(trans_t trans, SuperMatrix* L, SuperMatrix* U, int* perm_c, int* perm_r, SuperMatrix* B,
            SuperLUStat_t* stat, int* info);
int dQuerySpace(SuperMatrix* L, SuperMatrix* U, mem_usage_t* mem_usage);
void Destroy_SuperMatrix_Store(SuperMatrix* A);
void Destroy_CompCol_Permuted(SuperMatrix* A);
void Destroy_CompCol_Matrix(SuperMatrix* A);
void Destroy_SuperNode_Matrix(SuperMatrix* A);

#endif
