/*
 * Test-infrastructure shim (oracle only): the LAPACK routines the reference
 * FFTSVD path calls, written from their mathematical definitions.
 *
 *   dgesvd_  (Matrix.c:493, used by Matrix_pseudoinverse for the equivalent
 *             density fitting operators, Tree.c:357): full SVD, singular values
 *             in descending order, computed by one-sided (Hestenes) Jacobi.
 *   dsyev_   (QuadratureRule.c:97, Golub-Welsch Gauss-Legendre nodes): symmetric
 *             eigen-decomposition, eigenvalues ascending, by cyclic Jacobi.
 *
 * The other LAPACK entry points referenced by the compiled reference objects
 * are not reached on the PBE path; they abort loudly if they ever are.
 * LAPACK is absent from this image and unpinned by the reference build files.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* One-sided Jacobi on B (p x q, column-major, p >= q).  On exit the columns of
   B are mutually orthogonal (B = W), and V (q x q, column-major) holds the
   accumulated rotations with B_in * V = W. */
static void hestenes(int p, int q, double* B, double* V) {
   int i, j, k, sweep;
   for (i = 0; i < q * q; i++) V[i] = 0.0;
   for (i = 0; i < q; i++) V[i * q + i] = 1.0;
   for (sweep = 0; sweep < 80; sweep++) {
      double off = 0.0;
      for (j = 0; j < q - 1; j++)
         for (k = j + 1; k < q; k++) {
            double a = 0.0, b = 0.0, g = 0.0;
            double *bj = B + (size_t)j * p, *bk = B + (size_t)k * p;
            for (i = 0; i < p; i++) { a += bj[i] * bj[i]; b += bk[i] * bk[i]; g += bj[i] * bk[i]; }
            if (g == 0.0 || fabs(g) <= 1e-300) continue;
            {
               double rel = fabs(g) / sqrt(a * b);
               if (rel > off) off = rel;
               if (rel < 1e-17) continue;
            }
            {
               double zeta = (b - a) / (2.0 * g);
               double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
               double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
               double *vj = V + (size_t)j * q, *vk = V + (size_t)k * q;
               for (i = 0; i < p; i++) {
                  double x = bj[i], y = bk[i];
                  bj[i] = c * x - s * y;
                  bk[i] = s * x + c * y;
               }
               for (i = 0; i < q; i++) {
                  double x = vj[i], y = vk[i];
                  vj[i] = c * x - s * y;
                  vk[i] = s * x + c * y;
               }
            }
         }
      if (off < 1e-16) break;
   }
}

/* A = U diag(S) VT for A (m x n, column-major, lda).  JOBU = JOBVT = 'A'. */
void dgesvd_(char* jobu, char* jobvt, unsigned int* M, unsigned int* N, double* A, unsigned int* LDA,
             double* S, double* U, unsigned int* LDU, double* VT, unsigned int* LDVT, double* work,
             unsigned int* lwork, int* info) {
   int m = (int)*M, n = (int)*N, lda = (int)*LDA, ldu = (int)*LDU, ldvt = (int)*LDVT;
   int transposed = (m < n);
   int p = transposed ? n : m, q = transposed ? m : n;
   int i, j;
   double* B = (double*)malloc(sizeof(double) * (size_t)p * q);
   double* V = (double*)malloc(sizeof(double) * (size_t)q * q);
   double* sig = (double*)malloc(sizeof(double) * q);
   int* order = (int*)malloc(sizeof(int) * q);
   double* Ufull = (double*)calloc((size_t)p * p, sizeof(double)); /* left vectors of B, p x p */
   (void)jobu; (void)jobvt; (void)work; (void)lwork;

   for (j = 0; j < q; j++)
      for (i = 0; i < p; i++)
         B[(size_t)j * p + i] = transposed ? A[(size_t)i * lda + j] : A[(size_t)j * lda + i];
   hestenes(p, q, B, V);
   for (j = 0; j < q; j++) {
      double s = 0.0;
      for (i = 0; i < p; i++) s += B[(size_t)j * p + i] * B[(size_t)j * p + i];
      sig[j] = sqrt(s);
      order[j] = j;
   }
   for (i = 0; i < q; i++)             /* sort descending */
      for (j = i + 1; j < q; j++)
         if (sig[order[j]] > sig[order[i]]) { int t = order[i]; order[i] = order[j]; order[j] = t; }
   for (j = 0; j < q; j++) {
      int src = order[j];
      S[j] = sig[src];
      for (i = 0; i < p; i++)
         Ufull[(size_t)j * p + i] = sig[src] > 0.0 ? B[(size_t)src * p + i] / sig[src] : 0.0;
   }
   /* B = Ufull(:, :q) diag(S) V(:, order)^T.  Columns q..p-1 of Ufull stay zero:
      they only multiply zero singular values in every caller on this path. */
   if (!transposed) {
      for (j = 0; j < m; j++)
         for (i = 0; i < m; i++) U[(size_t)j * ldu + i] = Ufull[(size_t)j * p + i];
      for (j = 0; j < n; j++)           /* VT(r, c) = V(c, order[r]) */
         for (i = 0; i < n; i++) VT[(size_t)j * ldvt + i] = V[(size_t)order[i] * q + j];
   } else {
      /* A = B^T = V diag(S) Ufull^T: left vectors of A are V(:, order), right are Ufull */
      for (j = 0; j < m; j++)
         for (i = 0; i < m; i++) U[(size_t)j * ldu + i] = V[(size_t)order[j] * q + i];
      for (j = 0; j < n; j++)           /* VT(r, c) = Ufull(c, r) */
         for (i = 0; i < n; i++) VT[(size_t)j * ldvt + i] = Ufull[(size_t)i * p + j];
   }
   *info = 0;
   free(B); free(V); free(sig); free(order); free(Ufull);
}

/* Symmetric eigen-decomposition, upper triangle given, column-major. */
void dsyev_(char* jobz, char* uplo, unsigned int* Np, double* A, unsigned int* LDA, double* W, double* work,
            unsigned int* lwork, int* info) {
   int n = (int)*Np, lda = (int)*LDA, i, j, k, sweep;
   double* a = (double*)malloc(sizeof(double) * n * n);
   double* v = (double*)calloc((size_t)n * n, sizeof(double));
   int* order = (int*)malloc(sizeof(int) * n);
   (void)jobz; (void)uplo; (void)work; (void)lwork;
   for (j = 0; j < n; j++)
      for (i = 0; i <= j; i++) {
         a[i * n + j] = A[(size_t)j * lda + i];
         a[j * n + i] = A[(size_t)j * lda + i];
      }
   for (i = 0; i < n; i++) v[i * n + i] = 1.0;
   for (sweep = 0; sweep < 100; sweep++) {
      double off = 0.0;
      for (i = 0; i < n; i++)
         for (j = i + 1; j < n; j++) off += a[i * n + j] * a[i * n + j];
      if (off < 1e-300) break;
      for (i = 0; i < n - 1; i++)
         for (j = i + 1; j < n; j++) {
            double apq = a[i * n + j];
            if (fabs(apq) < 1e-300) continue;
            {
               double theta = (a[j * n + j] - a[i * n + i]) / (2.0 * apq);
               double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
               double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
               for (k = 0; k < n; k++) {   /* columns */
                  double x = a[k * n + i], y = a[k * n + j];
                  a[k * n + i] = c * x - s * y;
                  a[k * n + j] = s * x + c * y;
               }
               for (k = 0; k < n; k++) {   /* rows */
                  double x = a[i * n + k], y = a[j * n + k];
                  a[i * n + k] = c * x - s * y;
                  a[j * n + k] = s * x + c * y;
               }
               for (k = 0; k < n; k++) {
                  double x = v[k * n + i], y = v[k * n + j];
                  v[k * n + i] = c * x - s * y;
                  v[k * n + j] = s * x + c * y;
               }
            }
         }
   }
   for (i = 0; i < n; i++) order[i] = i;
   for (i = 0; i < n; i++)
      for (j = i + 1; j < n; j++)
         if (a[order[j] * n + order[j]] < a[order[i] * n + order[i]]) { int t = order[i]; order[i] = order[j]; order[j] = t; }
   for (j = 0; j < n; j++) {
      W[j] = a[order[j] * n + order[j]];
      for (i = 0; i < n; i++) A[(size_t)j * lda + i] = v[i * n + order[j]];
   }
   *info = 0;
   free(a); free(v); free(order);
}

static void unreachable(const char* name) {
   fprintf(stderr, "oracle lapack shim: %s is not on the FFTSVD PBE path and is not provided\n", name);
   abort();
}

void sgesvd_(void) { unreachable("sgesvd_"); }
void ssyev_(void) { unreachable("ssyev_"); }
void dgels_(void) { unreachable("dgels_"); }
void sgels_(void) { unreachable("sgels_"); }
void dgeqrf_(void) { unreachable("dgeqrf_"); }
void sgeqrf_(void) { unreachable("sgeqrf_"); }
void dorgqr_(void) { unreachable("dorgqr_"); }
void sorgqr_(void) { unreachable("sorgqr_"); }
void dsyevr_(void) { unreachable("dsyevr_"); }
void ssyevr_(void) { unreachable("ssyevr_"); }
