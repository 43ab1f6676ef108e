/*
 * Test-infrastructure shim (oracle only): 3-D real-data DFTs with FFTW3's
 * calling convention, for the small odd sizes (7..19) that FFTSVD's grid
 * convolution uses (FFT.c:10-150).  Implemented as separable direct DFTs,
 * accumulated in double precision; the float entry points round once at the
 * end.  See fftw3.h for the transform definitions.
 *
 * A plan holds the twiddle factors of its three lengths as full n x n tables
 * (entry a * n + k is exp(-2 pi i a k / n)), so an execution does no
 * trigonometry, no index reduction and no allocation: its work arrays are
 * per-thread buffers that grow to the largest plan a thread has executed (the
 * reference executes one static plan from several OpenMP threads at once,
 * FFT.c:49-55, Tree.c:630-656).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "fftw3.h"

struct oracle_fftw_plan_s {
   int n0, n1, n2;
   double *c0, *s0, *c1, *s1, *c2, *s2; /* n x n tables of cos and sin of 2 pi a k / n */
};

static void table(int n, double** c, double** s) {
   int a, k;
   *c = (double*)malloc(sizeof(double) * n * n);
   *s = (double*)malloc(sizeof(double) * n * n);
   for (a = 0; a < n; a++)
      for (k = 0; k < n; k++) {
         const double ang = 2.0 * M_PI * (double)((long)a * k % n) / (double)n;
         (*c)[a * n + k] = cos(ang);
         (*s)[a * n + k] = sin(ang);
      }
}

static struct oracle_fftw_plan_s* make_plan(int n0, int n1, int n2) {
   struct oracle_fftw_plan_s* p = (struct oracle_fftw_plan_s*)malloc(sizeof(*p));
   p->n0 = n0; p->n1 = n1; p->n2 = n2;
   table(n0, &p->c0, &p->s0);
   table(n1, &p->c1, &p->s1);
   table(n2, &p->c2, &p->s2);
   return p;
}

static void free_plan(struct oracle_fftw_plan_s* p) {
   if (!p) return;
   free(p->c0); free(p->s0); free(p->c1); free(p->s1); free(p->c2); free(p->s2);
   free(p);
}

/* per-thread work arrays: two complex half-spectra and one real grid */
static __thread double _Complex *w_t1 = NULL, *w_t2 = NULL, *w_cx = NULL;
static __thread double* w_re = NULL;
static __thread size_t w_cap_c = 0, w_cap_r = 0;

static void work(size_t nc, size_t nr) {
   if (nc > w_cap_c) {
      free(w_t1); free(w_t2); free(w_cx);
      w_t1 = (double _Complex*)malloc(sizeof(double _Complex) * nc);
      w_t2 = (double _Complex*)malloc(sizeof(double _Complex) * nc);
      w_cx = (double _Complex*)malloc(sizeof(double _Complex) * nc);
      w_cap_c = nc;
   }
   if (nr > w_cap_r) {
      free(w_re);
      w_re = (double*)malloc(sizeof(double) * nr);
      w_cap_r = nr;
   }
}

/* Forward r2c in double.  in: n0*n1*n2 reals, out: n0*n1*h complex (h=n2/2+1). */
static void r2c_double(const struct oracle_fftw_plan_s* p, const double* in, double _Complex* out) {
   const int n0 = p->n0, n1 = p->n1, n2 = p->n2, h = n2 / 2 + 1;
   int i, j, k, a, b;
   double _Complex *t1 = w_t1, *t2 = w_t2;
   /* last dimension: real -> half complex, exponent -1 */
   for (i = 0; i < n0; i++)
      for (j = 0; j < n1; j++) {
         const double* line = in + (i * n1 + j) * n2;
         for (b = 0; b < h; b++) {
            const double *cb = p->c2 + b * n2, *sb = p->s2 + b * n2;
            double re = 0.0, im = 0.0;
            for (k = 0; k < n2; k++) {
               re += line[k] * cb[k];
               im -= line[k] * sb[k];
            }
            t1[(i * n1 + j) * h + b] = re + I * im;
         }
      }
   /* middle dimension */
   for (i = 0; i < n0; i++)
      for (a = 0; a < n1; a++) {
         const double *ca = p->c1 + a * n1, *sa = p->s1 + a * n1;
         for (b = 0; b < h; b++) {
            double _Complex acc = 0.0;
            for (j = 0; j < n1; j++) acc += t1[(i * n1 + j) * h + b] * (ca[j] - I * sa[j]);
            t2[(i * n1 + a) * h + b] = acc;
         }
      }
   /* first dimension */
   for (a = 0; a < n0; a++) {
      const double *ca = p->c0 + a * n0, *sa = p->s0 + a * n0;
      for (j = 0; j < n1; j++)
         for (b = 0; b < h; b++) {
            double _Complex acc = 0.0;
            for (i = 0; i < n0; i++) acc += t2[(i * n1 + j) * h + b] * (ca[i] - I * sa[i]);
            out[(a * n1 + j) * h + b] = acc;
         }
   }
}

/* Backward c2r in double, unnormalised.  in: n0*n1*h complex, out: n0*n1*n2 reals. */
static void c2r_double(const struct oracle_fftw_plan_s* p, const double _Complex* in, double* out) {
   const int n0 = p->n0, n1 = p->n1, n2 = p->n2, h = n2 / 2 + 1;
   int i, j, k, a, b;
   double _Complex *t1 = w_t1, *t2 = w_t2;
   /* first dimension, exponent +1 */
   for (i = 0; i < n0; i++) {
      const double *ci = p->c0 + i * n0, *si = p->s0 + i * n0;
      for (j = 0; j < n1; j++)
         for (b = 0; b < h; b++) {
            double _Complex acc = 0.0;
            for (a = 0; a < n0; a++) acc += in[(a * n1 + j) * h + b] * (ci[a] + I * si[a]);
            t1[(i * n1 + j) * h + b] = acc;
         }
   }
   /* middle dimension */
   for (i = 0; i < n0; i++)
      for (j = 0; j < n1; j++) {
         const double *cj = p->c1 + j * n1, *sj = p->s1 + j * n1;
         for (b = 0; b < h; b++) {
            double _Complex acc = 0.0;
            for (a = 0; a < n1; a++) acc += t1[(i * n1 + a) * h + b] * (cj[a] + I * sj[a]);
            t2[(i * n1 + j) * h + b] = acc;
         }
      }
   /* last dimension: Hermitian half -> real */
   for (i = 0; i < n0; i++)
      for (j = 0; j < n1; j++) {
         const double _Complex* row = &t2[(i * n1 + j) * h];
         for (k = 0; k < n2; k++) {
            const double *ck = p->c2 + k * n2, *sk = p->s2 + k * n2;
            double acc = creal(row[0]);
            for (b = 1; b < h; b++) {
               const double term = creal(row[b]) * ck[b] - cimag(row[b]) * sk[b];
               if ((n2 % 2 == 0) && (b == n2 / 2))
                  acc += term;
               else
                  acc += 2.0 * term;
            }
            out[(i * n1 + j) * n2 + k] = acc;
         }
      }
}

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out, unsigned flags) {
   (void)in; (void)out; (void)flags;
   return make_plan(n0, n1, n2);
}
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out, unsigned flags) {
   (void)in; (void)out; (void)flags;
   return make_plan(n0, n1, n2);
}
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out) {
   work((size_t)p->n0 * p->n1 * (p->n2 / 2 + 1), 0);
   r2c_double(p, in, out);
}
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out) {
   work((size_t)p->n0 * p->n1 * (p->n2 / 2 + 1), 0);
   c2r_double(p, in, out);
}
void fftw_destroy_plan(fftw_plan p) { free_plan(p); }

fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float* in, fftwf_complex* out, unsigned flags) {
   (void)in; (void)out; (void)flags;
   return make_plan(n0, n1, n2);
}
fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex* in, float* out, unsigned flags) {
   (void)in; (void)out; (void)flags;
   return make_plan(n0, n1, n2);
}
void fftwf_execute_dft_r2c(const fftwf_plan p, float* in, fftwf_complex* out) {
   const int n = p->n0 * p->n1 * p->n2, nh = p->n0 * p->n1 * (p->n2 / 2 + 1);
   int i;
   work((size_t)nh, (size_t)n);
   for (i = 0; i < n; i++) w_re[i] = in[i];
   r2c_double(p, w_re, w_cx);
   for (i = 0; i < nh; i++) out[i] = (float)creal(w_cx[i]) + I * (float)cimag(w_cx[i]);
}
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex* in, float* out) {
   const int n = p->n0 * p->n1 * p->n2, nh = p->n0 * p->n1 * (p->n2 / 2 + 1);
   int i;
   work((size_t)nh, (size_t)n);
   for (i = 0; i < nh; i++) w_cx[i] = crealf(in[i]) + I * cimagf(in[i]);
   c2r_double(p, w_cx, w_re);
   for (i = 0; i < n; i++) out[i] = (float)w_re[i];
}
void fftwf_destroy_plan(fftwf_plan p) { free_plan(p); }
