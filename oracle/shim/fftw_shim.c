/*
 * Test-infrastructure shim (oracle only): 3-D real-data DFTs with FFTW3's
 * calling convention, for the small odd sizes (7..19) that FFTSVD's grid
 * convolution uses (FFT.c:10-150).  Implemented as separable direct DFTs,
 * accumulated in double precision; the float entry points round once at the
 * end.  See fftw3.h for the transform definitions.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include "fftw3.h"

struct oracle_fftw_plan_s {
   int n0, n1, n2;
};

static struct oracle_fftw_plan_s* make_plan(int n0, int n1, int n2) {
   struct oracle_fftw_plan_s* p = (struct oracle_fftw_plan_s*)malloc(sizeof(*p));
   p->n0 = n0; p->n1 = n1; p->n2 = n2;
   return p;
}

/* cos/sin tables for exp(sign * 2 pi i * a * b / n) */
static void twiddles(int n, double* c, double* s) {
   int k;
   for (k = 0; k < n; k++) {
      double ang = 2.0 * M_PI * (double)k / (double)n;
      c[k] = cos(ang);
      s[k] = sin(ang);
   }
}

/* Forward r2c in double.  in: n0*n1*n2 reals, out: n0*n1*h complex (h=n2/2+1). */
static void r2c_double(int n0, int n1, int n2, const double* in, double _Complex* out) {
   int h = n2 / 2 + 1;
   int i, j, k, a, b;
   double *c0 = malloc(sizeof(double) * n0), *s0 = malloc(sizeof(double) * n0);
   double *c1 = malloc(sizeof(double) * n1), *s1 = malloc(sizeof(double) * n1);
   double *c2 = malloc(sizeof(double) * n2), *s2 = malloc(sizeof(double) * n2);
   double _Complex* t1 = malloc(sizeof(double _Complex) * n0 * n1 * h);
   double _Complex* t2 = malloc(sizeof(double _Complex) * n0 * n1 * h);
   twiddles(n0, c0, s0); twiddles(n1, c1, s1); twiddles(n2, c2, s2);

   /* last dimension: real -> half complex, exponent -1 */
   for (i = 0; i < n0; i++)
      for (j = 0; j < n1; j++)
         for (b = 0; b < h; b++) {
            double re = 0.0, im = 0.0;
            for (k = 0; k < n2; k++) {
               int m = (int)(((long)b * k) % n2);
               double v = in[(i * n1 + j) * n2 + k];
               re += v * c2[m];
               im -= v * s2[m];
            }
            t1[(i * n1 + j) * h + b] = re + I * im;
         }
   /* middle dimension */
   for (i = 0; i < n0; i++)
      for (a = 0; a < n1; a++)
         for (b = 0; b < h; b++) {
            double _Complex acc = 0.0;
            for (j = 0; j < n1; j++) {
               int m = (int)(((long)a * j) % n1);
               acc += t1[(i * n1 + j) * h + b] * (c1[m] - I * s1[m]);
            }
            t2[(i * n1 + a) * h + b] = acc;
         }
   /* first dimension */
   for (a = 0; a < n0; a++)
      for (j = 0; j < n1; j++)
         for (b = 0; b < h; b++) {
            double _Complex acc = 0.0;
            for (i = 0; i < n0; i++) {
               int m = (int)(((long)a * i) % n0);
               acc += t2[(i * n1 + j) * h + b] * (c0[m] - I * s0[m]);
            }
            out[(a * n1 + j) * h + b] = acc;
         }
   free(c0); free(s0); free(c1); free(s1); free(c2); free(s2); free(t1); free(t2);
}

/* Backward c2r in double, unnormalised.  in: n0*n1*h complex, out: n0*n1*n2 reals. */
static void c2r_double(int n0, int n1, int n2, const double _Complex* in, double* out) {
   int h = n2 / 2 + 1;
   int i, j, k, a, b;
   double *c0 = malloc(sizeof(double) * n0), *s0 = malloc(sizeof(double) * n0);
   double *c1 = malloc(sizeof(double) * n1), *s1 = malloc(sizeof(double) * n1);
   double *c2 = malloc(sizeof(double) * n2), *s2 = malloc(sizeof(double) * n2);
   double _Complex* t1 = malloc(sizeof(double _Complex) * n0 * n1 * h);
   double _Complex* t2 = malloc(sizeof(double _Complex) * n0 * n1 * h);
   twiddles(n0, c0, s0); twiddles(n1, c1, s1); twiddles(n2, c2, s2);

   /* first dimension, exponent +1 */
   for (i = 0; i < n0; i++)
      for (j = 0; j < n1; j++)
         for (b = 0; b < h; b++) {
            double _Complex acc = 0.0;
            for (a = 0; a < n0; a++) {
               int m = (int)(((long)a * i) % n0);
               acc += in[(a * n1 + j) * h + b] * (c0[m] + I * s0[m]);
            }
            t1[(i * n1 + j) * h + b] = acc;
         }
   /* middle dimension */
   for (i = 0; i < n0; i++)
      for (j = 0; j < n1; j++)
         for (b = 0; b < h; b++) {
            double _Complex acc = 0.0;
            for (a = 0; a < n1; a++) {
               int m = (int)(((long)a * j) % n1);
               acc += t1[(i * n1 + a) * h + b] * (c1[m] + I * s1[m]);
            }
            t2[(i * n1 + j) * h + b] = acc;
         }
   /* last dimension: Hermitian half -> real */
   for (i = 0; i < n0; i++)
      for (j = 0; j < n1; j++)
         for (k = 0; k < n2; k++) {
            const double _Complex* row = &t2[(i * n1 + j) * h];
            double acc = creal(row[0]);
            for (b = 1; b < h; b++) {
               int m = (int)(((long)b * k) % n2);
               double term = creal(row[b]) * c2[m] - cimag(row[b]) * s2[m];
               if ((n2 % 2 == 0) && (b == n2 / 2))
                  acc += term;
               else
                  acc += 2.0 * term;
            }
            out[(i * n1 + j) * n2 + k] = acc;
         }
   free(c0); free(s0); free(c1); free(s1); free(c2); free(s2); free(t1); free(t2);
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
   r2c_double(p->n0, p->n1, p->n2, in, out);
}
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out) {
   c2r_double(p->n0, p->n1, p->n2, in, out);
}
void fftw_destroy_plan(fftw_plan p) { free(p); }

fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float* in, fftwf_complex* out, unsigned flags) {
   (void)in; (void)out; (void)flags;
   return make_plan(n0, n1, n2);
}
fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex* in, float* out, unsigned flags) {
   (void)in; (void)out; (void)flags;
   return make_plan(n0, n1, n2);
}
void fftwf_execute_dft_r2c(const fftwf_plan p, float* in, fftwf_complex* out) {
   int n = p->n0 * p->n1 * p->n2, nh = p->n0 * p->n1 * (p->n2 / 2 + 1), i;
   double* din = malloc(sizeof(double) * n);
   double _Complex* dout = malloc(sizeof(double _Complex) * nh);
   for (i = 0; i < n; i++) din[i] = in[i];
   r2c_double(p->n0, p->n1, p->n2, din, dout);
   for (i = 0; i < nh; i++) out[i] = (float)creal(dout[i]) + I * (float)cimag(dout[i]);
   free(din); free(dout);
}
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex* in, float* out) {
   int n = p->n0 * p->n1 * p->n2, nh = p->n0 * p->n1 * (p->n2 / 2 + 1), i;
   double _Complex* din = malloc(sizeof(double _Complex) * nh);
   double* dout = malloc(sizeof(double) * n);
   for (i = 0; i < nh; i++) din[i] = crealf(in[i]) + I * cimagf(in[i]);
   c2r_double(p->n0, p->n1, p->n2, din, dout);
   for (i = 0; i < n; i++) out[i] = (float)dout[i];
   free(din); free(dout);
}
void fftwf_destroy_plan(fftwf_plan p) { free(p); }
