/*
 * Test-infrastructure shim (oracle only): the subset of the FFTW3 API that the
 * reference FFTSVD code calls (FFT.c:41,54,88,100,124,135), implemented as a
 * direct separable DFT in fftw_shim.c.  FFTW itself is absent from this image
 * (no version is pinned by the reference build files, make-gcc.inc).
 *
 * Semantics follow FFTW's published definition of the multi-dimensional
 * real-data DFT: r2c computes the forward transform (exponent sign -1) of a
 * row-major n0 x n1 x n2 real array and stores the n0 x n1 x (n2/2+1)
 * non-redundant half; c2r computes the unnormalised backward transform
 * (exponent sign +1) assuming Hermitian symmetry of the logical input.
 *
 * Never linked into the product; only into oracle/_ref/.
 */
#ifndef FFTSVD_ORACLE_FFTW3_SHIM_H
#define FFTSVD_ORACLE_FFTW3_SHIM_H

#include <complex.h>

#define FFTW_ESTIMATE (1U << 6)
#define FFTW_UNALIGNED (1U << 1)

typedef float _Complex fftwf_complex;
typedef double _Complex fftw_complex;

typedef struct oracle_fftw_plan_s* fftwf_plan;
typedef struct oracle_fftw_plan_s* fftw_plan;

fftwf_plan fftwf_plan_dft_r2c_3d(int n0, int n1, int n2, float* in, fftwf_complex* out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_3d(int n0, int n1, int n2, fftwf_complex* in, float* out, unsigned flags);
void fftwf_execute_dft_r2c(const fftwf_plan p, float* in, fftwf_complex* out);
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex* in, float* out);
void fftwf_destroy_plan(fftwf_plan p);

fftw_plan fftw_plan_dft_r2c_3d(int n0, int n1, int n2, double* in, fftw_complex* out, unsigned flags);
fftw_plan fftw_plan_dft_c2r_3d(int n0, int n1, int n2, fftw_complex* in, double* out, unsigned flags);
void fftw_execute_dft_r2c(const fftw_plan p, double* in, fftw_complex* out);
void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex* in, double* out);
void fftw_destroy_plan(fftw_plan p);

#endif
