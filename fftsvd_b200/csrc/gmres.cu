// GMRES vector kernels (FP64).  The reference orthogonalises with modified
// Gram-Schmidt, one dot and one axpy per basis vector (GMRES.c:485-488); here
// each Arnoldi step uses classical Gram-Schmidt applied twice (two passes of
// one multi-dot and one multi-axpy over the whole basis), which is as stable as
// MGS and turns 2(i+1) dependent vector sweeps into four.  The multi-dot runs one
// block per (4096-row chunk, basis vector); updates four rows per thread.  Each thread
// issues all its loads of a chunk (or of four basis vectors) before it multiplies, so
// the sweeps are not bound by the latency of one load at a time.  All
// reductions are two-stage with a fixed order, so results are bitwise
// reproducible run to run.
#include <cmath>

#include "gmres.cuh"

namespace fftsvd {

__device__ inline double warp_sum_d(double v) {
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
   return v;
}

__global__ void precond_kernel(int nblocks, const int32_t* __restrict__ blk_ptr, const int32_t* __restrict__ blk_idx,
                               const int64_t* __restrict__ inv_off, const double* __restrict__ inv,
                               const double* __restrict__ r, double* __restrict__ z, int64_t col) {
   r += blockIdx.z * col;
   z += blockIdx.z * col;
   for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nblocks; b += gridDim.x * blockDim.x) {
      const int p0 = blk_ptr[b], k = blk_ptr[b + 1] - p0;
      double in[8], out[8];
      for (int i = 0; i < k; i++) in[i] = r[blk_idx[p0 + i]];
      const double* M = inv + inv_off[b];
      for (int i = 0; i < k; i++) {
         double s = 0.0;
         for (int j = 0; j < k; j++) s += M[i * k + j] * in[j];
         out[i] = s;
      }
      for (int i = 0; i < k; i++) z[blk_idx[p0 + i]] = out[i];
   }
}

// Sum of v over the block's threads, in a fixed order; valid in thread 0.
__device__ inline double block_sum(double v, double* red /* [kVecThreads / 32] */) {
   v = warp_sum_d(v);
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   if (lane == 0) red[warp] = v;
   __syncthreads();
   double s = 0.0;
   if (threadIdx.x == 0)
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
   return s;
}

__global__ void __launch_bounds__(kVecThreads) dots_partial_kernel(int64_t n, int nvec, const double* __restrict__ V,
                                                                   int64_t ldv, const double* __restrict__ w,
                                                                   double* __restrict__ partial, int64_t col,
                                                                   int64_t pcol) {
   __shared__ double red[kVecThreads / 32];
   const int j = blockIdx.y;
   V += blockIdx.z * col + (int64_t)j * ldv;
   w += blockIdx.z * col;
   partial += blockIdx.z * pcol;
   // a thread's kDotChunk / kVecThreads rows (k0 + t + kVecThreads i) are all loaded before
   // any is multiplied, so each thread has 2 R loads in flight instead of two
   constexpr int R = kDotChunk / kVecThreads;
   const int64_t k0 = (int64_t)blockIdx.x * kDotChunk + threadIdx.x;
   double a[R], b[R];
   if ((int64_t)(blockIdx.x + 1) * kDotChunk <= n) {  // a whole chunk: no row test
#pragma unroll
      for (int i = 0; i < R; i++) {
         a[i] = __ldg(V + k0 + (int64_t)i * kVecThreads);
         b[i] = __ldg(w + k0 + (int64_t)i * kVecThreads);
      }
   } else {
#pragma unroll
      for (int i = 0; i < R; i++) {
         const int64_t k = k0 + (int64_t)i * kVecThreads;
         a[i] = k < n ? V[k] : 0.0;
         b[i] = k < n ? w[k] : 0.0;
      }
   }
   double s4[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
   for (int i = 0; i < R; i++) s4[i & 3] = fma(a[i], b[i], s4[i & 3]);
   const double s = block_sum((s4[0] + s4[1]) + (s4[2] + s4[3]), red);
   if (threadIdx.x == 0) partial[(int64_t)j * gridDim.x + blockIdx.x] = s;
}

__global__ void reduce_partial_kernel(int nvec, int nblk, const double* __restrict__ partial, double* __restrict__ out,
                                      int accumulate, int64_t pcol, int64_t hcol) {
   __shared__ double red[32];
   partial += blockIdx.z * pcol;
   out += blockIdx.z * hcol;
   const int j = blockIdx.x;
   if (j >= nvec) return;
   double s = 0.0;
   for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += partial[(int64_t)j * nblk + b];
   s = warp_sum_d(s);
   if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
   __syncthreads();
   if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
      out[j] = accumulate ? out[j] + t : t;
   }
}

__global__ void __launch_bounds__(kVecThreads) update_kernel(int64_t n, int nvec, const double* __restrict__ V,
                                                             int64_t ldv, const double* __restrict__ partial,
                                                             int nblk, double* __restrict__ h_out,
                                                             const double* __restrict__ w, double* __restrict__ out,
                                                             double* __restrict__ norm_partial, int64_t col,
                                                             int64_t dcol, int64_t pcol, int64_t hcol) {
   extern __shared__ double hs[];  // [nvec]
   __shared__ double red[kVecThreads / 32];
   V += blockIdx.z * col;
   w += blockIdx.z * col;
   out += blockIdx.z * col;
   partial += blockIdx.z * dcol;
   // coefficients: h[j] = sum of the nblk chunk partials of dot j, one warp per j, fixed order
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
   for (int j = warp; j < nvec; j += nwarps) {
      double s = 0.0;
      for (int b = lane; b < nblk; b += 32) s += partial[(int64_t)j * nblk + b];
      s = warp_sum_d(s);
      if (lane == 0) {
         hs[j] = s;
         if (blockIdx.x == 0) h_out[blockIdx.z * hcol + j] = s;
      }
   }
   __syncthreads();
   // kRowsPerThread rows per thread, kVecThreads apart (coalesced); kUpdateGroup basis vectors
   // at a time, so each thread has kUpdateGroup kRowsPerThread loads in flight
   constexpr int RT = kRowsPerThread, G = kUpdateGroup;
   const int64_t k0 = (int64_t)blockIdx.x * kRowsPerBlock + threadIdx.x;
   double x[RT];
#pragma unroll
   for (int r = 0; r < RT; r++) {
      const int64_t k = k0 + (int64_t)r * kVecThreads;
      x[r] = k < n ? w[k] : 0.0;
   }
   const bool whole = (int64_t)(blockIdx.x + 1) * kRowsPerBlock <= n;  // no row test needed
   int j = 0;
   for (; j + G - 1 < nvec; j += G) {
      double a[G][RT];
      if (whole) {
#pragma unroll
         for (int q = 0; q < G; q++)
#pragma unroll
            for (int r = 0; r < RT; r++) a[q][r] = __ldg(V + (int64_t)(j + q) * ldv + k0 + (int64_t)r * kVecThreads);
      } else {
#pragma unroll
         for (int q = 0; q < G; q++)
#pragma unroll
            for (int r = 0; r < RT; r++) {
               const int64_t k = k0 + (int64_t)r * kVecThreads;
               a[q][r] = k < n ? V[(int64_t)(j + q) * ldv + k] : 0.0;
            }
      }
#pragma unroll
      for (int q = 0; q < G; q++)
#pragma unroll
         for (int r = 0; r < RT; r++) x[r] -= a[q][r] * hs[j + q];
   }
   for (; j < nvec; j++)
#pragma unroll
      for (int r = 0; r < RT; r++) {
         const int64_t k = k0 + (int64_t)r * kVecThreads;
         if (k < n) x[r] -= V[(int64_t)j * ldv + k] * hs[j];
      }
   double ss = 0.0;
#pragma unroll
   for (int r = 0; r < RT; r++) {
      const int64_t k = k0 + (int64_t)r * kVecThreads;
      if (k < n) {
         out[k] = x[r];
         ss = fma(x[r], x[r], ss);
      }
   }
   if (norm_partial) {
      const double s = block_sum(ss, red);
      if (threadIdx.x == 0) norm_partial[blockIdx.z * pcol + blockIdx.x] = s;
   }
}

__global__ void __launch_bounds__(kVecThreads) norm_partial_kernel(int64_t n, const double* __restrict__ w,
                                                                   double* __restrict__ partial, int64_t col,
                                                                   int64_t pcol) {
   __shared__ double red[kVecThreads / 32];
   w += blockIdx.z * col;
   partial += blockIdx.z * pcol;
   const int64_t k0 = (int64_t)blockIdx.x * kRowsPerBlock + threadIdx.x;
   double ss = 0.0;
#pragma unroll
   for (int r = 0; r < kRowsPerThread; r++) {
      const int64_t k = k0 + (int64_t)r * kVecThreads;
      const double x = k < n ? w[k] : 0.0;
      ss = fma(x, x, ss);
   }
   const double s = block_sum(ss, red);
   if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__device__ inline void rotate(double c, double s, double* a, double* b) {  // GMRES.c:17-22
   const double a1 = *a, b1 = *b;
   *a = a1 * c - b1 * s;
   *b = c * b1 + s * a1;
}

__global__ void givens_kernel(int i, int ldh, double* __restrict__ H, const double* __restrict__ h1,
                              const double* __restrict__ h2, const double* __restrict__ norm_partial, int nblk,
                              double* __restrict__ cs, double* __restrict__ sn, double* __restrict__ g,
                              GivensState* __restrict__ st, int64_t hcol, int64_t pcol,
                              const int32_t* __restrict__ active, double2* __restrict__ hist) {
   extern __shared__ double gsh[];  // the new column (i + 2), then the previous rotations cs[i], sn[i]
   __shared__ double red[256];
   // column blockIdx.x of a batch: its own Hessenberg (ldh x ldh), rotations, g and state
   const int colx = blockIdx.x;
   H += (int64_t)colx * ldh * ldh;
   h1 += colx * hcol;
   h2 += colx * hcol;
   norm_partial += colx * pcol;
   cs += (int64_t)colx * ldh;
   sn += (int64_t)colx * ldh;
   g += (int64_t)colx * ldh;
   st += colx;
   if (active && !active[colx]) {  // finished column: its next basis vectors become zero
      if (threadIdx.x == 0) st->inv_beta = 0.0;
      return;
   }
   double* colv = gsh;
   double* css = gsh + i + 2;
   double* sns = css + i;
   double s = 0.0;
   for (int b = threadIdx.x; b < nblk; b += blockDim.x) s += norm_partial[b];
   red[threadIdx.x] = s;
   // the column and the rotations are loaded in parallel; the rotations then run in shared memory
   bool bad = false;
   for (int j = threadIdx.x; j <= i; j += blockDim.x) {
      colv[j] = h1[j] + h2[j];
      bad = bad || !isfinite(colv[j]);
   }
   for (int k = threadIdx.x; k < i; k += blockDim.x) {
      css[k] = cs[k];
      sns[k] = sn[k];
   }
   const int any_bad = __syncthreads_or(bad);
   for (int w = blockDim.x / 2; w > 0; w >>= 1) {
      if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
   }
   if (threadIdx.x == 0) {
      const double beta = sqrt(red[0]);
      const bool finite = isfinite(beta) && !any_bad;
      colv[i + 1] = beta;
      for (int k = 0; k < i; k++) rotate(css[k], sns[k], &colv[k], &colv[k + 1]);
      // GMRES.c:3-15
      double c, sv;
      if (colv[i + 1] == 0.0) {
         c = 1.0;
         sv = 0.0;
      } else {
         const double r1 = fabs(colv[i]), r2 = fabs(colv[i + 1]);
         const double len = sqrt(r1 * r1 + r2 * r2);
         c = colv[i] / len;
         sv = -colv[i + 1] / len;
      }
      cs[i] = c;
      sn[i] = sv;
      rotate(c, sv, &colv[i], &colv[i + 1]);
      g[i + 1] = 0.0;
      rotate(c, sv, &g[i], &g[i + 1]);
      st->residual = fabs(g[i + 1]) / st->normr;
      st->inv_beta = beta > 0.0 ? 1.0 / beta : 0.0;
      st->flag = !finite ? 2 : (beta == 0.0 ? 1 : 0);
      if (hist) hist[i] = make_double2(st->residual, (double)st->flag);
   }
   __syncthreads();
   double* colh = H + (int64_t)i * ldh;
   for (int j = threadIdx.x; j <= i + 1; j += blockDim.x) colh[j] = colv[j];
}

__global__ void scale_kernel(int64_t n, const double* __restrict__ src, const double* __restrict__ factor_ptr,
                             double factor, double* __restrict__ dst, int64_t col, int64_t fcol,
                             double* __restrict__ dst2) {
   src += blockIdx.z * col;
   dst += blockIdx.z * col;
   const double f = factor_ptr ? factor_ptr[blockIdx.z * fcol] : factor;
   for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
      const double v = src[k] * f;
      dst[k] = v;
      if (dst2) dst2[k] = v;
   }
}

__global__ void combine_kernel(int64_t n, int nvec, const double* __restrict__ V, int64_t ldv,
                               const double* __restrict__ y, double* __restrict__ x, int64_t col, int64_t ycol) {
   extern __shared__ double ys[];
   V += blockIdx.z * col;
   x += blockIdx.z * col;
   y += blockIdx.z * ycol;
   for (int j = threadIdx.x; j < nvec; j += blockDim.x) ys[j] = y[j];
   __syncthreads();
   for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
      double s = x[k];
      for (int j = 0; j < nvec; j++) s += V[(int64_t)j * ldv + k] * ys[j];
      x[k] = s;
   }
}

__global__ void sub_kernel(int64_t n, const double* __restrict__ a, const double* __restrict__ b,
                           double* __restrict__ dst, int64_t col) {
   a += blockIdx.z * col;
   b += blockIdx.z * col;
   dst += blockIdx.z * col;
   for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
      dst[k] = a[k] - b[k];
}

__global__ void add_kernel(int64_t n, const double* __restrict__ a, double* __restrict__ dst, int64_t col) {
   a += blockIdx.z * col;
   dst += blockIdx.z * col;
   for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
      dst[k] += a[k];
}

}  // namespace fftsvd
