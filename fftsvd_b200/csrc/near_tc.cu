// Near field of a multi-vector matvec on the fifth-generation tensor cores (sm_100a).
//
// With many right-hand sides the near-field block product of Cube_multiply_D
// (Cube.c:1730-1798) is a GEMM per leaf: for 128 right-hand sides at a time,
//
//    Y (128 x nrows) = X (128 x 2 ncols) * D^T,
//
// X holding each right-hand side's gathered {single, double} layer densities of the
// leaf's columns and D the leaf's row-major {D_single, D_double} pairs (nrows x 2 ncols,
// K-major as stored).  One CTA of four warps computes one leaf for 128 right-hand
// sides: the chunks of 32 K values of X and D are split into TF32 heads and tails
// (split_tf32) and staged in shared memory in the K-major layout of tcgen05.cuh; one
// thread issues kind::tf32 MMAs, three per K-step (head x head, head x tail, tail x head:
// FP32-level products, Ootomo and Yokota 2022); the chunk's commit arrives on an mbarrier
// that every thread waits on (bounded) before the buffers are refilled.
//
// Accumulation: a tensor-core accumulator summed over a long K loses accuracy (measured on
// the B200 at K = 300: 2.2e-6 relative against 3e-7 for a sequential FP32 sum), while one
// K-chunk of 32 accumulates at FP32 level.  The chunks are therefore dealt round-robin to
// up to kTcAccCols / nrows accumulators of 128 lanes x nrows columns in TMEM (a new chunk
// starts a fresh accumulator while there are unused ones), and the epilogue reads them
// with tcgen05.ld (thread t = right-hand side t), sums them on the CUDA cores, adds the
// jump term and writes y.
//
// The densities come from xsd_t, the joined panel values transposed to [panel][rhs]
// (transpose_xsd_kernel), so the staging loads of X are coalesced over right-hand sides.
#include <cuda_runtime.h>

#include <cstdint>

#include "operator.h"
#include "tcgen05.cuh"

namespace fftsvd {

namespace {

constexpr int kTcRhs = 128;   // right-hand sides per CTA: the MMA's M
constexpr int kTcK = 32;      // K values per staged chunk (four K-steps of 8)
constexpr int kTcAccCols = 128;  // TMEM columns of the chunk accumulators of one CTA (four CTAs per SM)
constexpr uint32_t kTcPolls = 1u << 24;  // bound of every mbarrier wait

// xsd_t[p * ld + r] = xsd[r * panels + p] for panel p < np, right-hand side r < nrhs;
// tiles of 32 x 32 through shared memory, so both sides are coalesced
__global__ void transpose_xsd_kernel(const float2* __restrict__ xsd, int64_t panels, int np, int nrhs,
                                     float2* __restrict__ xsd_t, int64_t ld) {
   __shared__ float2 tile[32][33];
   const int p0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
   const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8 threads
   for (int j = ty; j < 32; j += 8) {
      const int r = r0 + j, p = p0 + tx;
      tile[j][tx] = (r < nrhs && p < np) ? xsd[(int64_t)r * panels + p] : make_float2(0.f, 0.f);
   }
   __syncthreads();
   for (int j = ty; j < 32; j += 8) {
      const int p = p0 + j, r = r0 + tx;
      if (p < np && r < nrhs) xsd_t[(int64_t)p * ld + r] = tile[tx][j];
   }
}

// byte offset of (row, k) of a chunk operand with `rows` rows in the K-major layout
__device__ __forceinline__ uint32_t tc_off(int row, int k, int rows) {
   return (uint32_t)((k >> 3) * (2 * rows * 16) + ((k >> 2) & 1) * (rows * 16) + row * 16 + (k & 3) * 4);
}

__global__ void __launch_bounds__(kTcRhs) near_tc_kernel(
    const LeafDesc* __restrict__ leaves, const int32_t* __restrict__ rows, const int32_t* __restrict__ cols,
    const float2* __restrict__ d, const float2* __restrict__ xsd_t, int64_t ld, const int32_t* __restrict__ point_out,
    const int32_t* __restrict__ point_panel, const double* __restrict__ point_jump,
    const int32_t* __restrict__ phi_idx, const double* __restrict__ phi_scale, const double* __restrict__ x,
    double* __restrict__ y, int nrhs, int64_t ldn, int np_max, int* __restrict__ status) {
   extern __shared__ __align__(1024) char smem[];
   const int np_cap = np_max;                    // B operand rows the buffers hold
   // two stages, each: A heads, A tails (kTcRhs x kTcK), B heads, B tails (np_cap x kTcK)
   const int a_bytes = kTcRhs * kTcK * 4, b_bytes = np_cap * kTcK * 4, stage_bytes = 2 * a_bytes + 2 * b_bytes;
   int* const row_out = reinterpret_cast<int*>(smem + 2 * stage_bytes);  // per leaf row
   int* const row_jk = row_out + np_cap;
   double* const row_jump = reinterpret_cast<double*>(row_jk + np_cap);
   __shared__ __align__(8) uint64_t mbar[2];     // one per stage: its chunk's MMAs completed
   __shared__ uint32_t tslot;
   const int t = threadIdx.x, warp = t >> 5;
   const LeafDesc L = leaves[blockIdx.x];
   const int rhs = blockIdx.y * kTcRhs + t;
   const int nr = L.nrows, np = max(8, (nr + 7) & ~7), kdim = 2 * L.ncols;
   const int nchunks = (kdim + kTcK - 1) / kTcK;
   const int acc_stride = (np + 15) & ~15;                          // TMEM columns between accumulators
   const int nacc = max(1, min(nchunks, kTcAccCols / acc_stride));  // chunk accumulators
   uint32_t ncols_tmem = 32;
   while ((int)ncols_tmem < nacc * acc_stride) ncols_tmem <<= 1;
   if (warp == 0) tc::tmem_alloc(tc::smem_addr(&tslot), ncols_tmem);
   if (t == 0) {
      tc::mbar_init(tc::smem_addr(&mbar[0]), 1);
      tc::mbar_init(tc::smem_addr(&mbar[1]), 1);
   }
   for (int i = t; i < nr; i += kTcRhs) {
      const int pnt = rows[L.row_off + i];
      const int k = point_panel[pnt];
      row_out[i] = point_out[pnt];
      row_jk[i] = k;
      row_jump[i] = k >= 0 ? point_jump[pnt] : 0.0;
   }
   tc::fence_before_sync();
   __syncthreads();
   tc::fence_after_sync();
   const uint32_t tmem = tslot;
   const uint32_t idesc = tc::idesc_tf32(kTcRhs, np);
   const float2* drow = d + L.d_off;
   bool ok = true;
   int committed = -1;  // last chunk whose MMAs were committed
   // Chunk k is staged into stage k & 1 while the MMAs of chunk k - 1 run on the other stage;
   // a stage is refilled once the MMAs of the chunk two back, which read it, have completed.
   for (int chunk = 0; chunk < nchunks; chunk++) {
      const int st = chunk & 1, k0 = chunk * kTcK;
      char* const Ah = smem + st * stage_bytes;
      char* const Al = Ah + a_bytes;
      char* const Bh = Al + a_bytes;
      char* const Bl = Bh + b_bytes;
      // X chunk: thread t is right-hand side t; K value 2 c + layer of column c.  All loads
      // are issued before any split and store.
      float2 xv[kTcK / 2];
#pragma unroll
      for (int c = 0; c < kTcK / 2; c++) {
         const int col = (k0 >> 1) + c;
         xv[c] = make_float2(0.f, 0.f);
         if (rhs < nrhs && 2 * col < kdim) xv[c] = xsd_t[(int64_t)cols[L.col_off + col] * ld + rhs];
      }
      constexpr int kDPer = 4;  // D pairs per thread and pass
      float2 dv[kDPer];
      const int dcount = np * (kTcK / 2);
      if (chunk >= 2 && !tc::mbar_wait(tc::smem_addr(&mbar[st]), (uint32_t)(((chunk - 2) >> 1) & 1), kTcPolls))
         ok = false;
      tc::fence_after_sync();
      if (__syncthreads_or(!ok)) break;  // the stage is free: the MMAs that read it completed
#pragma unroll
      for (int c = 0; c < kTcK / 2; c++) {
         float h0, l0, h1, l1;
         tc::split_tf32(xv[c].x, h0, l0);
         tc::split_tf32(xv[c].y, h1, l1);
         const uint32_t o0 = tc_off(t, 2 * c, kTcRhs), o1 = tc_off(t, 2 * c + 1, kTcRhs);
         *reinterpret_cast<float*>(Ah + o0) = h0;
         *reinterpret_cast<float*>(Al + o0) = l0;
         *reinterpret_cast<float*>(Ah + o1) = h1;
         *reinterpret_cast<float*>(Al + o1) = l1;
      }
      // D chunk: np rows (rows past nr are zero) x 16 columns of pairs
      for (int i0 = t; i0 < dcount; i0 += kTcRhs * kDPer) {
#pragma unroll
         for (int q = 0; q < kDPer; q++) {
            const int i = i0 + q * kTcRhs;
            const int row = i / (kTcK / 2), col = (k0 >> 1) + i % (kTcK / 2);
            dv[q] = make_float2(0.f, 0.f);
            if (i < dcount && row < nr && 2 * col < kdim) dv[q] = drow[(int64_t)row * L.ncols + col];
         }
#pragma unroll
         for (int q = 0; q < kDPer; q++) {
            const int i = i0 + q * kTcRhs;
            if (i >= dcount) break;
            const int row = i / (kTcK / 2), c = i % (kTcK / 2);
            float h0, l0, h1, l1;
            tc::split_tf32(dv[q].x, h0, l0);
            tc::split_tf32(dv[q].y, h1, l1);
            const uint32_t o0 = tc_off(row, 2 * c, np), o1 = tc_off(row, 2 * c + 1, np);
            *reinterpret_cast<float*>(Bh + o0) = h0;
            *reinterpret_cast<float*>(Bl + o0) = l0;
            *reinterpret_cast<float*>(Bh + o1) = h1;
            *reinterpret_cast<float*>(Bl + o1) = l1;
         }
      }
      tc::fence_proxy_async();
      __syncthreads();
      if (t == 0) {
         tc::fence_after_sync();
         const uint32_t a_h = tc::smem_addr(Ah), a_l = tc::smem_addr(Al);
         const uint32_t b_h = tc::smem_addr(Bh), b_l = tc::smem_addr(Bl);
         const uint32_t acc_col = tmem + (uint32_t)((chunk % nacc) * acc_stride);
#pragma unroll
         for (int s = 0; s < kTcK / 8; s++) {
            const uint32_t ao = (uint32_t)s * (2 * kTcRhs * 16), bo = (uint32_t)s * (2 * np * 16);
            const uint64_t ah = tc::smem_desc(a_h + ao, kTcRhs * 16, 128), al = tc::smem_desc(a_l + ao, kTcRhs * 16, 128);
            const uint64_t bh = tc::smem_desc(b_h + bo, np * 16, 128), bl = tc::smem_desc(b_l + bo, np * 16, 128);
            tc::mma_tf32(acc_col, ah, bh, idesc, (chunk >= nacc || s > 0) ? 1u : 0u);
            tc::mma_tf32(acc_col, ah, bl, idesc, 1u);
            tc::mma_tf32(acc_col, al, bh, idesc, 1u);
         }
         tc::commit(tc::smem_addr(&mbar[st]));  // arrives when every MMA issued so far completed
      }
      committed = chunk;
   }
   // the last chunk's commit covers every MMA before it: the accumulator is complete
   if (ok && nchunks > 0) {
      const int last = nchunks - 1;
      if (!tc::mbar_wait(tc::smem_addr(&mbar[last & 1]), (uint32_t)((last >> 1) & 1), kTcPolls)) ok = false;
      tc::fence_after_sync();
      if (__syncthreads_or(!ok)) ok = false;
   }
   if (!ok) {
      if (t == 0) atomicExch(status, 1);
      // one more bounded wait for the MMAs still in flight before the TMEM is released
      if (committed >= 0)
         tc::mbar_wait(tc::smem_addr(&mbar[committed & 1]), (uint32_t)((committed >> 1) & 1), kTcPolls);
   } else {
      // every lane takes part in the warp-wide TMEM loads; lanes past nrhs only skip the stores
      const double* xr = x + (int64_t)rhs * ldn;
      double* yr = y + (int64_t)rhs * ldn;
      const int used = min(nacc, nchunks);  // accumulators that hold a chunk
      for (int c0 = 0; c0 < np; c0 += 8) {
         float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
         for (int a = 0; a < used; a++) {
            float part[8];
            tc::tmem_ld8(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(a * acc_stride + c0), part);
#pragma unroll
            for (int j = 0; j < 8; j++) acc[j] += part[j];
         }
         if (rhs < nrhs) {
#pragma unroll
            for (int j = 0; j < 8; j++) {
               const int i = c0 + j;
               if (i < nr) {
                  double v = (double)acc[j];
                  const int k = row_jk[i];
                  if (k >= 0) v += row_jump[i] * (phi_scale[k] * xr[phi_idx[k]]);
                  yr[row_out[i]] = v;
               }
            }
         }
      }
   }
   tc::fence_before_sync();
   __syncthreads();
   if (warp == 0) tc::tmem_free(tmem, ncols_tmem);
}

// A wait that must give up: an mbarrier expecting one arrival that never comes, polled at
// most `polls` times.  Sets *status to 1 when the wait gave up, 2 when it (wrongly) completed.
__global__ void bounded_wait_selftest_kernel(uint32_t polls, int* __restrict__ status) {
   __shared__ __align__(8) uint64_t bar;
   if (threadIdx.x == 0) tc::mbar_init(tc::smem_addr(&bar), 1);
   __syncthreads();
   const bool done = tc::mbar_wait(tc::smem_addr(&bar), 0u, polls);
   if (__syncthreads_or(!done)) {
      if (threadIdx.x == 0) *status = 1;
   } else if (threadIdx.x == 0) {
      *status = 2;
   }
}

}  // namespace

int bounded_wait_selftest(int polls) {
   DevBuf<int> status(1);
   status.zero();
   bounded_wait_selftest_kernel<<<1, 32>>>((uint32_t)polls, status.get());
   FFTSVD_CHECK_LAUNCH();
   int v = 0;
   FFTSVD_CUDA(cudaMemcpy(&v, status.get(), sizeof(int), cudaMemcpyDeviceToHost));
   return v;
}

int near_tc_smem(int np_max) {
   return 2 * (2 * kTcRhs * kTcK * 4 + 2 * np_max * kTcK * 4) + np_max * (4 + 4 + 8);
}

void launch_near_tc(const LeafDesc* leaves, int n_leaf, const int32_t* rows, const int32_t* cols, const float2* d,
                    const float2* xsd, int64_t panels, int np_panels, float2* xsd_t, int64_t ld,
                    const int32_t* point_out, const int32_t* point_panel, const double* point_jump,
                    const int32_t* phi_idx, const double* phi_scale, const double* x, double* y, int nrhs, int64_t ldn,
                    int np_max, int* status, cudaStream_t stream) {
   {
      const dim3 grid((np_panels + 31) / 32, (nrhs + 31) / 32);
      transpose_xsd_kernel<<<grid, 256, 0, stream>>>(xsd, panels, np_panels, nrhs, xsd_t, ld);
      FFTSVD_CHECK_LAUNCH();
   }
   const int smem = near_tc_smem(np_max);
   const dim3 grid(n_leaf, (nrhs + kTcRhs - 1) / kTcRhs);
   near_tc_kernel<<<grid, kTcRhs, smem, stream>>>(leaves, rows, cols, d, xsd_t, ld, point_out, point_panel, point_jump,
                                                 phi_idx, phi_scale, x, y, nrhs, ldn, np_max, status);
   FFTSVD_CHECK_LAUNCH();
}

void prepare_near_tc(int np_max) {
   FFTSVD_CUDA(cudaFuncSetAttribute(near_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, near_tc_smem(np_max)));
}

}  // namespace fftsvd
