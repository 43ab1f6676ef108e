// Block GMRES least-squares update on the device (the storage is described in block_ls.h).
//
// One warp owns one column of a 2K-row window (K <= 256): lane l keeps rows q 32 + l,
// q < 16, in registers.  A reflector H = I - tau v v^T costs the warp one masked dot
// product, a shuffle reduction and one update.  The warps of a block apply the same
// reflectors to their columns, so the block copies the vectors and their scalars into
// shared memory eight at a time, the next eight while the current ones are applied (a
// warp that read each vector from global memory waited on two dependent loads per
// reflector).  The transformation of a
// block column by the earlier blocks is independent per column: one launch applies every
// earlier block to all K columns, block after block (block i's window is rows
// iK .. iK + 2K).  The 2K x K panel of the new block is factored left-looking in panels
// of 16 columns, one block of 16 warps each: a warp first applies the reflectors of the
// earlier panels to its column, then the panel's columns are reduced one after another,
// the owner warp forming the reflector (the dlarfg convention: beta = -sign(alpha)
// ||x||, tau = (beta - alpha) / beta, v = x / (alpha - beta) below the pivot) and the
// warps to its right applying it through shared memory.
#include "block_ls.h"

#include <algorithm>
#include <atomic>

#include "common.h"

namespace fftsvd {
namespace lsq {

namespace {

constexpr int kWin = 16;         // window rows per lane: 2K <= 512
constexpr int kRowsMax = 32 * kWin;
constexpr int kApplyWarps = 4;   // columns per block of apply_kernel
constexpr int kPanel = 16;       // columns per panel_kernel launch
constexpr int kChunk = 8;        // reflectors per shared-memory stage
constexpr unsigned kFull = 0xffffffffu;

// dynamic shared memory of the staged reflector application: two stages of kChunk
// vectors of L = 2K doubles rounded up to 32
size_t stage_bytes(int K) { return sizeof(double) * 2 * kChunk * (size_t)((2 * K + 31) & ~31); }

__device__ __forceinline__ double warp_sum(double s) {
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
   return s;
}

// x <- (I - tau v v^T) x on the window x for the reflector v with pivot row r: v holds
// every row of the window (zeros above r, and zeros from L up to 32 nq, where nq = the
// window's 32-row chunks), so no row needs a test; chunks of 32 rows wholly above r are
// skipped by the whole warp.
__device__ __forceinline__ void reflect(double (&x)[kWin], const double* __restrict__ v, double tau, int r, int nq,
                                        int lane) {
   const int qlo = r >> 5;
   double vv[kWin];
#pragma unroll
   for (int q = 0; q < kWin; q++) vv[q] = q >= qlo && q < nq ? v[q * 32 + lane] : 0.0;
   // four independent partial sums (rows q = 0, 4, 8, 12 | 1, 5, ... ) shorten the chain
   double p4[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
   for (int q = 0; q < kWin; q++) p4[q & 3] = fma(vv[q], x[q], p4[q & 3]);
   const double s = warp_sum((p4[0] + p4[1]) + (p4[2] + p4[3])) * tau;
#pragma unroll
   for (int q = 0; q < kWin; q++)
      if (q >= qlo && q < nq) x[q] = fma(-s, vv[q], x[q]);
}

__device__ __forceinline__ void load_window(double (&x)[kWin], const double* w, int L, int lane) {
#pragma unroll
   for (int q = 0; q < kWin; q++) {
      const int t = q * 32 + lane;
      x[q] = t < L ? w[t] : 0.0;
   }
}

__device__ __forceinline__ void store_window(const double (&x)[kWin], double* w, int L, int lane) {
#pragma unroll
   for (int q = 0; q < kWin; q++) {
      const int t = q * 32 + lane;
      if (t < L) w[t] = x[q];
   }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
   const unsigned d = (unsigned)__cvta_generic_to_shared(smem);
   asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
   asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Reflectors rb .. re-1 of one block (vectors V + r L, scalars tau) applied in order to the
// window x of every warp with `active` set.  All threads of the block copy the vectors into
// shared memory, kChunk at a time through two stages (the next stage is copied while the
// current one is applied), together with their scalars.  A staged vector has L32 = 32 nq
// rows: the L rows of V (zeros above the pivot included) and zeros after them.  Every
// thread of the block must call this with the same arguments but `active` and x.
// sv: 2 kChunk L32 doubles, st: 2 kChunk doubles.
__device__ __forceinline__ void apply_staged(double (&x)[kWin], bool active, const double* __restrict__ V,
                                             const double* __restrict__ tau, int rb, int re, int L, int lane,
                                             double* sv, double* st) {
   const int L32 = (L + 31) & ~31, nq = L32 >> 5;
   const int nchunks = (re - rb + kChunk - 1) / kChunk;
   // the rows from L to L32 of every slot: zero (the copies below never write them)
   for (int i = threadIdx.x; i < 2 * kChunk * (L32 - L); i += blockDim.x)
      sv[(i / (L32 - L)) * L32 + L + i % (L32 - L)] = 0.0;
   auto stage = [&](int ch, int buf) {
      const int r0 = rb + ch * kChunk, nr = min(kChunk, re - r0);
      double* dst = sv + buf * kChunk * L32;
      for (int k = 0; k < nr; k++)  // 16-byte pieces (L even)
         for (int t = 2 * (int)threadIdx.x; t < L; t += 2 * (int)blockDim.x)
            cp_async16(dst + k * L32 + t, V + (int64_t)(r0 + k) * L + t);
      if (threadIdx.x < nr) st[buf * kChunk + threadIdx.x] = tau[r0 + threadIdx.x];
      cp_async_commit();
   };
   if (nchunks > 0) stage(0, 0);
   for (int ch = 0; ch < nchunks; ch++) {
      const int buf = ch & 1, r0 = rb + ch * kChunk, nr = min(kChunk, re - r0);
      if (ch + 1 < nchunks) {
         stage(ch + 1, buf ^ 1);
         cp_async_wait<1>();
      } else {
         cp_async_wait<0>();
      }
      __syncthreads();
      if (active)
         for (int k = 0; k < nr; k++) {
            const double tr = st[buf * kChunk + k];
            if (tr != 0.0) reflect(x, sv + (buf * kChunk + k) * L32, tr, r0 + k, nq, lane);
         }
      __syncthreads();  // stage buf is refilled by the copies of chunk ch + 2
   }
}

// grid (ldg rows x K, grid-stride)
__global__ void init_kernel(int K, const double* __restrict__ S0, double* __restrict__ g, int64_t ldg) {
   const int64_t total = ldg * K;
   for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < total;
        idx += (int64_t)gridDim.x * blockDim.x) {
      const int64_t r = idx % ldg, c = idx / ldg;
      g[idx] = r < K && r <= c ? S0[c * K + r] : 0.0;
   }
}

// one block of 128 threads per column c
__global__ void __launch_bounds__(128) gather_kernel(int K, int hrows, const double* __restrict__ h, int64_t ldh,
                                                     const double* __restrict__ sub, int64_t ldsub,
                                                     const int32_t* __restrict__ flag, double* __restrict__ col,
                                                     int64_t ldc, double* __restrict__ stat) {
   __shared__ double part[2][4];
   const int c = blockIdx.x, tid = threadIdx.x;
   double* out = col + (int64_t)c * ldc;
   double sh = 0.0, sr = 0.0;
   for (int r = tid; r < hrows; r += blockDim.x) {
      const double v = h[(int64_t)c * ldh + r];
      out[r] = v;
      sh = fma(v, v, sh);
   }
   for (int r = tid; r < K; r += blockDim.x) {
      const double v = r <= c ? sub[(int64_t)c * ldsub + r] : 0.0;
      out[hrows + r] = v;
      sr = fma(v, v, sr);
   }
   sh = warp_sum(sh);
   sr = warp_sum(sr);
   if ((tid & 31) == 0) {
      part[0][tid >> 5] = sh;
      part[1][tid >> 5] = sr;
   }
   __syncthreads();
   if (tid == 0) {
      stat[K + c] = part[0][0] + part[0][1] + part[0][2] + part[0][3];
      stat[2 * K + c] = part[1][0] + part[1][1] + part[1][2] + part[1][3];
      if (c == 0) stat[3 * K] = flag ? (double)*flag : 0.0;
   }
}

// Blocks i0 <= i < i1 of reflectors applied in order to columns 0 .. ncols-1 of X (ld ldx),
// block i to rows iK .. iK + 2K.  When res is set, res[c] = the norm of rows i1 K .. (i1+1) K
// of column c afterwards.
__global__ void __launch_bounds__(kApplyWarps * 32)
    apply_kernel(int K, int i0, int i1, const double* __restrict__ V, const double* __restrict__ tau,
                 double* __restrict__ X, int64_t ldx, int ncols, double* __restrict__ res) {
   extern __shared__ __align__(16) double lsm[];
   __shared__ double st[2 * kChunk];
   const int lane = threadIdx.x & 31;
   const int c = blockIdx.x * kApplyWarps + (threadIdx.x >> 5);
   const bool active = c < ncols;  // the other warps still help to stage the vectors
   const int L = 2 * K;
   double* column = X + (int64_t)min(c, ncols - 1) * ldx;
   double x[kWin];
   for (int i = i0; i < i1; i++) {
      double* w = column + (int64_t)i * K;
      if (active) load_window(x, w, L, lane);
      apply_staged(x, active, V + (int64_t)i * L * K, tau + (int64_t)i * K, 0, K, L, lane, lsm, st);
      if (active) store_window(x, w, L, lane);
      __syncwarp();  // the next window starts K rows down, in rows other lanes wrote
   }
   if (res && active) {
      double s = 0.0;
#pragma unroll
      for (int q = 0; q < kWin; q++) {
         const int t = q * 32 + lane;
         if (t >= K && t < L) s = fma(x[q], x[q], s);
      }
      s = warp_sum(s);
      if (lane == 0) res[c] = sqrt(s);
   }
}

// Columns b0 .. b0 + nb - 1 (nb = blockDim.x / 32) of the 2K x K panel W (ld ldc): warp w
// takes column b0 + w, applies reflectors 0 .. b0-1 (V, tau: this block's, from the
// earlier panels), then the panel's columns are reduced in order.  The reflector of
// column r goes to V + r 2K (all 2K entries) and tau[r].
__global__ void __launch_bounds__(kPanel * 32)
    panel_kernel(int K, int b0, double* __restrict__ W, int64_t ldc, double* __restrict__ V,
                 double* __restrict__ tau) {
   extern __shared__ __align__(16) double lsm[];
   __shared__ double vs[2][kRowsMax];
   __shared__ double ts[2];
   __shared__ double st[2 * kChunk];
   const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nb = blockDim.x >> 5;
   const int L = 2 * K, c = b0 + w, nq = (L + 31) >> 5;
   double* column = W + (int64_t)c * ldc;
   double x[kWin];
   load_window(x, column, L, lane);
   apply_staged(x, true, V, tau, 0, b0, L, lane, lsm, st);
   for (int k = 0; k < nb; k++) {
      const int r = b0 + k;
      if (w == k) {
         // the pivot x[r] from lane r % 32 (every chunk is shuffled and one kept, so that the
         // window stays in registers)
         double alpha = 0.0, sg = 0.0;
#pragma unroll
         for (int q = 0; q < kWin; q++) {
            const int t = q * 32 + lane;
            const double a = __shfl_sync(kFull, x[q], r & 31);
            if (q == (r >> 5)) alpha = a;
            if (t > r && t < L) sg = fma(x[q], x[q], sg);
         }
         const double sigma = warp_sum(sg);
         double* vk = vs[k & 1];
         double* vg = V + (int64_t)r * L;
         double tr = 0.0;
         // the shared slot gets all 32 nq rows (zeros after L), V the L rows
         if (sigma == 0.0) {
#pragma unroll
            for (int q = 0; q < kWin; q++) {
               const int t = q * 32 + lane;
               const double v = t == r ? 1.0 : 0.0;
               if (q < nq) vk[t] = v;
               if (t < L) vg[t] = v;
            }
         } else {
            const double normx = sqrt(alpha * alpha + sigma);
            const double beta = alpha <= 0.0 ? normx : -normx;
            tr = (beta - alpha) / beta;
            const double scale = 1.0 / (alpha - beta);
#pragma unroll
            for (int q = 0; q < kWin; q++) {
               const int t = q * 32 + lane;
               const double v = t > r && t < L ? x[q] * scale : (t == r ? 1.0 : 0.0);
               if (q < nq) vk[t] = v;
               if (t < L) {
                  vg[t] = v;
                  if (t > r) x[q] = 0.0;
                  if (t == r) x[q] = beta;
               }
            }
         }
         if (lane == 0) {
            ts[k & 1] = tr;
            tau[r] = tr;
         }
      }
      // Slot k & 1 is rewritten at step k + 2, by a warp that has passed the barrier of
      // step k + 1, which every reader of step k reaches only after reading.
      __syncthreads();
      if (w > k) {
         const double tr = ts[k & 1];
         if (tr != 0.0) reflect(x, vs[k & 1], tr, r, nq, lane);
      }
   }
   store_window(x, column, L, lane);
}

// raises the staged kernels' dynamic shared-memory limits (K = 256), once per device
void prepare() {
   static std::atomic<uint64_t> done{0};
   int dev = 0;
   FFTSVD_CUDA(cudaGetDevice(&dev));
   const uint64_t bit = dev < 64 ? uint64_t(1) << dev : 0;
   if (bit && (done.load(std::memory_order_acquire) & bit)) return;
   const int bytes = (int)stage_bytes(kRowsMax / 2);
   FFTSVD_CUDA(cudaFuncSetAttribute(apply_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
   FFTSVD_CUDA(cudaFuncSetAttribute(panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
   done.fetch_or(bit, std::memory_order_acq_rel);
}

}  // namespace

void init(int K, const double* S0, double* g, int64_t ldg, cudaStream_t s) {
   FFTSVD_REQUIRE(K > 0 && K <= kRowsMax / 2 && ldg >= 2 * K, "block least squares: sizes");
   const int64_t total = ldg * K;
   const int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 8);
   init_kernel<<<blocks, 256, 0, s>>>(K, S0, g, ldg);
   FFTSVD_CHECK_LAUNCH();
}

void gather(int j, int K, const double* h, int64_t ldh, const double* sub, int64_t ldsub, const int32_t* flag,
            double* col, int64_t ldc, double* stat, cudaStream_t s) {
   const int hrows = (j + 1) * K;
   FFTSVD_REQUIRE(K > 0 && K <= kRowsMax / 2 && j >= 0 && ldh >= hrows && ldsub >= K && ldc >= hrows + K,
                  "block least squares: sizes");
   gather_kernel<<<K, 128, 0, s>>>(K, hrows, h, ldh, sub, ldsub, flag, col, ldc, stat);
   FFTSVD_CHECK_LAUNCH();
}

void step(int j, int K, double* col, int64_t ldc, double* V, double* tau, double* g, int64_t ldg, double* Rd,
          int64_t ldr, double* stat, cudaStream_t s) {
   FFTSVD_REQUIRE(K > 0 && K <= kRowsMax / 2 && j >= 0 && ldc >= (int64_t)(j + 2) * K && ldg >= (int64_t)(j + 2) * K,
                  "block least squares: sizes");
   FFTSVD_REQUIRE(!Rd || ldr >= (int64_t)(j + 1) * K, "block least squares: factor rows");
   prepare();
   const int L = 2 * K;
   const size_t smem = stage_bytes(K);
   const int apply_blocks = (K + kApplyWarps - 1) / kApplyWarps;
   if (j > 0) {
      apply_kernel<<<apply_blocks, kApplyWarps * 32, smem, s>>>(K, 0, j, V, tau, col, ldc, K, nullptr);
      FFTSVD_CHECK_LAUNCH();
   }
   double* Vj = V + (int64_t)j * L * K;
   double* tj = tau + (int64_t)j * K;
   for (int b0 = 0; b0 < K; b0 += kPanel) {
      const int nb = std::min(kPanel, K - b0);
      panel_kernel<<<1, nb * 32, smem, s>>>(K, b0, col + (int64_t)j * K, ldc, Vj, tj);
      FFTSVD_CHECK_LAUNCH();
   }
   if (Rd)
      FFTSVD_CUDA(cudaMemcpy2DAsync(Rd + (int64_t)j * K * ldr, sizeof(double) * ldr, col, sizeof(double) * ldc,
                                    sizeof(double) * (j + 1) * K, K, cudaMemcpyDeviceToDevice, s));
   apply_kernel<<<apply_blocks, kApplyWarps * 32, smem, s>>>(K, j, j + 1, V, tau, g, ldg, K, stat);
   FFTSVD_CHECK_LAUNCH();
}

}  // namespace lsq
}  // namespace fftsvd
