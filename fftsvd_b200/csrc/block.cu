// Block GMRES: many right-hand sides of one surface in one shared Krylov space.
//
// Where the lockstep batch (batch.cu) gives every column its own Krylov basis, block
// GMRES grows one basis by a block of K vectors per step: V_{j+1} R_{j+1,j} =
// P^-1 A V_j - sum_i V_i H_ij, with the block Gram-Schmidt coefficients H_ij and the
// block QR factor R_{j+1,j}.  Each column's solution is sought in the span of all
// blocks, so the columns help one another: on 256 charge-group right-hand sides of
// an 81 920-unknown surface every column reaches 1e-6 in about 14 block steps, where a
// column alone takes about 46 GMRES steps.  The Krylov spaces differ from the single
// solves', so the columns agree with single solves to the tolerance, not bit for bit.
//
// Device: the multi-vector matvec and preconditioner of the batch, the block
// Gram-Schmidt and the products with the basis as FP64 tensor-core GEMMs (dense.cu), the
// block QR as CholQR2 (Gram matrix, Cholesky factor in a one-block kernel, product with
// the factor's inverse; twice), the final block triangular solve (dense.cu).  Gram-Schmidt
// is one classical pass while no column of a new block loses more than five digits in it
// (the new block is then orthogonal to the basis to about 1e-11, far below what a solve to
// 1e-6 needs), two passes from the first step where one does.  The block Hessenberg
// least-squares problem is updated on the device too (block_ls.cu), on a second stream:
// step j's update runs while the main stream runs step j + 1, and the host reads back
// only the residual estimates, the block's norms and the rank flag (3K + 1 numbers).
//
// Refinement: each pass gathers the columns still above the tolerance, scales their
// residuals to unit norm, pads them to a multiple of 8 with seeded random directions
// (which keep the block full rank and are not monitored), runs one block GMRES cycle
// and adds the scaled corrections back; the residual is then recomputed with the outer
// operator (FP64 for the mixed mode, as the single solve's refinement).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <string>
#include <vector>

#include "block.h"
#include "block_ls.h"
#include "dense.h"
#include "surface.h"

namespace fftsvd {

namespace {

constexpr int kCholThreads = 1024;
constexpr int kCholBlock = 32;
constexpr int kMaxPasses = 16;
// A column whose norm falls below this fraction in the first Gram-Schmidt pass would be
// left orthogonal to the basis only to eps / fraction: later steps then take two passes.
constexpr double kReorthRatio = 1e-5;
// Inner target of a mixed-precision pass, as a fraction of the tolerance.
constexpr double kMixedTarget = 0.9;

// G (K x K, symmetric, column-major, K <= kBlockMax) = R^T R: writes the upper-triangular
// R (zero below the diagonal).  Right-looking, blocked by 32 rows: one warp factors the
// 32 x 32 diagonal block in shared memory, one thread per column solves the panel to its
// right (kept in shared memory), and all threads update the trailing upper triangle from
// the panel.  *flag = 1 when a pivot is not above 1e-24 of the largest diagonal entry of G
// (or not finite): the columns are numerically dependent; that pivot is then taken as 1
// so that nothing turns into NaN.  One block, chol_smem(K) bytes of dynamic shared memory.
__global__ void __launch_bounds__(kCholThreads) chol_kernel(int K, const double* __restrict__ G,
                                                            double* __restrict__ R, int32_t* __restrict__ flag) {
   extern __shared__ double sm[];
   double* D = sm;                            // diagonal block, D[c * 32 + r]
   double* P = sm + kCholBlock * kCholBlock;  // panel, P[l * K + c] (row l of the block, column c)
   __shared__ double gmax;
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
   for (int idx = tid; idx < K * K; idx += blockDim.x) {
      const int r = idx % K, c = idx / K;
      R[idx] = r <= c ? G[idx] : 0.0;
   }
   if (warp == 0) {
      double m = 0.0;
      for (int k = lane; k < K; k += 32) m = fmax(m, G[(int64_t)k * K + k]);
      for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
      if (lane == 0) gmax = m;
   }
   __syncthreads();
   for (int k0 = 0; k0 < K; k0 += kCholBlock) {
      const int bs = min(kCholBlock, K - k0), k1 = k0 + bs, m = K - k1;
      if (warp == 0) {  // lane = column of the diagonal block
         for (int r = 0; r < bs; r++)
            if (lane < bs) D[lane * 32 + r] = R[(int64_t)(k0 + lane) * K + k0 + r];
         __syncwarp();
         for (int kk = 0; kk < bs; kk++) {
            double a = D[kk * 32 + kk];
            const bool bad = !(a > 1e-24 * gmax) || !isfinite(a);
            if (bad) a = 1.0;
            const double p = sqrt(a);
            if (lane == 0 && bad) *flag = 1;
            __syncwarp();
            double dk = 0.0;
            if (lane > kk && lane < bs) {
               dk = D[lane * 32 + kk] / p;
               D[lane * 32 + kk] = dk;
            }
            if (lane == kk) D[kk * 32 + kk] = p;
            __syncwarp();
            if (lane > kk && lane < bs)
               for (int i = kk + 1; i <= lane; i++) D[lane * 32 + i] -= D[i * 32 + kk] * dk;
            __syncwarp();
         }
         for (int r = 0; r < bs; r++)
            if (lane < bs && r <= lane) R[(int64_t)(k0 + lane) * K + k0 + r] = D[lane * 32 + r];
      }
      __syncthreads();
      // panel: D^T X = R[k0:k1, k1:K] by forward substitution, one column per thread
      for (int t = tid; t < m; t += blockDim.x) {
         const int c = k1 + t;
         for (int r = 0; r < bs; r++) {
            double v = R[(int64_t)c * K + k0 + r];
            for (int l = 0; l < r; l++) v -= D[r * 32 + l] * P[l * K + c];
            v /= D[r * 32 + r];
            P[r * K + c] = v;
            R[(int64_t)c * K + k0 + r] = v;
         }
      }
      __syncthreads();
      // trailing upper triangle: R[i, c] -= sum over the panel rows of P[l, i] P[l, c]
      for (int idx = tid; idx < m * m; idx += blockDim.x) {
         const int ii = idx % m, cc = idx / m;
         if (ii > cc) continue;
         const int i = k1 + ii, c = k1 + cc;
         double v = 0.0;
         for (int l = 0; l < bs; l++) v += P[l * K + i] * P[l * K + c];
         R[(int64_t)c * K + i] -= v;
      }
      __syncthreads();
   }
}

size_t chol_smem(int K) { return sizeof(double) * ((size_t)kCholBlock * kCholBlock + (size_t)kCholBlock * K); }

// Columns c0 <= c < c1 of v (column c at v + c * n): seeded uniform values in
// [-scale, scale), the splitmix64 generator on the element index.
__global__ void seeded_fill_kernel(int64_t n, int c0, int c1, double scale, double* __restrict__ v) {
   const int64_t total = (int64_t)(c1 - c0) * n;
   for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
      uint64_t z = (uint64_t)(k + (int64_t)c0 * n + 1) * 0x9E3779B97F4A7C15ull;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      z ^= z >> 31;
      v[(int64_t)c0 * n + k] = scale * ((double)(z >> 11) * (2.0 / 9007199254740992.0) - 1.0);
   }
}

// grid (blocks, 1, columns): dst column a = fac[a] * src column idx[a]
__global__ void gather_scale_kernel(int64_t n, const double* __restrict__ src, const int32_t* __restrict__ idx,
                                    const double* __restrict__ fac, double* __restrict__ dst) {
   const int a = blockIdx.z;
   const double* s = src + (int64_t)idx[a] * n;
   double* d = dst + (int64_t)a * n;
   const double f = fac[a];
   for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      d[i] = f * s[i];
}

// grid (blocks, 1, columns): dst column idx[a] = src column a
__global__ void scatter_copy_kernel(int64_t n, const double* __restrict__ src, const int32_t* __restrict__ idx,
                                    double* __restrict__ dst) {
   const int a = blockIdx.z;
   const double* s = src + (int64_t)a * n;
   double* d = dst + (int64_t)idx[a] * n;
   for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      d[i] = s[i];
}

// grid (blocks, 1, columns): dst column idx[a] += fac[a] * src column a
__global__ void scatter_add_kernel(int64_t n, const double* __restrict__ src, const int32_t* __restrict__ idx,
                                   const double* __restrict__ fac, double* __restrict__ dst) {
   const int a = blockIdx.z;
   const double* s = src + (int64_t)a * n;
   double* d = dst + (int64_t)idx[a] * n;
   const double f = fac[a];
   for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
      d[i] += f * s[i];
}

int pad8(int k) { return (k + kBatchGroup - 1) / kBatchGroup * kBatchGroup; }

}  // namespace

BlockWorkspace::~BlockWorkspace() {
   if (ls_stream) cudaStreamSynchronize(ls_stream);
   for (auto& e : done)
      if (e) cudaEventDestroy(e);
   for (auto& e : ls_done)
      if (e) cudaEventDestroy(e);
   if (ls_stream) cudaStreamDestroy(ls_stream);
   for (auto& p : stat_h)
      if (p) cudaFreeHost(p);
   if (flag_h) cudaFreeHost(flag_h);
}

void BlockWorkspace::ensure(int64_t n_, int K_, int mmax_, cudaStream_t stream) {
   (void)stream;
   if (!flag_h) {
      for (auto& e : done) FFTSVD_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      for (auto& e : ls_done) FFTSVD_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      // the least-squares kernels take few SMs for a short time; the greatest priority lets
      // them start while the next step's matvec fills the device
      int least = 0, greatest = 0;
      FFTSVD_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
      FFTSVD_CUDA(cudaStreamCreateWithPriority(&ls_stream, cudaStreamNonBlocking, greatest));
      FFTSVD_CUDA(cudaMallocHost(&flag_h, 2 * sizeof(int)));
      FFTSVD_CUDA(cudaFuncSetAttribute(chol_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)chol_smem(kBlockMax)));
   }
   if (n_ == n && K_ <= K && mmax_ <= mmax) return;
   if (n_ != n) K = mmax = 0;
   n = n_;
   K = std::max(K, K_);
   mmax = std::max(mmax, mmax_);
   const size_t kn = (size_t)K * n, kk = (size_t)K * K;
   V.alloc((size_t)(mmax + 1) * kn);
   for (DevBuf<double>* b : {&W, &R0, &T, &Bc, &Xc, &Rc, &Tc, &Qs}) b->alloc(kn);
   H.alloc((size_t)(mmax + 1) * kk);
   H2.alloc((size_t)(mmax + 1) * kk);
   for (DevBuf<double>* b : {&G, &R1, &R2, &R, &Rinv}) b->alloc(kk);
   Y.alloc((size_t)mmax * kk);
   Yo.alloc((size_t)mmax * kk);
   Dinv.alloc((size_t)mmax * kk);
   // split-K partials of the Gram matrices (K x K) and of the projections on up to mmax blocks
   int64_t wmax = dense::gemm_tn_work(K, K, n);
   for (int j = 1; j <= mmax; j++) wmax = std::max(wmax, dense::gemm_tn_work(j * K, K, n));
   gwork.alloc((size_t)std::max<int64_t>(wmax, 1));
   Rd.alloc((size_t)mmax * K * (size_t)mmax * K);
   Lv.alloc((size_t)mmax * 2 * kk);
   Ltau.alloc((size_t)mmax * K);
   Lg.alloc((size_t)(mmax + 1) * kk);
   for (int s = 0; s < 2; s++) {
      Lcol[s].alloc((size_t)(mmax + 1) * kk);
      Lstat[s].alloc((size_t)3 * K + 1);
      if (stat_h[s]) cudaFreeHost(stat_h[s]);
      stat_h[s] = nullptr;
      FFTSVD_CUDA(cudaMallocHost(&stat_h[s], sizeof(double) * ((size_t)3 * K + 1)));
   }
   scal.alloc(K);
   part.alloc((size_t)K * vec_blocks(n));
   fac.alloc(K);
   idx.alloc(K);
   flag.alloc(1);
}

// Q R = X (n x K, both column-major with ld n; X may be Q) by CholQR2: twice the Gram
// matrix, its Cholesky factor R_p and the product with R_p^-1 (out of place, through the
// scratch block Qs).  R = R_2 R_1 (K x K) is left in blk->R and a rank deficiency raises
// blk->flag.
void Surface::block_qr(const double* X, double* Q, int K) {
   BlockWorkspace& B = *blk;
   const double* src = X;
   for (int pass = 0; pass < 2; pass++) {
      double* Rp = pass ? B.R2.get() : B.R1.get();
      double* dst = pass ? Q : B.Qs.get();
      dense::gemm_tn(K, K, n, 1.0, src, n, src, n, 0.0, B.G.get(), K, B.gwork.get(), stream);
      chol_kernel<<<1, kCholThreads, chol_smem(K), stream>>>(K, B.G.get(), Rp, B.flag.get());
      FFTSVD_CHECK_LAUNCH();
      dense::trinv_upper(K, 1, Rp, K, 0, B.Rinv.get(), K, 0, stream);
      dense::gemm_nn(n, K, K, 1.0, src, n, B.Rinv.get(), K, 0.0, dst, n, stream);
      src = dst;
   }
   dense::gemm_nn(K, K, K, 1.0, B.R2.get(), K, B.R1.get(), K, 0.0, B.R.get(), K, stream);
}

// One cycle of block GMRES on P^-1 A T = R0 (K columns, A the operator `precision`),
// T += the minimiser over the block Krylov space of up to mmax blocks.  Stops when each
// monitored column c < nmon has residual <= target[c] (absolute, preconditioned), after
// mmax block steps, or when a new block is numerically dependent on the basis (the
// cycle then keeps the blocks before it).  res receives the residual estimates of the
// K columns; returns the block steps used, 0 when the columns of R0 are dependent.
int Surface::gmres_block(int precision, int K, const double* R0, double* T, int nmon, const std::vector<double>& target,
                         int mmax, std::vector<double>& res) {
   BlockWorkspace& B = *blk;
   const int64_t vblk = (int64_t)K * n;
   double* V = B.V.get();
   res.assign(K, 0.0);
   // nothing of an earlier cycle may still run on the least-squares stream (a cycle left by
   // an error does not wait for it): its buffers are rewritten below
   FFTSVD_CUDA(cudaStreamSynchronize(B.ls_stream));
   // V_0 S0 = R0
   FFTSVD_CUDA(cudaMemsetAsync(B.flag.get(), 0, sizeof(int32_t), stream));
   block_qr(R0, V, K);
   std::vector<double> S0((size_t)K * K);
   FFTSVD_CUDA(cudaMemcpyAsync(S0.data(), B.R.get(), sizeof(double) * K * K, cudaMemcpyDeviceToHost, stream));
   FFTSVD_CUDA(cudaMemcpyAsync(B.flag_h, B.flag.get(), sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
   FFTSVD_CUDA(cudaStreamSynchronize(stream));
   if (B.flag_h[0]) return 0;
   // least squares on the device (block_ls.h): the transformed right-hand side starts as S0
   const int64_t ldl = (int64_t)(B.mmax + 1) * B.K;  // rows of Lg and Lcol
   const int64_t ldr = (int64_t)B.mmax * B.K;        // rows of Rd
   lsq::init(K, B.R.get(), B.Lg.get(), ldl, stream);
   // step j: W = P^-1 A V_j, block Gram-Schmidt against V_0 .. V_j (a second pass once
   // `reorth` is set), V_{j+1} R = W; the coefficients, R and the rank flag are gathered
   // into slot j & 1, and the least-squares update of step j then runs on the side stream
   // while the main stream goes on with step j + 1
   bool reorth = false;
   auto issue = [&](int j) {
      const int rows = (j + 1) * K;
      const int slot = j & 1;
      apply_batch(precision, V + j * vblk, B.W.get(), K);
      precond_batch(B.W.get(), B.W.get(), K);
      dense::gemm_tn(rows, K, n, 1.0, V, n, B.W.get(), n, 0.0, B.H.get(), rows, B.gwork.get(), stream);
      dense::gemm_nn(n, K, rows, -1.0, V, n, B.H.get(), rows, 1.0, B.W.get(), n, stream);
      if (reorth) {
         dense::gemm_tn(rows, K, n, 1.0, V, n, B.W.get(), n, 0.0, B.H2.get(), rows, B.gwork.get(), stream);
         dense::gemm_nn(n, K, rows, -1.0, V, n, B.H2.get(), rows, 1.0, B.W.get(), n, stream);
         dense::add(rows, K, B.H.get(), rows, B.H2.get(), rows, B.H.get(), rows, stream);
      }
      FFTSVD_CUDA(cudaMemsetAsync(B.flag.get(), 0, sizeof(int32_t), stream));
      block_qr(B.W.get(), V + (j + 1) * vblk, K);
      lsq::gather(j, K, B.H.get(), rows, B.R.get(), K, B.flag.get(), B.Lcol[slot].get(), ldl, B.Lstat[slot].get(),
                  stream);
      FFTSVD_CUDA(cudaEventRecord(B.done[slot], stream));
      FFTSVD_CUDA(cudaStreamWaitEvent(B.ls_stream, B.done[slot], 0));
      lsq::step(j, K, B.Lcol[slot].get(), ldl, B.Lv.get(), B.Ltau.get(), B.Lg.get(), ldl, B.Rd.get(), ldr,
                B.Lstat[slot].get(), B.ls_stream);
      FFTSVD_CUDA(cudaMemcpyAsync(B.stat_h[slot], B.Lstat[slot].get(), sizeof(double) * (3 * (size_t)K + 1),
                                  cudaMemcpyDeviceToHost, B.ls_stream));
      FFTSVD_CUDA(cudaEventRecord(B.ls_done[slot], B.ls_stream));
   };
   // residual estimates after the last two steps (before any step: the columns' norms)
   std::vector<double> prev(K), prev2(K);
   for (int c = 0; c < K; c++) {
      double s = 0.0;
      for (int r = 0; r <= c; r++) s += S0[(size_t)c * K + r] * S0[(size_t)c * K + r];
      prev[c] = prev2[c] = std::sqrt(s);
   }
   // Step j + 1 is issued before the host takes step j unless the last convergence rate
   // predicts that step j meets every target (then it would be wasted).
   auto speculate = [&](int j) {
      if (j == 0) return true;
      for (int c = 0; c < nmon; c++) {
         const double q = prev2[c] > 0.0 ? std::min(1.0, prev[c] / prev2[c]) : 1.0;
         if (prev[c] * q > 2.0 * target[c]) return true;
      }
      return false;
   };
   int m = 0, issued = 0;
   issue(0);
   issued = 1;
   for (int j = 0; j < mmax; j++) {
      if (issued == j + 1 && j + 1 < mmax && speculate(j)) issue(issued++);
      FFTSVD_CUDA(cudaEventSynchronize(B.ls_done[j & 1]));
      const double* st = B.stat_h[j & 1];
      if (st[3 * K] != 0.0) break;  // V_{j+1} is not a basis: keep the first j blocks
      std::copy(st, st + K, res.begin());
      m = j + 1;
      // the new block's norms after the projection against those before it
      for (int c = 0; c < K && !reorth; c++) {
         const double sh = st[K + c], sr = st[2 * K + c];
         if (sr < kReorthRatio * kReorthRatio * (sh + sr)) reorth = true;
      }
      bool all = true;
      for (int c = 0; c < nmon && all; c++) all = res[c] <= target[c];
      if (all) break;
      prev2.swap(prev);
      prev = res;
      if (issued == j + 1 && j + 1 < mmax) issue(issued++);
   }
   // a speculative step and its least-squares update may still run; neither writes the
   // rows and block columns of the first m steps
   FFTSVD_CUDA(cudaStreamSynchronize(stream));
   FFTSVD_CUDA(cudaStreamSynchronize(B.ls_stream));
   if (m == 0) return 0;
   // Y = R^-1 g_top: g's first mK rows into Y (ld mK), block triangular solve on Rd
   const int rows = m * K;
   FFTSVD_CUDA(cudaMemcpy2DAsync(B.Y.get(), sizeof(double) * rows, B.Lg.get(), sizeof(double) * ldl,
                                 sizeof(double) * rows, K, cudaMemcpyDeviceToDevice, stream));
   dense::trsm_upper_left(rows, K, K, B.Rd.get(), ldr, B.Y.get(), B.Dinv.get(), B.Yo.get(), stream);
   dense::gemm_nn(n, K, rows, 1.0, V, n, B.Yo.get(), rows, 1.0, T, n, stream);
   return m;
}

int Surface::solve_block(int precision, int k, const double* rhs, double* x, double tol, int maxit,
                         fftsvd_solve_info* info) {
   FFTSVD_REQUIRE(k > 0 && k <= kMaxBatch, "right-hand side count");
   FFTSVD_REQUIRE(tol > 0.0 && maxit > 0, "tolerance and iteration cap must be positive");
   FFTSVD_REQUIRE(precision == FFTSVD_PREC_FP64 || precision == FFTSVD_PREC_FP32 || precision == FFTSVD_PREC_MIXED,
                  "unknown precision mode");
   const auto clock_start = std::chrono::steady_clock::now();
   const bool mixed = precision == FFTSVD_PREC_MIXED;
   const int inner = mixed ? FFTSVD_PREC_FP32 : precision, outer = mixed ? FFTSVD_PREC_FP64 : precision;
   if (!blk) blk = std::make_unique<BlockWorkspace>();
   // the FP32 multi-vector matvecs of the block solve take the tensor-core near field
   struct TensorNear {
      DeviceOperator<float>& op;
      explicit TensorNear(DeviceOperator<float>& o) : op(o) { op.set_tensor_near(true); }
      ~TensorNear() { op.set_tensor_near(false); }
   } tensor_near(op32);
   const int ew_blocks = std::max(1, std::min((n + 255) / 256, 148 * 8));
   const int nb = vec_blocks(n);
   std::vector<int> iters(k, 0), refinements(k, 0), status(k, FFTSVD_OK);
   std::vector<double> resid(k, 0.0);
   for (int c0 = 0; c0 < k; c0 += kBlockMax) {
      const int nc = std::min(kBlockMax, k - c0), ncp = pad8(nc);
      // basis: up to maxit blocks (at most 64), as many as a third of the device memory
      // that is free or already held by the basis allows, counting the mmax + 11 blocks of
      // K x n (basis and work vectors), the dense (mmax K)^2 least-squares factor and the
      // least-squares update's 5 K^2 per block (reflectors, right-hand side, column slots)
      size_t free_b = 0, total_b = 0;
      FFTSVD_CUDA(cudaMemGetInfo(&free_b, &total_b));
      if (blk->n == n) free_b += blk->V.bytes() + blk->Rd.bytes();
      const size_t per_blk = sizeof(double) * ((size_t)ncp * n + 5 * (size_t)ncp * ncp);
      int mmax = std::max(1, std::min(maxit, 64));
      while (mmax > 1 && (mmax + 11) * per_blk + sizeof(double) * (size_t)mmax * ncp * (size_t)mmax * ncp > free_b / 3)
         mmax--;
      blk->ensure(n, ncp, mmax, stream);
      BlockWorkspace& B = *blk;
      FFTSVD_CUDA(cudaMemsetAsync(B.Bc.get(), 0, sizeof(double) * (size_t)ncp * n, stream));
      FFTSVD_CUDA(cudaMemcpyAsync(B.Bc.get(), rhs + (int64_t)c0 * n, sizeof(double) * (size_t)nc * n,
                                  cudaMemcpyDeviceToDevice, stream));
      FFTSVD_CUDA(cudaMemsetAsync(B.Xc.get(), 0, sizeof(double) * (size_t)ncp * n, stream));
      std::vector<double> bn(nc, 0.0), rn(ncp, 0.0);
      std::vector<int32_t> last;  // columns corrected by the last pass
      int used = 0;
      bool fallback = false;
      for (int pass = 0;; pass++) {
         // Rc = P^-1 (B - A X), the outer operator (P^-1 B on the first pass).  Only the
         // columns corrected by the last pass change; when they are fewer than all, their
         // residuals are computed as a compact block and scattered back.
         if (pass == 0) {
            precond_batch(B.Bc.get(), B.Rc.get(), ncp);
         } else if ((int)last.size() == nc) {
            apply_batch(outer, B.Xc.get(), B.Tc.get(), ncp);
            sub_kernel<<<dim3(ew_blocks, 1, ncp), 256, 0, stream>>>(n, B.Bc.get(), B.Tc.get(), B.Tc.get(), n);
            FFTSVD_CHECK_LAUNCH();
            precond_batch(B.Tc.get(), B.Rc.get(), ncp);
         } else {
            const int nl = (int)last.size(), Kl = pad8(nl);
            const std::vector<double> ones(nl, 1.0);
            FFTSVD_CUDA(cudaMemcpyAsync(B.idx.get(), last.data(), sizeof(int32_t) * nl, cudaMemcpyHostToDevice, stream));
            FFTSVD_CUDA(cudaMemcpyAsync(B.fac.get(), ones.data(), sizeof(double) * nl, cudaMemcpyHostToDevice, stream));
            FFTSVD_CUDA(cudaMemsetAsync(B.R0.get(), 0, sizeof(double) * (size_t)Kl * n, stream));
            FFTSVD_CUDA(cudaMemsetAsync(B.T.get(), 0, sizeof(double) * (size_t)Kl * n, stream));
            gather_scale_kernel<<<dim3(ew_blocks, 1, nl), 256, 0, stream>>>(n, B.Xc.get(), B.idx.get(), B.fac.get(),
                                                                          B.R0.get());
            FFTSVD_CHECK_LAUNCH();
            gather_scale_kernel<<<dim3(ew_blocks, 1, nl), 256, 0, stream>>>(n, B.Bc.get(), B.idx.get(), B.fac.get(),
                                                                          B.T.get());
            FFTSVD_CHECK_LAUNCH();
            apply_batch(outer, B.R0.get(), B.W.get(), Kl);
            sub_kernel<<<dim3(ew_blocks, 1, Kl), 256, 0, stream>>>(n, B.T.get(), B.W.get(), B.W.get(), n);
            FFTSVD_CHECK_LAUNCH();
            precond_batch(B.W.get(), B.R0.get(), Kl);
            scatter_copy_kernel<<<dim3(ew_blocks, 1, nl), 256, 0, stream>>>(n, B.R0.get(), B.idx.get(), B.Rc.get());
            FFTSVD_CHECK_LAUNCH();
         }
         norm_partial_kernel<<<dim3(nb, 1, ncp), kVecThreads, 0, stream>>>(n, B.Rc.get(), B.part.get(), n, nb);
         FFTSVD_CHECK_LAUNCH();
         reduce_partial_kernel<<<dim3(1, 1, ncp), 256, 0, stream>>>(1, nb, B.part.get(), B.scal.get(), 0, nb, 1);
         FFTSVD_CHECK_LAUNCH();
         FFTSVD_CUDA(cudaMemcpyAsync(rn.data(), B.scal.get(), sizeof(double) * ncp, cudaMemcpyDeviceToHost, stream));
         FFTSVD_CUDA(cudaStreamSynchronize(stream));
         std::vector<int32_t> act;
         std::vector<double> target;
         for (int a = 0; a < nc; a++) {
            const int c = c0 + a;
            rn[a] = std::sqrt(rn[a]);
            if (pass == 0) {
               bn[a] = rn[a];
               if (!std::isfinite(bn[a])) {  // left out; its solution stays zero
                  status[c] = FFTSVD_ERR_NONFINITE;
                  resid[c] = bn[a];
               }
            }
            if (status[c] != FFTSVD_OK || bn[a] == 0.0) continue;  // zero right-hand side: zero solution
            resid[c] = rn[a] / bn[a];
            if (!std::isfinite(resid[c])) {
               status[c] = FFTSVD_ERR_NONFINITE;
               continue;
            }
            if (resid[c] < tol) continue;
            act.push_back(a);
            // relative to the column's current residual: for a mixed correction 0.9 tol /
            // residual (the FP32 operator's share of the FP64 residual is far below 0.1 tol on
            // these surfaces, and a column that still misses the tolerance takes a short
            // pass of its own), else the tolerance itself
            target.push_back(mixed ? std::min(0.1, std::max(kMixedTarget * tol / resid[c], 1e-13)) : tol / resid[c]);
         }
         if (act.empty() || used >= maxit || pass >= kMaxPasses) break;
         last = act;
         const int na = (int)act.size(), K = pad8(na);
         std::vector<double> f(na);
         for (int a = 0; a < na; a++) f[a] = 1.0 / rn[act[a]];
         FFTSVD_CUDA(cudaMemcpyAsync(B.idx.get(), act.data(), sizeof(int32_t) * na, cudaMemcpyHostToDevice, stream));
         FFTSVD_CUDA(cudaMemcpyAsync(B.fac.get(), f.data(), sizeof(double) * na, cudaMemcpyHostToDevice, stream));
         gather_scale_kernel<<<dim3(ew_blocks, 1, na), 256, 0, stream>>>(n, B.Rc.get(), B.idx.get(), B.fac.get(),
                                                                       B.R0.get());
         FFTSVD_CHECK_LAUNCH();
         if (K > na) {
            seeded_fill_kernel<<<ew_blocks, 256, 0, stream>>>(n, na, K, std::sqrt(3.0 / n), B.R0.get());
            FFTSVD_CHECK_LAUNCH();
         }
         FFTSVD_CUDA(cudaMemsetAsync(B.T.get(), 0, sizeof(double) * (size_t)K * n, stream));
         std::vector<double> est;
         const int m = gmres_block(inner, K, B.R0.get(), B.T.get(), na, target, std::min(mmax, maxit - used), est);
         if (m == 0) {
            // dependent right-hand sides (or residuals): the lockstep batch handles them
            fallback = pass == 0;
            break;
         }
         for (int a = 0; a < na; a++) f[a] = rn[act[a]];
         FFTSVD_CUDA(cudaMemcpyAsync(B.fac.get(), f.data(), sizeof(double) * na, cudaMemcpyHostToDevice, stream));
         scatter_add_kernel<<<dim3(ew_blocks, 1, na), 256, 0, stream>>>(n, B.T.get(), B.idx.get(), B.fac.get(),
                                                                      B.Xc.get());
         FFTSVD_CHECK_LAUNCH();
         used += m;
         for (int a : act) {
            iters[c0 + a] += m;
            if (mixed) refinements[c0 + a]++;
         }
      }
      if (fallback) {
         std::vector<fftsvd_solve_info> sub(nc);
         solve_batch(precision, nc, rhs + (int64_t)c0 * n, B.Xc.get(), tol, maxit, sub.data());
         for (int a = 0; a < nc; a++) {
            iters[c0 + a] = sub[a].iterations;
            refinements[c0 + a] = sub[a].refinements;
            status[c0 + a] = sub[a].status;
            resid[c0 + a] = sub[a].residual;
         }
      }
      for (int a = 0; a < nc; a++) {
         const int c = c0 + a;
         if (status[c] == FFTSVD_OK && !(resid[c] < tol) && bn[a] != 0.0) status[c] = FFTSVD_ERR_NOT_CONVERGED;
      }
      FFTSVD_CUDA(cudaMemcpyAsync(x + (int64_t)c0 * n, B.Xc.get(), sizeof(double) * (size_t)nc * n,
                                  cudaMemcpyDeviceToDevice, stream));
      FFTSVD_CUDA(cudaStreamSynchronize(stream));
   }
   const auto clock_end = std::chrono::steady_clock::now();
   const double ms = std::chrono::duration<double, std::milli>(clock_end - clock_start).count();
   if (op32.tensor_status(true))
      throw Error(FFTSVD_ERR_TIMEOUT, "a tensor-core near-field wait gave up (results discarded)");
   int first_bad = FFTSVD_OK;
   for (int c = 0; c < k; c++) {
      if (first_bad == FFTSVD_OK && status[c] != FFTSVD_OK) first_bad = status[c];
      if (info) {
         info[c].iterations = iters[c];
         info[c].refinements = refinements[c];
         info[c].status = status[c];
         info[c].residual = resid[c];
         info[c].setup_ms = 0.0;
         info[c].solve_ms = ms;
      }
   }
   return first_bad;
}

}  // namespace fftsvd

using namespace fftsvd;

extern "C" {

int fftsvd_b200_solve_block_device(fftsvd_surface* s, int32_t nrhs, int32_t precision, const double* rhs, double* sol,
                                   double tol, int32_t max_iterations, fftsvd_solve_info* info) {
   if (!s || !rhs || !sol || nrhs <= 0) return FFTSVD_ERR_ARGUMENT;
   int status = FFTSVD_OK;
   const int rc = guarded([&] { status = s->s.solve_block(precision, nrhs, rhs, sol, tol, max_iterations, info); });
   return rc != FFTSVD_OK ? rc : status;
}

int fftsvd_b200_solve_block(fftsvd_surface* s, int32_t nrhs, int32_t precision, const double* rhs, double* sol,
                            double tol, int32_t max_iterations, fftsvd_solve_info* info) {
   if (!s || !rhs || !sol || nrhs <= 0) return FFTSVD_ERR_ARGUMENT;
   int status = FFTSVD_OK;
   const int rc = guarded([&] {
      Surface& S = s->s;
      const size_t bytes = sizeof(double) * (size_t)nrhs * S.n;
      DevBuf<double> din((size_t)nrhs * S.n), dout((size_t)nrhs * S.n);
      FFTSVD_CUDA(cudaMemcpyAsync(din.get(), rhs, bytes, cudaMemcpyHostToDevice, S.stream));
      status = S.solve_block(precision, nrhs, din.get(), dout.get(), tol, max_iterations, info);
      FFTSVD_CUDA(cudaMemcpyAsync(sol, dout.get(), bytes, cudaMemcpyDeviceToHost, S.stream));
      FFTSVD_CUDA(cudaStreamSynchronize(S.stream));
   });
   return rc != FFTSVD_OK ? rc : status;
}

}  // extern "C"
