// Dense FP64 kernels of the block GMRES solve, on the FP64 tensor-core MMA of sm_100a
// (mma.sync m8n8k4 f64; the fifth-generation tcgen05 MMA has no FP64 kind).
//
// GEMM: a CTA computes a 128 x 64 tile of C with eight warps of 32 x 32 (4 x 4 MMA tiles of
// 8 x 8 each).  K runs in slabs of 16 staged in shared memory by cp.async through a
// three-stage ring; operands are stored with rows padded to a multiple of 4 doubles plus
// 4, so that the MMA fragment loads (8 rows x 4 consecutive k, or 4 rows x 8 consecutive
// m) fall on distinct banks.  gemm_tn splits its long inner dimension into slices whose
// partial tiles a second kernel sums in slice order.
//
// Triangular inverse: one warp per column j of X = R^-1 sweeps k = j .. 0 (x_k /= r_kk,
// then x_i -= r_ik x_k for i < k), reading column k of R coalesced.  The left triangular
// solve of the block least squares inverts the diagonal blocks and runs the block back
// substitution as GEMMs, as blocked GPU triangular solvers do.
#include "dense.h"

#include <algorithm>
#include <atomic>

#include "common.h"

namespace fftsvd {
namespace dense {

namespace {

constexpr int BM = 128, BN = 64, BK = 16, kThreads = 256, kStages = 3;
constexpr int KP = BK + 4;  // row length (doubles) of a K-contiguous tile
constexpr int MP = BM + 4;  // row length of an M-contiguous tile
// A tiles: K-contiguous (Aop[m][k] = A[m lda + k], the transposed operand of gemm_tn) hold BM
// rows of KP; M-contiguous (Aop[m][k] = A[k lda + m], gemm_nn) hold BK rows of MP
constexpr int kATileK = BM * KP, kATileM = BK * MP;
constexpr int kATile = kATileK > kATileM ? kATileK : kATileM;
constexpr int kBTile = BN * KP;  // B is K-contiguous in both: Bop[k][n] = B[n ldb + k]
constexpr int kGemmSmem = kStages * (kATile + kBTile) * 8;
constexpr int kTrinvWarps = 8;

__device__ __forceinline__ void cp16(double* dst, const double* src, bool valid) {
   const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
   asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
   asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// c (8 x 8) += a (8 x 4) b (4 x 8): lane l holds a[l / 4][l % 4], b[l % 4][l / 4] and
// c[l / 4][2 (l % 4) + {0, 1}]
__device__ __forceinline__ void dmma(double (&c)[2], double a, double b) {
   asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                : "+d"(c[0]), "+d"(c[1])
                : "d"(a), "d"(b));
}

// One BM x BN tile of alpha Aop Bop + beta C over k in the slice blockIdx.z (k_slice long):
// written to C, or as a raw partial product to part[z][n][m] when part is set.  Chunks of
// two doubles are either wholly inside or wholly outside the operands (M of an
// M-contiguous A, K and the slice bounds are even), and those outside read as zero.
template <bool kContigA>
__global__ void __launch_bounds__(kThreads, 2)
    dgemm_kernel(int64_t M, int N, int64_t K, int64_t k_slice, const double* __restrict__ A, int64_t lda,
                 const double* __restrict__ B, int64_t ldb, double alpha, double beta, double* __restrict__ C,
                 int64_t ldc, double* __restrict__ part) {
   extern __shared__ __align__(16) double sm[];
   double* const As = sm;
   double* const Bs = sm + kStages * kATile;
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
   const int wm = warp & 3, wn = warp >> 2;
   const int g = lane >> 2, t = lane & 3;
   const int64_t m0 = (int64_t)blockIdx.x * BM;
   const int n0 = blockIdx.y * BN;
   const int64_t kb = (int64_t)blockIdx.z * k_slice, ke = K < kb + k_slice ? K : kb + k_slice;
   const int nk = ke > kb ? (int)((ke - kb + BK - 1) / BK) : 0;

   auto load = [&](int stage, int64_t k0) {
      double* as = As + stage * kATile;
      double* bs = Bs + stage * kBTile;
      if (kContigA) {
         for (int c = tid; c < BM * (BK / 2); c += kThreads) {
            const int row = c >> 3, kc = (c & 7) * 2;
            const int64_t m = m0 + row, k = k0 + kc;
            const bool ok = m < M && k < ke;
            cp16(as + row * KP + kc, ok ? A + m * lda + k : A, ok);
         }
      } else {
         for (int c = tid; c < BK * (BM / 2); c += kThreads) {
            const int krow = c / (BM / 2), mc = (c % (BM / 2)) * 2;
            const int64_t m = m0 + mc, k = k0 + krow;
            const bool ok = m < M && k < ke;
            cp16(as + krow * MP + mc, ok ? A + k * lda + m : A, ok);
         }
      }
      for (int c = tid; c < BN * (BK / 2); c += kThreads) {
         const int row = c >> 3, kc = (c & 7) * 2;
         const int n = n0 + row;
         const int64_t k = k0 + kc;
         const bool ok = n < N && k < ke;
         cp16(bs + row * KP + kc, ok ? B + (int64_t)n * ldb + k : B, ok);
      }
   };

   double acc[4][4][2];
#pragma unroll
   for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
   for (int s = 0; s < kStages - 1; s++) {
      if (s < nk) load(s, kb + (int64_t)s * BK);
      cp_commit();
   }
   for (int kt = 0; kt < nk; kt++) {
      cp_wait<kStages - 2>();
      __syncthreads();  // slab kt is in; every warp is done with the stage refilled next
      const int nxt = kt + kStages - 1;
      if (nxt < nk) load(nxt % kStages, kb + (int64_t)nxt * BK);
      cp_commit();
      const double* as = As + (kt % kStages) * kATile;
      const double* bs = Bs + (kt % kStages) * kBTile;
#pragma unroll
      for (int kk = 0; kk < BK; kk += 4) {
         double a[4], b[4];
#pragma unroll
         for (int i = 0; i < 4; i++) {
            const int m = wm * 32 + i * 8 + g;
            a[i] = kContigA ? as[m * KP + kk + t] : as[(kk + t) * MP + m];
         }
#pragma unroll
         for (int j = 0; j < 4; j++) b[j] = bs[(wn * 32 + j * 8 + g) * KP + kk + t];
#pragma unroll
         for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) dmma(acc[i][j], a[i], b[j]);
      }
   }
   cp_wait<0>();

#pragma unroll
   for (int i = 0; i < 4; i++)
#pragma unroll
      for (int j = 0; j < 4; j++)
#pragma unroll
         for (int e = 0; e < 2; e++) {
            const int64_t m = m0 + wm * 32 + i * 8 + g;
            const int n = n0 + wn * 32 + j * 8 + 2 * t + e;
            if (m >= M || n >= N) continue;
            if (part) {
               part[((int64_t)blockIdx.z * N + n) * M + m] = acc[i][j][e];
            } else {
               double v = alpha * acc[i][j][e];
               if (beta != 0.0) v += beta * C[(int64_t)n * ldc + m];
               C[(int64_t)n * ldc + m] = v;
            }
         }
}

// C = alpha sum_z part[z] + beta C, slices summed in order
__global__ void splitk_reduce_kernel(int M, int N, int S, const double* __restrict__ part, double alpha, double beta,
                                     double* __restrict__ C, int64_t ldc) {
   const int64_t mn = (int64_t)M * N;
   for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < mn; idx += (int64_t)gridDim.x * blockDim.x) {
      double s = 0.0;
      for (int z = 0; z < S; z++) s += part[z * mn + idx];
      const int64_t m = idx % M, n = idx / M;
      double v = alpha * s;
      if (beta != 0.0) v += beta * C[n * ldc + m];
      C[n * ldc + m] = v;
   }
}

__global__ void __launch_bounds__(kTrinvWarps * 32)
    trinv_upper_kernel(int n, const double* __restrict__ R, int64_t ldr, int64_t r_step, double* __restrict__ X,
                       int64_t ldx, int64_t x_step) {
   extern __shared__ double tsm[];
   double* const rdiag = tsm;  // reciprocals of the diagonal
   const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
   double* const x = tsm + n + warp * n;
   const double* Rb = R + blockIdx.y * r_step;
   double* Xb = X + blockIdx.y * x_step;
   for (int i = threadIdx.x; i < n; i += blockDim.x) rdiag[i] = 1.0 / Rb[(int64_t)i * ldr + i];
   __syncthreads();
   const int j = blockIdx.x * kTrinvWarps + warp;
   if (j >= n) return;
   for (int i = lane; i <= j; i += 32) x[i] = i == j ? 1.0 : 0.0;
   __syncwarp();
   for (int k = j; k >= 0; k--) {
      const double xk = x[k] * rdiag[k];
      __syncwarp();  // every lane has read x[k] before lane 0 replaces it
      const double* rk = Rb + (int64_t)k * ldr;
      for (int i = lane; i < k; i += 32) x[i] -= rk[i] * xk;
      if (lane == 0) x[k] = xk;
      __syncwarp();
   }
   for (int i = lane; i < n; i += 32) Xb[(int64_t)j * ldx + i] = i <= j ? x[i] : 0.0;
}

__global__ void add_kernel(int M, int N, const double* A, int64_t lda, const double* B, int64_t ldb, double* C,
                           int64_t ldc) {
   const int64_t mn = (int64_t)M * N;
   for (int64_t idx = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; idx < mn; idx += (int64_t)gridDim.x * blockDim.x) {
      const int64_t m = idx % M, n = idx / M;
      C[n * ldc + m] = A[n * lda + m] + B[n * ldb + m];
   }
}

int sm_count() {
   int dev = 0, sms = 0;
   FFTSVD_CUDA(cudaGetDevice(&dev));
   FFTSVD_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
   return std::max(1, sms);
}

// raises the kernels' dynamic shared-memory limits, once per device
void prepare_gemm() {
   static std::atomic<uint64_t> done{0};
   int dev = 0;
   FFTSVD_CUDA(cudaGetDevice(&dev));
   const uint64_t bit = dev < 64 ? uint64_t(1) << dev : 0;
   if (bit && (done.load(std::memory_order_acquire) & bit)) return;
   FFTSVD_CUDA(cudaFuncSetAttribute(dgemm_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem));
   FFTSVD_CUDA(cudaFuncSetAttribute(dgemm_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem));
   FFTSVD_CUDA(cudaFuncSetAttribute(trinv_upper_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (1 + kTrinvWarps) * 1024 * 8));
   done.fetch_or(bit, std::memory_order_acq_rel);
}

// slices of the inner dimension of gemm_tn: about four CTAs per SM in all, at least eight
// K slabs per slice
int64_t tn_slices(int M, int N, int64_t K, int64_t* k_slice) {
   const int64_t tiles = (int64_t)((M + BM - 1) / BM) * ((N + BN - 1) / BN);
   const int64_t ktiles = std::max<int64_t>(1, (K + BK - 1) / BK);
   const int64_t target = 4 * (int64_t)sm_count();
   int64_t S = std::max<int64_t>(1, (target + tiles - 1) / tiles);
   S = std::min(S, std::max<int64_t>(1, ktiles / 8));
   const int64_t per = (ktiles + S - 1) / S;
   *k_slice = per * BK;
   return (ktiles + per - 1) / per;
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

}  // namespace

int64_t gemm_tn_work(int M, int N, int64_t K) {
   int64_t ks = 0;
   const int64_t S = tn_slices(M, N, K, &ks);
   return S > 1 ? S * M * N : 0;
}

void gemm_tn(int M, int N, int64_t K, double alpha, const double* A, int64_t lda, const double* B, int64_t ldb,
             double beta, double* C, int64_t ldc, double* work, cudaStream_t s) {
   if (M <= 0 || N <= 0) return;
   FFTSVD_REQUIRE(K % 2 == 0 && lda % 2 == 0 && ldb % 2 == 0 && aligned16(A) && aligned16(B),
                  "gemm_tn: K, lda and ldb must be even and the operands 16-byte aligned");
   prepare_gemm();
   int64_t ks = 0;
   const int64_t S = tn_slices(M, N, K, &ks);
   const dim3 grid((M + BM - 1) / BM, (N + BN - 1) / BN, (unsigned)S);
   dgemm_kernel<true><<<grid, kThreads, kGemmSmem, s>>>(M, N, K, ks, A, lda, B, ldb, alpha, beta, C, ldc,
                                                       S > 1 ? work : nullptr);
   FFTSVD_CHECK_LAUNCH();
   if (S > 1) {
      const int64_t mn = (int64_t)M * N;
      const int blocks = (int)std::min<int64_t>((mn + 255) / 256, 8 * (int64_t)sm_count());
      splitk_reduce_kernel<<<blocks, 256, 0, s>>>(M, N, (int)S, work, alpha, beta, C, ldc);
      FFTSVD_CHECK_LAUNCH();
   }
}

void gemm_nn(int64_t M, int N, int K, double alpha, const double* A, int64_t lda, const double* B, int64_t ldb,
             double beta, double* C, int64_t ldc, cudaStream_t s) {
   if (M <= 0 || N <= 0) return;
   FFTSVD_REQUIRE(M % 2 == 0 && K % 2 == 0 && lda % 2 == 0 && ldb % 2 == 0 && aligned16(A) && aligned16(B),
                  "gemm_nn: M, K, lda and ldb must be even and the operands 16-byte aligned");
   prepare_gemm();
   const dim3 grid((unsigned)((M + BM - 1) / BM), (N + BN - 1) / BN, 1);
   dgemm_kernel<false><<<grid, kThreads, kGemmSmem, s>>>(M, N, K, std::max(K, 1), A, lda, B, ldb, alpha, beta, C,
                                                        ldc, nullptr);
   FFTSVD_CHECK_LAUNCH();
}

void trinv_upper(int n, int count, const double* R, int64_t ldr, int64_t r_step, double* X, int64_t ldx,
                 int64_t x_step, cudaStream_t s) {
   if (n <= 0 || count <= 0) return;
   FFTSVD_REQUIRE(n <= 1024, "trinv_upper: at most 1024 rows");
   prepare_gemm();
   const dim3 grid((n + kTrinvWarps - 1) / kTrinvWarps, count);
   trinv_upper_kernel<<<grid, kTrinvWarps * 32, (size_t)(1 + kTrinvWarps) * n * 8, s>>>(n, R, ldr, r_step, X, ldx,
                                                                                       x_step);
   FFTSVD_CHECK_LAUNCH();
}

void trsm_upper_left(int rows, int N, int bs, const double* R, int64_t ldr, double* Y, double* dinv, double* Out,
                     cudaStream_t s) {
   if (rows <= 0 || N <= 0) return;
   FFTSVD_REQUIRE(bs > 0 && bs % 2 == 0 && rows % bs == 0, "trsm_upper_left: rows must be a multiple of an even bs");
   const int nb = rows / bs;
   trinv_upper(bs, nb, R, ldr, (int64_t)bs * ldr + bs, dinv, bs, (int64_t)bs * bs, s);
   for (int b = nb - 1; b >= 0; b--) {
      const int64_t off = (int64_t)b * bs;
      gemm_nn(bs, N, bs, 1.0, dinv + off * bs, bs, Y + off, rows, 0.0, Out + off, rows, s);
      if (b > 0) gemm_nn(off, N, bs, -1.0, R + off * ldr, ldr, Out + off, rows, 1.0, Y, rows, s);
   }
}

void add(int M, int N, const double* A, int64_t lda, const double* B, int64_t ldb, double* C, int64_t ldc,
         cudaStream_t s) {
   const int64_t mn = (int64_t)M * N;
   if (mn <= 0) return;
   const int blocks = (int)std::min<int64_t>((mn + 255) / 256, 8 * (int64_t)sm_count());
   add_kernel<<<blocks, 256, 0, s>>>(M, N, A, lda, B, ldb, C, ldc);
   FFTSVD_CHECK_LAUNCH();
}

}  // namespace dense
}  // namespace fftsvd
