// Blackwell (sm_100a) fifth-generation tensor-core primitives in inline PTX:
// tensor-memory (TMEM) allocation, UMMA shared-memory and instruction descriptors,
// kind::tf32 MMA issue, commit to an mbarrier with a bounded wait, and TMEM loads.
//
// Operand layout (K-major, no swizzle).  An operand of R rows (the M rows of A or the
// N rows of B) and 8 K elements (32 bytes of TF32, one MMA K-step) is stored as two
// blocks of 16 bytes per row, the first four K elements of every row, then the last
// four: byte (row, k) = (k / 4) * R * 16 + row * 16 + (k % 4) * 4.  In the descriptor's
// terms the 8-row core matrices are 128 contiguous bytes, 8-row groups are 128 bytes
// apart (stride byte offset) and the two K halves R * 16 bytes apart (leading byte
// offset).  Consecutive K-steps follow each other, 2 * R * 16 bytes apart.
#pragma once

#include <cstdint>

namespace fftsvd {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor of a K-major operand without swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lead_bytes, uint32_t stride_bytes) {
   uint64_t d = 0;
   d |= (uint64_t)((saddr >> 4) & 0x3FFFu);              // start address, 16-byte units
   d |= (uint64_t)((lead_bytes >> 4) & 0x3FFFu) << 16;   // leading byte offset (K direction)
   d |= (uint64_t)((stride_bytes >> 4) & 0x3FFFu) << 32; // stride byte offset (8-row groups)
   d |= (uint64_t)1 << 46;                               // descriptor version of sm_100
   return d;                                             // base offset 0, no swizzle
}

// instruction descriptor of kind::tf32 with FP32 accumulation, A and B K-major, M x N
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N) {
   return (1u << 4)                       // accumulator format F32
          | (2u << 7)                     // A format TF32
          | (2u << 10)                    // B format TF32
          | ((uint32_t)(N >> 3) << 17)    // N / 8
          | ((uint32_t)(M >> 4) << 24);   // M / 16
}

// D[tmem] (+)= A * B^T, one thread issues
__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
   asm volatile(
       "{\n\t.reg .pred p;\n\t"
       "setp.ne.b32 p, %4, 0;\n\t"
       "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
       "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0)
       : "memory");
}

// the mbarrier receives one arrival when every MMA this thread issued before has completed
__device__ __forceinline__ void commit(uint32_t mbar) {
   asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
   asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}

// Waits for the phase with the given parity to complete, polling at most max_polls
// times; returns false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint32_t max_polls) {
   for (uint32_t i = 0; i < max_polls; i++) {
      uint32_t done = 0;
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}\n"
          : "=r"(done)
          : "r"(mbar), "r"(parity)
          : "memory");
      if (done) return true;
   }
   return false;
}

// TMEM allocation of ncols columns (a power of two >= 32) by one whole warp; the
// address is written to shared memory at slot
__device__ __forceinline__ void tmem_alloc(uint32_t slot, uint32_t ncols) {
   asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(slot), "r"(ncols)
                : "memory");
   asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
   asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Eight consecutive 32-bit accumulator columns of this thread's TMEM lane: warp w of the
// CTA reads lanes 32 w .. 32 w + 31 (taddr must carry that lane base)
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float (&v)[8]) {
   uint32_t r[8];
   asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                : "r"(taddr)
                : "memory");
   asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
   for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

// Split of an FP32 value into a TF32 head (the nearest TF32 value) and the FP32 tail, for
// the three-product TF32 scheme (Ootomo and Yokota, 2022): a b ~ ah bh + ah bl + al bh.
__device__ __forceinline__ float round_tf32(float x) {
   uint32_t h;
   asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
   return __uint_as_float(h);
}
__device__ __forceinline__ void split_tf32(float x, float& hi, float& lo) {
   hi = round_tf32(x);
   lo = round_tf32(x - hi);
}

}  // namespace tc
}  // namespace fftsvd
