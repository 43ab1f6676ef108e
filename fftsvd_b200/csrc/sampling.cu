// Panel integrals of the operator setup on the GPU (FP64): the near-field blocks
// (Cube_fill_D, Cube.c:715-793) and the sampled matrices of the low-rank bases and
// of the equivalent-density fits (Cube.c:1104-1281, 795-1002).  The host describes
// each dense block of (points x panels) integrals it needs (setup.h, IntegralBatch);
// one launch evaluates every block of a batch with the same host/device integral
// routines as the host path (integrals.h: FlatIntegration_oneoverr and the Yukawa
// edge integrals, FlatIntegration.c:295-429, 882-949).
//
// Work split: the host cuts every block into tiles of at most kTilePairs consecutive
// (point, panel) pairs in row-major order; one CUDA block per tile, one thread per pair.
// A thread's pairs share the point and walk consecutive panels, so the panel records of
// a tile come through L1/L2 once per tile.  The integrals are FP64 ALU work (the Yukawa
// integral evaluates about a hundred transcendental functions), not memory traffic.
#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <string>
#include <vector>

#include "common.h"
#include "integrals.h"
#include "fill_later.h"
#include "setup.h"

namespace fftsvd {
namespace setup {
namespace {

constexpr int kTilePairs = 128;

struct PairTile {
   int32_t block;  // index into the block list
   int32_t first;  // first pair of the tile within its block (row-major)
};

struct DevBlock {
   int32_t npts, npan;
   int64_t pt_off, pan_off, out_s, out_d;
   int32_t ld_s, ld_d;
};

// status[0] counts Yukawa integrals whose angular subdivision did not terminate
__global__ void __launch_bounds__(kTilePairs) panel_integrals_kernel(
    const PairTile* __restrict__ tiles, const DevBlock* __restrict__ blocks, const double* __restrict__ pts,
    const int32_t* __restrict__ pan_idx, const FlatPanel* __restrict__ panels, int yukawa, double kappa,
    double* __restrict__ out, unsigned int* __restrict__ status) {
   const PairTile t = tiles[blockIdx.x];
   const DevBlock b = blocks[t.block];
   const int64_t pair = (int64_t)t.first + threadIdx.x;
   if (pair >= (int64_t)b.npts * b.npan) return;
   const int i = (int)(pair / b.npan), k = (int)(pair % b.npan);
   const double* p = pts + 3 * (b.pt_off + i);
   const double point[3] = {p[0], p[1], p[2]};
   const FlatPanel& P = panels[pan_idx[b.pan_off + k]];
   double s = 0.0, d = 0.0;
   if (yukawa) {
      if (!yukawa_panel(point, P, kappa, &s, &d)) atomicAdd(status, 1u);
   } else {
      laplace_panel(point, P, &s, &d);
   }
   out[b.out_s + (int64_t)i * b.ld_s + k] = s;
   out[b.out_d + (int64_t)i * b.ld_d + k] = d;
}

void cuda_check(cudaError_t e, const char* what) {
   if (e != cudaSuccess) throw DeviceError(FFTSVD_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
struct Buf {  // device allocation owned by the evaluator (freed on scope exit)
   T* p = nullptr;
   size_t n = 0;
   void alloc(size_t count) {
      release();
      n = count;
      if (count) {
         g_device_allocs.fetch_add(1, std::memory_order_relaxed);
         cuda_check(cudaMalloc(&p, count * sizeof(T)), "cudaMalloc (setup integrals)");
      }
   }
   void upload(const T* h, size_t count, cudaStream_t s) {
      alloc(count);
      if (count) cuda_check(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s), "copy to device");
   }
   // at least count elements, reallocated only to grow (the contents are not kept)
   void reserve(size_t count) {
      if (count > n) alloc(count);
   }
   void upload_grow(const T* h, size_t count, cudaStream_t s) {
      reserve(count);
      if (count) cuda_check(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s), "copy to device");
   }
   void release() {
      if (p) cudaFree(p);
      p = nullptr;
      n = 0;
   }
   ~Buf() { release(); }
};

struct DeviceSampler {
   cudaStream_t stream = nullptr;
   Buf<FlatPanel> panels;
   const FlatPanel* host_panels = nullptr;  // the panel list the device copy was made from
   size_t host_count = 0;
   // Host copy of the last batch's output, grown to the largest batch and reused by the
   // setup's later batches.  Pageable, not pinned: page-locking a buffer of several GB
   // (3.6 GB of samples at 327 680 panels) took seconds, far longer than the copy itself.
   std::vector<double, FillLater<double>> host_out;
   // device buffers of the batches, grown to the largest and reused (a setup's batches
   // would otherwise allocate and free several GB each)
   Buf<DevBlock> d_blocks;
   Buf<PairTile> d_tiles;
   Buf<double> d_pts, d_out;
   Buf<int32_t> d_pan;
   Buf<unsigned int> d_status;
   ~DeviceSampler() {
      if (stream) cudaStreamDestroy(stream);
   }

   double* host_output(size_t elems) {
      if (elems > host_out.size()) {
         host_out = std::vector<double, FillLater<double>>();  // the old contents are not needed
         host_out.resize(elems);                               // every entry is copied in below
         // one write per 4 KB page on all host threads: the copy then lands in mapped pages,
         // instead of taking a fresh buffer's page faults one at a time (1.2 s for 3.6 GB)
         double* p = host_out.data();
         const int64_t n = (int64_t)elems;
#pragma omp parallel for schedule(static)
         for (int64_t i = 0; i < n; i += 512) p[i] = 0.0;
      }
      return host_out.data();
   }

   const double* operator()(const Kernel& kern, const std::vector<FlatPanel>& pl, const IntegralBatch& B) {
      if (B.out_elems == 0) return nullptr;
      if (!stream) cuda_check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
      double* out = host_output((size_t)B.out_elems);
      if (B.blocks.empty()) {
         std::fill(out, out + B.out_elems, 0.0);
         return out;
      }
      if (host_panels != pl.data() || host_count != pl.size()) {
         panels.upload(pl.data(), pl.size(), stream);
         host_panels = pl.data();
         host_count = pl.size();
      }
      // every index the kernel forms is checked here, before the launch
      const int64_t npts = (int64_t)B.points.size() / 3, npan_idx = (int64_t)B.panels.size();
      for (int32_t v : B.panels)
         if (v < 0 || (size_t)v >= pl.size()) throw std::runtime_error("setup integrals: panel index out of range");
      std::vector<DevBlock> blocks(B.blocks.size());
      std::vector<PairTile> tiles;
      for (size_t bi = 0; bi < B.blocks.size(); bi++) {
         const IntegralBlock& b = B.blocks[bi];
         const int64_t pairs = (int64_t)b.npts * b.npan;
         if (b.npts < 0 || b.npan < 0 || b.pt_off < 0 || b.pt_off + b.npts > npts || b.pan_off < 0 ||
             b.pan_off + b.npan > npan_idx)
            throw std::runtime_error("setup integrals: block outside the point or panel lists");
         if (pairs > 0) {
            const int64_t last_s = b.out_s + (int64_t)(b.npts - 1) * b.ld_s + b.npan - 1;
            const int64_t last_d = b.out_d + (int64_t)(b.npts - 1) * b.ld_d + b.npan - 1;
            if (b.out_s < 0 || b.out_d < 0 || b.ld_s < b.npan || b.ld_d < b.npan || last_s >= B.out_elems ||
                last_d >= B.out_elems)
               throw std::runtime_error("setup integrals: block outside the output");
            if (pairs > (int64_t)INT32_MAX) throw std::runtime_error("setup integrals: block too large");
         }
         blocks[bi] = DevBlock{b.npts, b.npan, b.pt_off, b.pan_off, b.out_s, b.out_d, b.ld_s, b.ld_d};
         for (int64_t f = 0; f < pairs; f += kTilePairs) tiles.push_back(PairTile{(int32_t)bi, (int32_t)f});
      }
      if (tiles.empty()) {
         std::fill(out, out + B.out_elems, 0.0);
         return out;
      }
      d_blocks.upload_grow(blocks.data(), blocks.size(), stream);
      d_tiles.upload_grow(tiles.data(), tiles.size(), stream);
      d_pts.upload_grow(B.points.data(), B.points.size(), stream);
      d_pan.upload_grow(B.panels.data(), B.panels.size(), stream);
      d_out.reserve((size_t)B.out_elems);
      // output entries no block covers (none in the batches built by setup.cpp) read as zero
      cuda_check(cudaMemsetAsync(d_out.p, 0, sizeof(double) * (size_t)B.out_elems, stream), "memset");
      d_status.reserve(1);
      cuda_check(cudaMemsetAsync(d_status.p, 0, sizeof(unsigned int), stream), "memset");
      // grid x is limited to 2^31 - 1 blocks; split longer tile lists into launches
      const size_t max_grid = 1u << 30;
      for (size_t t0 = 0; t0 < tiles.size(); t0 += max_grid) {
         const unsigned int nb = (unsigned int)std::min(max_grid, tiles.size() - t0);
         panel_integrals_kernel<<<nb, kTilePairs, 0, stream>>>(d_tiles.p + t0, d_blocks.p, d_pts.p, d_pan.p, panels.p,
                                                              kern.yukawa ? 1 : 0, kern.kappa, d_out.p, d_status.p);
         g_kernel_launches.fetch_add(1, std::memory_order_relaxed);
         cuda_check(cudaGetLastError(), "panel_integrals_kernel launch");
      }
      unsigned int bad = 0;
      cuda_check(cudaMemcpyAsync(out, d_out.p, sizeof(double) * (size_t)B.out_elems, cudaMemcpyDeviceToHost, stream),
                 "copy to host");
      cuda_check(cudaMemcpyAsync(&bad, d_status.p, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream),
                 "copy to host");
      cuda_check(cudaStreamSynchronize(stream), "setup integrals");
      if (bad) throw std::runtime_error("Yukawa panel integration did not converge");
      return out;
   }
};

}  // namespace

BatchEvaluator device_evaluator() {
   int ndev = 0;
   if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
      throw DeviceError(FFTSVD_ERR_NO_DEVICE, "no CUDA device visible");
   auto sampler = std::make_shared<DeviceSampler>();
   return [sampler](const Kernel& k, const std::vector<FlatPanel>& pl, const IntegralBatch& b) {
      return (*sampler)(k, pl, b);
   };
}

}  // namespace setup
}  // namespace fftsvd
