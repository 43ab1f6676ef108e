// Charge <-> panel interaction kernels (FP64):
//   right-hand side          SurfaceOperator_makeRHS                 SurfaceOperator.c:291-321
//   reaction potentials      SurfaceOperator_calculateReactionPotentials, direct branch
//                                                                     SurfaceOperator.c:364-396
//   energy                   FFTSVDsalt.c:167-170
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "nbody.h"
#include "surface.h"

namespace fftsvd {

void set_geometry(Surface& S, int num_panels, const double* vertices, const int32_t* phi_row, const int32_t* dphi_row) {
   FFTSVD_REQUIRE(num_panels > 0 && vertices && phi_row && dphi_row, "bad panel geometry");
   auto g = std::make_shared<PanelGeometry>();
   g->num_panels = num_panels;
   g->host.resize(num_panels);
   for (int i = 0; i < num_panels; i++) {
      const double* v = vertices + 9 * (size_t)i;
      make_flat_panel(g->host[i], v, v + 3, v + 6);
      FFTSVD_REQUIRE(g->host[i].area > 0.0, "degenerate panel " + std::to_string(i));
   }
   for (int i = 0; i < num_panels; i++)
      FFTSVD_REQUIRE(phi_row[i] >= 0 && phi_row[i] < S.n && dphi_row[i] >= 0 && dphi_row[i] < S.n,
                     "panel row out of range");
   g->panels.upload(g->host);
   g->phi_row.upload(phi_row, num_panels);
   g->dphi_row.upload(dphi_row, num_panels);
   S.geom = g;
}

void set_charges(Surface& S, int num_charges, const double* pos, const double* q) {
   FFTSVD_REQUIRE(num_charges >= 0, "negative charge count");
   S.num_charges = num_charges;
   if (num_charges == 0) return;
   FFTSVD_REQUIRE(pos && q, "null charge arrays");
   for (int i = 0; i < num_charges; i++)
      FFTSVD_REQUIRE(std::isfinite(q[i]) && std::isfinite(pos[3 * i]) && std::isfinite(pos[3 * i + 1]) &&
                         std::isfinite(pos[3 * i + 2]),
                     "non-finite charge input");
   S.charge_pos.upload(pos, 3 * (size_t)num_charges);
   S.charge_q.upload(q, num_charges);
   S.charge_q_host.assign(q, q + num_charges);
}

constexpr int kRhsThreads = 256;
constexpr int kRhsTile = 256;

// Target centroids of the right-hand-side kernel: the library's flat panels, or
// plain xyz triples (the drop-in reads them from the caller's reference panels).
struct PanelTargets {
   const FlatPanel* __restrict__ p;
   __device__ void get(int i, double c[3]) const {
      c[0] = p[i].centroid[0];
      c[1] = p[i].centroid[1];
      c[2] = p[i].centroid[2];
   }
};
struct PointTargets {
   const double* __restrict__ xyz;
   __device__ void get(int i, double c[3]) const {
      c[0] = xyz[3 * i];
      c[1] = xyz[3 * i + 1];
      c[2] = xyz[3 * i + 2];
   }
};

// One thread per target; charges streamed through shared memory in order, so each
// target accumulates over charges in the reference's order (charge-major loop,
// SurfaceOperator.c:298-312), and rhs[row[i]] += the sum.
// With gptr, blockIdx.y is a charge group: charges [gptr[g], gptr[g+1]) and
// output column rhs + g * col.
template <typename Targets>
__global__ void __launch_bounds__(kRhsThreads) rhs_kernel(int np, Targets targets, const int32_t* __restrict__ row,
                                                          int nq, const double* __restrict__ qpos,
                                                          const double* __restrict__ q, double* __restrict__ rhs,
                                                          const int32_t* __restrict__ gptr, int64_t col) {
   __shared__ double4 tile[kRhsTile];
   if (gptr) {
      const int q0 = gptr[blockIdx.y];
      nq = gptr[blockIdx.y + 1] - q0;
      qpos += 3 * (int64_t)q0;
      q += q0;
      rhs += blockIdx.y * col;
   }
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   double c[3] = {0, 0, 0};
   if (i < np) targets.get(i, c);
   double acc = 0.0;
   for (int base = 0; base < nq; base += kRhsTile) {
      const int cnt = min(kRhsTile, nq - base);
      __syncthreads();
      for (int j = threadIdx.x; j < cnt; j += blockDim.x)
         tile[j] = make_double4(qpos[3 * (base + j)], qpos[3 * (base + j) + 1], qpos[3 * (base + j) + 2], q[base + j]);
      __syncthreads();
      if (i < np)
         for (int j = 0; j < cnt; j++) {
            const double4 t = tile[j];
            if (t.w == 0.0) continue;
            const double dx = t.x - c[0], dy = t.y - c[1], dz = t.z - c[2];
            acc += t.w / sqrt(dx * dx + dy * dy + dz * dz);
         }
   }
   if (i < np) rhs[row[i]] += acc;
}

void rhs_points_device(int nt, const double* centroids, const int32_t* rows, int nq, const double* qpos,
                       const double* q, double* rhs, cudaStream_t stream) {
   FFTSVD_REQUIRE(nt >= 0 && nq >= 0, "negative target or charge count");
   if (nt == 0) return;
   rhs_kernel<<<(nt + kRhsThreads - 1) / kRhsThreads, kRhsThreads, 0, stream>>>(
       nt, PointTargets{centroids}, rows, nq, qpos, q, rhs, nullptr, 0);
   FFTSVD_CHECK_LAUNCH();
}

constexpr int kReactThreads = 128;
constexpr int kReactPanelTile = 16;
constexpr int kReactChunks = 64;

// Block (charge chunk, panel chunk): each thread owns one charge and sums the
// panel integrals of its panel chunk; panels staged through shared memory.
// With gptr, blockIdx.z is a charge group: its charges [gptr[g], gptr[g+1])
// against its own solution column sol + g * col (partial still indexed by the
// global charge number).
__global__ void __launch_bounds__(kReactThreads) reaction_partial_kernel(
    int np, const FlatPanel* __restrict__ panels, const int32_t* __restrict__ phi_row,
    const int32_t* __restrict__ dphi_row, const double* __restrict__ sol, int nq, const double* __restrict__ qpos,
    double* __restrict__ partial, const int32_t* __restrict__ gptr, int64_t col) {
   __shared__ FlatPanel tile[kReactPanelTile];
   __shared__ double2 dens[kReactPanelTile];
   const int nq_all = nq;
   int j = blockIdx.x * blockDim.x + threadIdx.x;
   if (gptr) {
      const int q0 = gptr[blockIdx.z], q1 = gptr[blockIdx.z + 1];
      j = q0 + j < q1 ? q0 + j : nq_all;  // past the group: idle
      sol += blockIdx.z * col;
   }
   const int per = (np + gridDim.y - 1) / gridDim.y;
   const int p0 = blockIdx.y * per, p1 = min(np, p0 + per);
   double pt[3] = {0, 0, 0};
   if (j < nq) { pt[0] = qpos[3 * j]; pt[1] = qpos[3 * j + 1]; pt[2] = qpos[3 * j + 2]; }
   double acc = 0.0;
   for (int base = p0; base < p1; base += kReactPanelTile) {
      const int cnt = min(kReactPanelTile, p1 - base);
      __syncthreads();
      {
         const double* src = reinterpret_cast<const double*>(panels + base);
         double* dst = reinterpret_cast<double*>(tile);
         const int words = cnt * (int)(sizeof(FlatPanel) / sizeof(double));
         for (int w = threadIdx.x; w < words; w += blockDim.x) dst[w] = src[w];
         for (int k = threadIdx.x; k < cnt; k += blockDim.x)
            dens[k] = make_double2(sol[phi_row[base + k]], sol[dphi_row[base + k]]);
      }
      __syncthreads();
      if (j < nq)
         for (int k = 0; k < cnt; k++) {
            double s, d;
            laplace_panel(pt, tile[k], &s, &d);
            const double2 dn = dens[k];
            acc += dn.y * s - dn.x * d;
            if (tile[k].centroid[0] == pt[0] && tile[k].centroid[1] == pt[1] && tile[k].centroid[2] == pt[2])
               acc -= 4.0 * M_PI * dn.x;
         }
   }
   if (j < nq) partial[(size_t)blockIdx.y * nq_all + j] = acc;
}

__global__ void reaction_reduce_kernel(int nq, int chunks, const double* __restrict__ partial, double* __restrict__ phi) {
   const int j = blockIdx.x * blockDim.x + threadIdx.x;
   if (j >= nq) return;
   double s = 0.0;
   for (int c = 0; c < chunks; c++) s += partial[(size_t)c * nq + j];
   phi[j] = s;
}

void rhs_device(Surface& S, double* rhs) {
   FFTSVD_REQUIRE(S.geom, "surface has no panel geometry");
   FFTSVD_CUDA(cudaMemsetAsync(rhs, 0, sizeof(double) * S.n, S.stream));
   const int np = S.geom->num_panels;
   rhs_kernel<<<(np + kRhsThreads - 1) / kRhsThreads, kRhsThreads, 0, S.stream>>>(
       np, PanelTargets{S.geom->panels.get()}, S.geom->phi_row.get(), S.num_charges, S.charge_pos.get(),
       S.charge_q.get(), rhs, nullptr, 0);
   FFTSVD_CHECK_LAUNCH();
}

void reaction_device(Surface& S, const double* sol, double* phi) {
   FFTSVD_REQUIRE(S.geom, "surface has no panel geometry");
   const int nq = S.num_charges, np = S.geom->num_panels;
   if (nq == 0) return;
   const int chunks = std::max(1, std::min(kReactChunks, (np + kReactPanelTile - 1) / kReactPanelTile));
   double* const partial = S.work_buf(Surface::kWorkReact, (size_t)chunks * nq);
   dim3 grid((nq + kReactThreads - 1) / kReactThreads, chunks);
   reaction_partial_kernel<<<grid, kReactThreads, 0, S.stream>>>(np, S.geom->panels.get(), S.geom->phi_row.get(),
                                                                 S.geom->dphi_row.get(), sol, nq,
                                                                 S.charge_pos.get(), partial, nullptr, 0);
   FFTSVD_CHECK_LAUNCH();
   reaction_reduce_kernel<<<(nq + 255) / 256, 256, 0, S.stream>>>(nq, chunks, partial, phi);
   FFTSVD_CHECK_LAUNCH();
   FFTSVD_CUDA(cudaStreamSynchronize(S.stream));
}

void reaction_points_device(int np, const FlatPanel* panels, const int32_t* phi_row, const int32_t* dphi_row,
                            const double* dens, int nq, const double* qpos, double* phi, cudaStream_t stream) {
   FFTSVD_REQUIRE(np >= 0 && nq >= 0, "negative panel or point count");
   if (nq == 0) return;
   if (np == 0) {
      FFTSVD_CUDA(cudaMemsetAsync(phi, 0, sizeof(double) * nq, stream));
      FFTSVD_CUDA(cudaStreamSynchronize(stream));
      return;
   }
   const int chunks = std::max(1, std::min(kReactChunks, (np + kReactPanelTile - 1) / kReactPanelTile));
   DevBuf<double> partial((size_t)chunks * nq);
   dim3 grid((nq + kReactThreads - 1) / kReactThreads, chunks);
   reaction_partial_kernel<<<grid, kReactThreads, 0, stream>>>(np, panels, phi_row, dphi_row, dens, nq, qpos,
                                                               partial.get(), nullptr, 0);
   FFTSVD_CHECK_LAUNCH();
   reaction_reduce_kernel<<<(nq + 255) / 256, 256, 0, stream>>>(nq, chunks, partial.get(), phi);
   FFTSVD_CHECK_LAUNCH();
   FFTSVD_CUDA(cudaStreamSynchronize(stream));
}

double energy_device(Surface& S, const double* phi) {
   std::vector<double> h(S.num_charges);
   if (S.num_charges == 0) return 0.0;
   FFTSVD_CUDA(cudaMemcpyAsync(h.data(), phi, sizeof(double) * S.num_charges, cudaMemcpyDeviceToHost, S.stream));
   FFTSVD_CUDA(cudaStreamSynchronize(S.stream));
   double e = 0.0;
   for (int c = 0; c < S.num_charges; c++) e += 0.5 * S.charge_q_host[c] * h[c];
   return e * 332.112 / S.eps_in;
}

// Host group boundaries: group g is charges [gptr[g], gptr[g+1]), increasing, within the charge list.
static void check_groups(const Surface& S, int ngroups, const int32_t* gptr, int* max_size) {
   FFTSVD_REQUIRE(ngroups > 0 && ngroups <= 65535 && gptr, "charge groups");
   FFTSVD_REQUIRE(gptr[0] >= 0 && gptr[ngroups] <= S.num_charges, "charge group outside the charge list");
   *max_size = 0;
   for (int g = 0; g < ngroups; g++) {
      FFTSVD_REQUIRE(gptr[g + 1] >= gptr[g], "charge group boundaries must not decrease");
      *max_size = std::max(*max_size, gptr[g + 1] - gptr[g]);
   }
}

void rhs_groups_device(Surface& S, int ngroups, const int32_t* gptr_host, double* rhs) {
   FFTSVD_REQUIRE(S.geom, "surface has no panel geometry");
   int maxg = 0;
   check_groups(S, ngroups, gptr_host, &maxg);
   DevBuf<int32_t> gptr;
   gptr.upload(gptr_host, ngroups + 1);
   FFTSVD_CUDA(cudaMemsetAsync(rhs, 0, sizeof(double) * S.n * ngroups, S.stream));
   const int np = S.geom->num_panels;
   rhs_kernel<<<dim3((np + kRhsThreads - 1) / kRhsThreads, ngroups), kRhsThreads, 0, S.stream>>>(
       np, PanelTargets{S.geom->panels.get()}, S.geom->phi_row.get(), 0, S.charge_pos.get(), S.charge_q.get(), rhs,
       gptr.get(), S.n);
   FFTSVD_CHECK_LAUNCH();
   FFTSVD_CUDA(cudaStreamSynchronize(S.stream));
}

void group_energies_device(Surface& S, int ngroups, const int32_t* gptr_host, const double* sol, double* energies) {
   FFTSVD_REQUIRE(S.geom, "surface has no panel geometry");
   int maxg = 0;
   check_groups(S, ngroups, gptr_host, &maxg);
   const int nq = S.num_charges, np = S.geom->num_panels;
   for (int g = 0; g < ngroups; g++) energies[g] = 0.0;
   if (nq == 0 || maxg == 0) return;
   DevBuf<int32_t> gptr;
   gptr.upload(gptr_host, ngroups + 1);
   const int chunks = std::max(1, std::min(kReactChunks, (np + kReactPanelTile - 1) / kReactPanelTile));
   DevBuf<double> partial((size_t)chunks * nq), phi(nq);
   partial.zero(S.stream);
   dim3 grid((maxg + kReactThreads - 1) / kReactThreads, chunks, ngroups);
   reaction_partial_kernel<<<grid, kReactThreads, 0, S.stream>>>(np, S.geom->panels.get(), S.geom->phi_row.get(),
                                                                 S.geom->dphi_row.get(), sol, nq, S.charge_pos.get(),
                                                                 partial.get(), gptr.get(), S.n);
   FFTSVD_CHECK_LAUNCH();
   reaction_reduce_kernel<<<(nq + 255) / 256, 256, 0, S.stream>>>(nq, chunks, partial.get(), phi.get());
   FFTSVD_CHECK_LAUNCH();
   std::vector<double> h(nq);
   FFTSVD_CUDA(cudaMemcpyAsync(h.data(), phi.get(), sizeof(double) * nq, cudaMemcpyDeviceToHost, S.stream));
   FFTSVD_CUDA(cudaStreamSynchronize(S.stream));
   for (int g = 0; g < ngroups; g++) {
      double e = 0.0;
      for (int c = gptr_host[g]; c < gptr_host[g + 1]; c++) e += 0.5 * S.charge_q_host[c] * h[c];
      energies[g] = e * 332.112 / S.eps_in;
   }
}

}  // namespace fftsvd

using namespace fftsvd;

extern "C" {

int fftsvd_b200_set_geometry(fftsvd_surface* s, int32_t num_panels, const double* vertices, const int32_t* phi_row,
                             const int32_t* dphi_row) {
   if (!s) return FFTSVD_ERR_ARGUMENT;
   try {
      set_geometry(s->s, num_panels, vertices, phi_row, dphi_row);
      return FFTSVD_OK;
   } catch (const Error& e) {
      set_last_error(e.what());
      return e.code;
   }
}

int fftsvd_b200_rhs(fftsvd_surface* s, double* rhs) {
   if (!s || !rhs) return FFTSVD_ERR_ARGUMENT;
   try {
      Surface& S = s->s;
      rhs_device(S, S.t2.get());
      FFTSVD_CUDA(cudaMemcpyAsync(rhs, S.t2.get(), sizeof(double) * S.n, cudaMemcpyDeviceToHost, S.stream));
      FFTSVD_CUDA(cudaStreamSynchronize(S.stream));
      return FFTSVD_OK;
   } catch (const Error& e) {
      set_last_error(e.what());
      return e.code;
   }
}

int fftsvd_b200_rhs_device(fftsvd_surface* s, double* rhs) {
   if (!s || !rhs) return FFTSVD_ERR_ARGUMENT;
   try {
      rhs_device(s->s, rhs);
      return FFTSVD_OK;
   } catch (const Error& e) {
      set_last_error(e.what());
      return e.code;
   }
}

int fftsvd_b200_reaction_potentials(fftsvd_surface* s, const double* sol, double* phi) {
   if (!s || !sol || !phi) return FFTSVD_ERR_ARGUMENT;
   try {
      Surface& S = s->s;
      if (S.num_charges == 0) return FFTSVD_OK;
      DevBuf<double> dsol, dphi(S.num_charges);
      dsol.upload(sol, S.n);
      reaction_device(S, dsol.get(), dphi.get());
      FFTSVD_CUDA(cudaMemcpy(phi, dphi.get(), sizeof(double) * S.num_charges, cudaMemcpyDeviceToHost));
      return FFTSVD_OK;
   } catch (const Error& e) {
      set_last_error(e.what());
      return e.code;
   }
}

int fftsvd_b200_reaction_potentials_device(fftsvd_surface* s, const double* sol, double* phi) {
   if (!s || !sol || !phi) return FFTSVD_ERR_ARGUMENT;
   try {
      reaction_device(s->s, sol, phi);
      return FFTSVD_OK;
   } catch (const Error& e) {
      set_last_error(e.what());
      return e.code;
   }
}

}  // extern "C"

namespace fftsvd {

// Scratch of fftsvd_b200_reaction_potentials_noalloc: the per-chunk partial
// sums of the collection, at most kNoAllocScratchDoubles doubles (4 MiB).
// Every GPU that loads this library holds one copy until the process exits.
constexpr size_t kNoAllocScratchDoubles = 524288;
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

// Device address of the scratch array per device ordinal, looked up once per
// device with that device current.  In host code the array's name is only a
// host-side stand-in, so kernels are always given this looked-up address.
static std::mutex g_noalloc_mutex;
static double* g_noalloc_addr[128] = {nullptr};

static double* noalloc_scratch(int device) {
   FFTSVD_REQUIRE(device >= 0 && device < 128, "device ordinal out of range");
   std::lock_guard<std::mutex> lock(g_noalloc_mutex);
   if (!g_noalloc_addr[device]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
         throw Error(FFTSVD_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
      g_noalloc_addr[device] = static_cast<double*>(p);
   }
   return g_noalloc_addr[device];
}

}  // namespace fftsvd

extern "C" {

// Reaction potentials without any device allocation: for callers that cannot
// call cudaMalloc (see include/fftsvd_b200.h).  sol and phi are device pointers.
int fftsvd_b200_reaction_potentials_noalloc(fftsvd_surface* s, const double* sol, double* phi) {
   if (!s || !sol || !phi) return FFTSVD_ERR_ARGUMENT;
   int previous = -1;
   try {
      Surface& S = s->s;
      FFTSVD_REQUIRE(S.geom, "surface has no panel geometry");
      const int nq = S.num_charges, np = S.geom->num_panels;
      if (nq == 0) return FFTSVD_OK;
      if ((size_t)nq > kNoAllocScratchDoubles)
         throw Error(FFTSVD_ERR_ARGUMENT, "fftsvd_b200_reaction_potentials_noalloc: " + std::to_string(nq) +
                                              " charges exceed the scratch limit of " +
                                              std::to_string(kNoAllocScratchDoubles) + " charges");
      FFTSVD_CUDA(cudaGetDevice(&previous));
      if (previous != S.device) FFTSVD_CUDA(cudaSetDevice(S.device));
      double* scratch = noalloc_scratch(S.device);
      // same chunking as the allocating path, reduced until chunks x charges fits the scratch
      int chunks = std::max(1, std::min(kReactChunks, (np + kReactPanelTile - 1) / kReactPanelTile));
      chunks = std::max(1, std::min<int>(chunks, (int)(kNoAllocScratchDoubles / (size_t)nq)));
      dim3 grid((nq + kReactThreads - 1) / kReactThreads, chunks);
      // every scratch entry the reduction reads is written by the partial kernel of this call
      reaction_partial_kernel<<<grid, kReactThreads, 0, S.stream>>>(np, S.geom->panels.get(), S.geom->phi_row.get(),
                                                                    S.geom->dphi_row.get(), sol, nq,
                                                                    S.charge_pos.get(), scratch, nullptr, 0);
      FFTSVD_CHECK_LAUNCH();
      reaction_reduce_kernel<<<(nq + 255) / 256, 256, 0, S.stream>>>(nq, chunks, scratch, phi);
      FFTSVD_CHECK_LAUNCH();
      FFTSVD_CUDA(cudaStreamSynchronize(S.stream));
      if (previous != S.device) FFTSVD_CUDA(cudaSetDevice(previous));
      return FFTSVD_OK;
   } catch (const Error& e) {
      if (previous >= 0) cudaSetDevice(previous);
      set_last_error(e.what());
      return e.code;
   }
}

int fftsvd_b200_energy(fftsvd_surface* s, const double* phi, double* energy) {
   if (!s || !phi || !energy) return FFTSVD_ERR_ARGUMENT;
   double e = 0.0;
   for (int c = 0; c < s->s.num_charges; c++) e += 0.5 * s->s.charge_q_host[c] * phi[c];
   *energy = e * 332.112 / s->s.eps_in;
   return FFTSVD_OK;
}

int fftsvd_b200_rhs_groups_device(fftsvd_surface* s, int32_t ngroups, const int32_t* group_ptr, double* rhs) {
   if (!s || !group_ptr || !rhs) return FFTSVD_ERR_ARGUMENT;
   return guarded([&] { rhs_groups_device(s->s, ngroups, group_ptr, rhs); });
}

int fftsvd_b200_group_energies_device(fftsvd_surface* s, int32_t ngroups, const int32_t* group_ptr, const double* sol,
                                      double* energies) {
   if (!s || !group_ptr || !sol || !energies) return FFTSVD_ERR_ARGUMENT;
   return guarded([&] { group_energies_device(s->s, ngroups, group_ptr, sol, energies); });
}

}  // extern "C"
