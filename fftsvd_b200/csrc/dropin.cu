// Drop-in replacements for the reference PBE API entry points
// (FFTSVDpbeAPI.h:150,153) over a caller's reference-built SurfaceOperator:
//
//   solveSurfaceOperator  FFTSVDpbeAPI.c:1884-1888 -> GMRES_SurfaceOperator (GMRES.c:446-539)
//   generateRHS           FFTSVDpbeAPI.c:1871-1876 -> SurfaceOperator_makeRHS (SurfaceOperator.c:291-321)
//   collectPotentials     FFTSVDpbeAPI.c:1896-1922 -> SurfaceOperator_calculateReactionPotentials,
//                         direct branch (SurfaceOperator.c:364-401), plus the optional Coulomb sum
//
// The reference structures (layout in refabi.h) are read, never modified.  On
// the first solve for a given (SurfaceOperator, Preconditioner) pair the
// operator of every region tree is flattened and uploaded; later solves with
// the same pair reuse the device copy while a sampled signature of the
// operator (sizes, parameters, centroids, near-field blocks, preconditioner)
// still matches; an operator changed in place in a way the sample misses must
// not be passed again under the same addresses.  Errors are reported on stderr and leave *solution / *rhs NULL instead
// of exiting the process.
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <array>
#include <cctype>
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <utility>
#include <vector>

#include "nbody.h"
#include "refabi.h"
#include "setup.h"
#include "surface.h"

// The reference keeps the GMRES tolerance in this process global
// (FFTSVDpbeAPI.c:25); weak so that the library also links without it.
extern "C" double errortolerance __attribute__((weak));
// Parameters of collectPotentials, process globals of the reference API
// (FFTSVDpbeAPI.c:20, 29).  Weak references make a program linked with the
// reference objects export them to this library; a program that loads the
// reference objects at run time is searched with dlsym instead.
extern "C" double innerdielectric __attribute__((weak));
extern "C" unsigned int addcoulombic __attribute__((weak));

namespace fftsvd {
namespace {

void collect_cubes(ref::Cube* c, std::vector<ref::Cube*>& all) {
   if (!c) return;
   all.push_back(c);
   if (!c->leaf)
      for (int x = 0; x < 2; x++)
         for (int y = 0; y < 2; y++)
            for (int z = 0; z < 2; z++) collect_cubes(c->children[x][y][z], all);
}

// Reference Tree/Cube objects -> flat arrays (the fields Tree_multiplyboth reads).
void flatten_reference_tree(const ref::Tree* t, setup::FlatTree& F) {
   FFTSVD_REQUIRE(t && t->root, "region without a tree");
   FFTSVD_REQUIRE(t->partitioningdepth >= 1 && t->partitioningdepth <= FFTSVD_MAX_DEPTH, "tree depth out of range");
   F = setup::FlatTree();
   F.num_panels = (int)t->numpanels;
   F.num_points = (int)t->numpoints;
   F.depth = (int)t->partitioningdepth;
   for (int d = 0; d < F.depth; d++) F.grid.push_back((int)t->gridpointsperlevel[d]);
   std::vector<ref::Cube*> all;
   collect_cubes(t->root, all);
   std::map<const ref::Cube*, int> far_index;
   for (ref::Cube* c : all) {
      if (c->leaf && c->drows > 0 && c->dcolumns > 0) {
         FFTSVD_REQUIRE(c->D_single && c->D_double, "leaf without near-field blocks");
         F.leaf_row_ptr.push_back((int32_t)F.leaf_rows.size());
         F.leaf_col_ptr.push_back((int32_t)F.leaf_cols.size());
         F.leaf_d_ptr.push_back((int64_t)F.d_single.size());
         for (unsigned i = 0; i < c->numpointindices; i++) F.leaf_rows.push_back((int32_t)c->pointindices[i]);
         for (unsigned i = 0; i < c->numpanelindices; i++) F.leaf_cols.push_back((int32_t)c->panelindices[i]);
         for (unsigned l = 0; l < c->numlocalcubes; l++)
            for (unsigned j = 0; j < c->localcubes[l]->numpanelindices; j++)
               F.leaf_cols.push_back((int32_t)c->localcubes[l]->panelindices[j]);
         FFTSVD_REQUIRE(F.leaf_rows.size() - F.leaf_row_ptr.back() == c->drows, "leaf rows do not match drows");
         FFTSVD_REQUIRE(F.leaf_cols.size() - F.leaf_col_ptr.back() == c->dcolumns, "leaf columns do not match dcolumns");
         const size_t cnt = (size_t)c->drows * c->dcolumns;
         F.d_single.insert(F.d_single.end(), c->D_single[0], c->D_single[0] + cnt);
         F.d_double.insert(F.d_double.end(), c->D_double[0], c->D_double[0] + cnt);
      }
      if (c->numinteractingcubes > 0) far_index[c] = (int)far_index.size();
   }
   F.leaf_row_ptr.push_back((int32_t)F.leaf_rows.size());
   F.leaf_col_ptr.push_back((int32_t)F.leaf_cols.size());
   F.leaf_d_ptr.push_back((int64_t)F.d_single.size());
   for (ref::Cube* c : all) {
      if (c->numinteractingcubes == 0) continue;
      const unsigned n = t->gridpointsperlevel[c->level], gp3 = n * n * n;
      F.cube_level.push_back((int32_t)c->level);
      for (int k = 0; k < 3; k++) F.cube_index.push_back((int32_t)c->indices[k]);
      F.cube_panel_ptr.push_back((int32_t)F.cube_panels.size());
      for (unsigned i = 0; i < c->numpanelindices; i++) F.cube_panels.push_back((int32_t)c->panelindices[i]);
      F.cube_point_ptr.push_back((int32_t)F.cube_points.size());
      for (unsigned i = 0; i < c->numpointindices; i++) F.cube_points.push_back((int32_t)c->pointindices[i]);
      const bool src = c->numpanelindices > 0 && c->rowrank > 0 && c->VTsrc && c->PV_single && c->PV_double;
      const bool dst = c->numpointindices > 0 && c->columnrank > 0 && c->Udest && c->UTI;
      F.cube_row_rank.push_back(src ? (int32_t)c->rowrank : 0);
      F.cube_col_rank.push_back(dst ? (int32_t)c->columnrank : 0);
      F.cube_vt_ptr.push_back((int64_t)F.vt.size());
      F.cube_pv_ptr.push_back((int64_t)F.pv_single.size());
      F.cube_uti_ptr.push_back((int64_t)F.uti.size());
      F.cube_u_ptr.push_back((int64_t)F.u.size());
      if (src) {
         F.vt.insert(F.vt.end(), c->VTsrc[0], c->VTsrc[0] + (size_t)c->rowrank * c->numpanelindices);
         F.pv_single.insert(F.pv_single.end(), c->PV_single[0], c->PV_single[0] + (size_t)gp3 * c->rowrank);
         F.pv_double.insert(F.pv_double.end(), c->PV_double[0], c->PV_double[0] + (size_t)gp3 * c->rowrank);
      }
      if (dst) {
         F.uti.insert(F.uti.end(), c->UTI[0], c->UTI[0] + (size_t)c->columnrank * gp3);
         F.u.insert(F.u.end(), c->Udest[0], c->Udest[0] + (size_t)c->numpointindices * c->columnrank);
      }
      F.inter_ptr.push_back((int32_t)F.inter_cubes.size());
      for (unsigned i = 0; i < c->numinteractingcubes; i++) {
         auto it = far_index.find(c->interactingcubes[i]);
         FFTSVD_REQUIRE(it != far_index.end(), "interacting cube outside the tree");
         F.inter_cubes.push_back(it->second);
      }
   }
   F.num_cubes = (int)far_index.size();
   F.cube_panel_ptr.push_back((int32_t)F.cube_panels.size());
   F.cube_point_ptr.push_back((int32_t)F.cube_points.size());
   F.cube_vt_ptr.push_back((int64_t)F.vt.size());
   F.cube_pv_ptr.push_back((int64_t)F.pv_single.size());
   F.cube_uti_ptr.push_back((int64_t)F.uti.size());
   F.cube_u_ptr.push_back((int64_t)F.u.size());
   F.inter_ptr.push_back((int32_t)F.inter_cubes.size());
   int64_t off = 0;
   for (int d = 0; d < F.depth; d++) {
      const int np = 2 * F.grid[d] - 1, pg = np * np * F.grid[d];
      F.t_level_ptr.push_back(off);
      for (int s = 0; s < 343; s++) {
         const float* tv = t->Tprecomputed ? t->Tprecomputed[d][s / 49][(s / 7) % 7][s % 7] : nullptr;
         for (int f = 0; f < pg; f++) {
            F.t_ops.push_back(tv ? tv[2 * f] : 0.0);
            F.t_ops.push_back(tv ? tv[2 * f + 1] : 0.0);
         }
      }
      off += 343LL * pg;
   }
   F.t_level_ptr.push_back(off);
}

struct RegionArrays {
   setup::FlatTree flat;
   std::vector<int32_t> phi_idx, dphi_idx, out_idx;
   std::vector<double> phi_s, dphi_s, jump;
};

// Region maps of SurfaceOperator_multiply (SurfaceOperator.c:51-158) for every region.
void gather_regions(const ref::SurfaceOperator* so, std::vector<std::unique_ptr<RegionArrays>>& out) {
   if (so->tree && so->tree->numpanels > 0) {
      auto R = std::make_unique<RegionArrays>();
      for (unsigned k = 0; k < so->mynumpanels; k++) {
         R->phi_idx.push_back((int32_t)(so->startphi + k));
         R->phi_s.push_back(1.0);
         R->dphi_idx.push_back((int32_t)(so->startdphi + k));
         R->dphi_s.push_back(-1.0);
         R->out_idx.push_back((int32_t)(so->startphi + k));
         R->jump.push_back(0.0);
      }
      for (unsigned c = 0; c < so->numchildren; c++) {
         const ref::SurfaceOperator* ch = so->children[c];
         for (unsigned j = 0; j < ch->mynumpanels; j++) {
            R->phi_idx.push_back((int32_t)(ch->startphi + j));
            R->phi_s.push_back(-1.0);
            R->dphi_idx.push_back((int32_t)(ch->startdphi + j));
            R->dphi_s.push_back(ch->epsilon / so->epsilon);
            R->out_idx.push_back((int32_t)(ch->startdphi + j));
            R->jump.push_back(-4.0 * M_PI);
         }
      }
      FFTSVD_REQUIRE(R->phi_idx.size() == so->tree->numpanels && so->tree->numpoints == so->tree->numpanels,
                     "region panels do not match its tree (only collocation at panel centroids is supported)");
      flatten_reference_tree(so->tree, R->flat);
      out.push_back(std::move(R));
   }
   for (unsigned c = 0; c < so->numchildren; c++) gather_regions(so->children[c], out);
}

// 64-bit signature of a caller's operator, built from its sizes, parameters
// and a strided sample of its panel centroids, near-field blocks and
// preconditioner values.  A cached device copy is reused only when the
// signature still matches, so an operator allocated at the addresses of a
// freed one (or rebuilt in place with another kappa or mesh) is uploaded anew.
struct Signature {
   uint64_t h = 1469598103934665603ull;
   void add(uint64_t v) {
      h ^= v + 0x9e3779b97f4a7c15ull + (h << 6) + (h >> 2);
      h *= 1099511628211ull;
   }
   void add(double d) {
      uint64_t v;
      std::memcpy(&v, &d, sizeof v);
      add(v);
   }
   void add_floats(const float* p, size_t n) {
      for (size_t i = 0; i < n; i++) {
         uint32_t v;
         std::memcpy(&v, p + i, sizeof v);
         add((uint64_t)v);
      }
   }
};

constexpr size_t kSignatureSamples = 4096;

void region_signature(const ref::SurfaceOperator* so, Signature& sg) {
   sg.add(so->epsilon);
   sg.add(so->kappa);
   sg.add(((uint64_t)so->mynumpanels << 32) ^ so->numchildren);
   sg.add(((uint64_t)so->startphi << 32) ^ so->startdphi);
   const ref::Tree* t = so->tree;
   if (t && t->numpanels > 0) {
      sg.add(((uint64_t)t->numpanels << 32) ^ t->numpoints);
      sg.add(((uint64_t)t->partitioningdepth << 32) ^ t->gridpoints);
      sg.add(t->epsilon);
      const size_t stride = std::max<size_t>(1, t->numpanels / kSignatureSamples);
      for (size_t i = 0; i < t->numpanels; i += stride) {
         const ref::Vec3* c = t->panels[i]->centroid;
         sg.add(c->x);
         sg.add(c->y);
         sg.add(c->z);
      }
      std::vector<ref::Cube*> all;
      collect_cubes(t->root, all);
      std::vector<const ref::Cube*> leaves;
      for (const ref::Cube* c : all)
         if (c->leaf && c->drows > 0 && c->dcolumns > 0 && c->D_single && c->D_double) leaves.push_back(c);
      const size_t lstride = std::max<size_t>(1, leaves.size() / 64);
      for (size_t l = 0; l < leaves.size(); l += lstride) {
         const ref::Cube* c = leaves[l];
         const size_t cnt = std::min<size_t>((size_t)c->drows * c->dcolumns, 64);
         sg.add_floats(c->D_single[0], cnt);
         sg.add_floats(c->D_double[0], cnt);
      }
   }
   for (unsigned c = 0; c < so->numchildren; c++) region_signature(so->children[c], sg);
}

uint64_t operator_signature(const ref::SurfaceOperator* so, const ref::Preconditioner* P) {
   Signature sg;
   region_signature(so, sg);
   const size_t stride = std::max<size_t>(1, P->columns / kSignatureSamples);
   for (size_t c = 0; c < P->columns; c += stride) {
      sg.add((uint64_t)P->numelements[c]);
      for (unsigned e = 0; e < P->numelements[c]; e++) {
         sg.add((uint64_t)P->P[c][e].row);
         sg.add(P->P[c][e].value);
      }
   }
   return sg.h;
}

struct CachedSurface {
   uint64_t signature = 0;
   std::unique_ptr<fftsvd_surface> surface;
};

std::mutex g_cache_mutex;
std::map<std::pair<const void*, const void*>, CachedSurface> g_cache;

fftsvd_surface* surface_for(const ref::SurfaceOperator* so, const ref::Preconditioner* P, unsigned numtotalpanels) {
   std::lock_guard<std::mutex> lock(g_cache_mutex);
   const int n = 2 * (int)numtotalpanels;
   FFTSVD_REQUIRE(P && P->rows == (unsigned)n && P->columns == (unsigned)n, "preconditioner size mismatch");
   const uint64_t signature = operator_signature(so, P);
   auto key = std::make_pair((const void*)so, (const void*)P);
   auto it = g_cache.find(key);
   if (it != g_cache.end()) {
      if (it->second.signature == signature) return it->second.surface.get();
      g_cache.erase(it);  // another operator now lives at these addresses
   }
   std::vector<std::unique_ptr<RegionArrays>> regions;
   gather_regions(so, regions);
   FFTSVD_REQUIRE(!regions.empty(), "surface operator without panels");
   std::vector<fftsvd_tree_flat> views(regions.size());
   std::vector<fftsvd_region_map> maps(regions.size());
   for (size_t r = 0; r < regions.size(); r++) {
      regions[r]->flat.view(views[r]);
      RegionArrays& R = *regions[r];
      maps[r] = {R.phi_idx.data(), R.phi_s.data(), R.dphi_idx.data(), R.dphi_s.data(), R.out_idx.data(), R.jump.data()};
   }
   std::vector<int32_t> col_ptr(n + 1, 0), rows;
   std::vector<double> vals;
   for (int c = 0; c < n; c++) {
      for (unsigned e = 0; e < P->numelements[c]; e++) {
         rows.push_back((int32_t)P->P[c][e].row);
         vals.push_back(P->P[c][e].value);
      }
      col_ptr[c + 1] = (int32_t)rows.size();
   }
   fftsvd_precond_csc pc{n, col_ptr.data(), rows.data(), vals.data()};
   auto s = std::make_unique<fftsvd_surface>();
   init_surface(s->s, n, (int)regions.size(), views.data(), maps.data(), &pc);
   fftsvd_surface* out = s.get();
   g_cache[key] = CachedSurface{signature, std::move(s)};
   return out;
}

// The stream the drop-in right-hand side and collection run on: one non-blocking
// stream per device, created on first use and owned by the library, so these
// calls neither use nor wait on the legacy default stream.
cudaStream_t dropin_stream() {
   static std::mutex mu;
   static std::map<int, cudaStream_t> streams;
   int dev = 0;
   FFTSVD_CUDA(cudaGetDevice(&dev));
   std::lock_guard<std::mutex> lock(mu);
   auto it = streams.find(dev);
   if (it != streams.end()) return it->second;
   cudaStream_t st = nullptr;
   FFTSVD_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
   streams[dev] = st;
   return st;
}

// SurfaceOperator_makeRHS (SurfaceOperator.c:291-321) over the caller's region tree:
// one launch of the library's tiled right-hand-side kernel per region with charges,
// its own panels' phi rows and its children's dphi rows as targets.
void rhs_region(const ref::SurfaceOperator* so, double* drhs) {
   if (so->charges && so->charges->numcharges > 0) {
      std::vector<double> cent;
      std::vector<int32_t> rows;
      for (unsigned j = 0; j < so->mynumpanels; j++) {
         const ref::Vec3* c = so->tree->panels[j]->centroid;
         cent.insert(cent.end(), {c->x, c->y, c->z});
         rows.push_back((int32_t)(so->startphi + j));
      }
      for (unsigned k = 0; k < so->numchildren; k++) {
         const ref::SurfaceOperator* ch = so->children[k];
         for (unsigned j = 0; j < ch->mynumpanels; j++) {
            const ref::Vec3* c = ch->tree->panels[j]->centroid;
            cent.insert(cent.end(), {c->x, c->y, c->z});
            rows.push_back((int32_t)(ch->startdphi + j));
         }
      }
      const ref::Charge* Q = so->charges;
      std::vector<double> qpos, qv(Q->charges, Q->charges + Q->numcharges);
      for (unsigned i = 0; i < Q->numcharges; i++) qpos.insert(qpos.end(), {Q->points[i]->x, Q->points[i]->y, Q->points[i]->z});
      if (!rows.empty()) {
         DevBuf<double> dc, dq, dqp;
         DevBuf<int32_t> dr;
         dc.upload(cent);
         dr.upload(rows);
         dq.upload(qv);
         dqp.upload(qpos);
         const int nt = (int)rows.size();
         const cudaStream_t stream = dropin_stream();
         rhs_points_device(nt, dc.get(), dr.get(), (int)qv.size(), dqp.get(), dq.get(), drhs, stream);
         // the staging buffers are freed on return
         FFTSVD_CUDA(cudaStreamSynchronize(stream));
      }
   }
   for (unsigned k = 0; k < so->numchildren; k++) rhs_region(so->children[k], drhs);
}

template <typename T>
const T* api_global(const T* weak_address, const char* name) {
   if (weak_address) return weak_address;
   return static_cast<const T*>(dlsym(RTLD_DEFAULT, name));
}

// Geometry of a reference flat panel from its stored vertices (FlatPanel.c:5-35).
void reference_flat_panel(const ref::Panel* p, FlatPanel& out) {
   FFTSVD_REQUIRE(p && p->type == 0 && p->realpanel, "only flat panels are supported");
   const ref::FlatPanel* f = static_cast<const ref::FlatPanel*>(p->realpanel);
   double v[3][3];
   for (int k = 0; k < 3; k++) {
      FFTSVD_REQUIRE(f->vertex[k], "flat panel without vertices");
      v[k][0] = f->vertex[k]->x;
      v[k][1] = f->vertex[k]->y;
      v[k][2] = f->vertex[k]->z;
   }
   make_flat_panel(out, v[0], v[1], v[2]);
}

// Reaction potentials of every region that holds charges, added at
// pot[charges->globalindexstart + j] (SurfaceOperator.c:364-401, direct
// branch, recursing over the children).  A region's own panels enter with
// (phi, dphi) and the coincidence term; its children's panels with
// (-phi, -eps_child/eps dphi) and no coincidence term.  One launch serves both:
// the scaled densities are laid out per panel, and the coincidence term the
// kernel adds for a child panel (+4 pi phi) is taken off on the host.
void reaction_regions(const ref::SurfaceOperator* so, const double* sol, std::vector<double>& pot) {
   FFTSVD_REQUIRE(!so->M3, "regions with an M3 tree (accelerateM3) are not supported");
   const ref::Charge* Q = so->charges;
   if (Q && Q->numcharges > 0) {
      const size_t nq = Q->numcharges, g0 = Q->globalindexstart;
      FFTSVD_REQUIRE(g0 + nq <= pot.size(), "charges of a region lie beyond the collected entries");
      std::vector<FlatPanel> panels;
      std::vector<double> dens;
      std::vector<int32_t> phi_row, dphi_row;
      auto add_panel = [&](const ref::Panel* p, double phi, double dphi) {
         panels.emplace_back();
         reference_flat_panel(p, panels.back());
         phi_row.push_back((int32_t)dens.size());
         dens.push_back(phi);
         dphi_row.push_back((int32_t)dens.size());
         dens.push_back(dphi);
      };
      FFTSVD_REQUIRE(so->mynumpanels == 0 || (so->tree && so->tree->numpanels >= so->mynumpanels),
                     "region panels do not match its tree");
      for (unsigned i = 0; i < so->mynumpanels; i++)
         add_panel(so->tree->panels[i], sol[so->startphi + i], sol[so->startdphi + i]);
      // child panel centroid -> sum of phi over the child panels there (matched by exact equality)
      std::map<std::array<double, 3>, double> child_centroid_phi;
      for (unsigned k = 0; k < so->numchildren; k++) {
         const ref::SurfaceOperator* ch = so->children[k];
         FFTSVD_REQUIRE(ch->mynumpanels == 0 || (ch->tree && ch->tree->numpanels >= ch->mynumpanels),
                        "child region panels do not match its tree");
         const double ratio = -ch->epsilon / so->epsilon;
         for (unsigned i = 0; i < ch->mynumpanels; i++) {
            const double phi = sol[ch->startphi + i];
            add_panel(ch->tree->panels[i], -phi, ratio * sol[ch->startdphi + i]);
            const FlatPanel& P = panels.back();
            child_centroid_phi[{P.centroid[0], P.centroid[1], P.centroid[2]}] += phi;
         }
      }
      std::vector<double> qpos(3 * nq);
      for (size_t j = 0; j < nq; j++) {
         FFTSVD_REQUIRE(Q->points[j], "charge without a position");
         qpos[3 * j] = Q->points[j]->x;
         qpos[3 * j + 1] = Q->points[j]->y;
         qpos[3 * j + 2] = Q->points[j]->z;
      }
      std::vector<double> phi(nq, 0.0);
      if (!panels.empty()) {
         DevBuf<FlatPanel> d_panels;
         DevBuf<int32_t> d_phi_row, d_dphi_row;
         DevBuf<double> d_dens, d_qpos, d_out(nq);
         d_panels.upload(panels);
         d_phi_row.upload(phi_row);
         d_dphi_row.upload(dphi_row);
         d_dens.upload(dens);
         d_qpos.upload(qpos);
         const cudaStream_t stream = dropin_stream();
         reaction_points_device((int)panels.size(), d_panels.get(), d_phi_row.get(), d_dphi_row.get(), d_dens.get(),
                                (int)nq, d_qpos.get(), d_out.get(), stream);
         FFTSVD_CUDA(cudaMemcpyAsync(phi.data(), d_out.get(), sizeof(double) * nq, cudaMemcpyDeviceToHost, stream));
         FFTSVD_CUDA(cudaStreamSynchronize(stream));
      }
      for (size_t j = 0; j < nq; j++) {
         if (!child_centroid_phi.empty()) {
            auto it = child_centroid_phi.find({qpos[3 * j], qpos[3 * j + 1], qpos[3 * j + 2]});
            if (it != child_centroid_phi.end()) phi[j] -= 4.0 * M_PI * it->second;
         }
         pot[g0 + j] += phi[j];
      }
   }
   for (unsigned k = 0; k < so->numchildren; k++) reaction_regions(so->children[k], sol, pot);
}

// The Coulomb term of collectPotentials (FFTSVDpbeAPI.c:1906-1919): one thread
// per collected atom, input atoms in their order, pot[c] += kt q_a / (eps d).
__global__ void coulomb_kernel(int nc, const double* __restrict__ cpos, int ni, const double* __restrict__ ipos,
                               const double* __restrict__ iq, double kt, double eps, double* __restrict__ pot) {
   const int c = blockIdx.x * blockDim.x + threadIdx.x;
   if (c >= nc) return;
   const double x = cpos[3 * c], y = cpos[3 * c + 1], z = cpos[3 * c + 2];
   double p = pot[c];
   for (int a = 0; a < ni; a++) {
      const double dx = ipos[3 * a] - x, dy = ipos[3 * a + 1] - y, dz = ipos[3 * a + 2] - z;
      const double d = sqrt(dx * dx + dy * dy + dz * dz);
      if (d > 0.0) p += kt * iq[a] / (eps * d);
   }
   pot[c] = p;
}

void charge_epsilons(const ref::SurfaceOperator* so, std::vector<double>& eps) {
   if (so->charges && so->charges->numcharges > 0) eps.push_back(so->epsilon);
   for (unsigned k = 0; k < so->numchildren; k++) charge_epsilons(so->children[k], eps);
}

}  // namespace
}  // namespace fftsvd

using namespace fftsvd;

extern "C" void solveSurfaceOperator(double** solution, struct _SurfaceOperator* pbesurfaceoperator,
                                     struct _Preconditioner* preconditioner, double* rhs, unsigned int numtotalpanels) {
   if (!solution) return;
   *solution = nullptr;
   const double tol = &errortolerance ? errortolerance : 1e-6;
   try {
      FFTSVD_REQUIRE(pbesurfaceoperator && preconditioner && rhs && numtotalpanels > 0, "null argument");
      fftsvd_surface* s = surface_for(reinterpret_cast<const ref::SurfaceOperator*>(pbesurfaceoperator),
                                      reinterpret_cast<const ref::Preconditioner*>(preconditioner), numtotalpanels);
      const int n = 2 * (int)numtotalpanels;
      int precision = FFTSVD_PREC_MIXED;
      if (const char* e = std::getenv("FFTSVD_B200_PRECISION")) {
         if (!strcmp(e, "fp64")) precision = FFTSVD_PREC_FP64;
         else if (!strcmp(e, "fp32")) precision = FFTSVD_PREC_FP32;
      }
      double* out = static_cast<double*>(std::calloc((size_t)n, sizeof(double)));
      FFTSVD_REQUIRE(out, "host allocation failed");
      fftsvd_solve_info info{};
      const int rc = fftsvd_b200_solve(s, precision, rhs, out, tol, 1000, &info);
      if (rc != FFTSVD_OK && rc != FFTSVD_ERR_NOT_CONVERGED) {
         std::free(out);
         throw Error(rc, fftsvd_b200_last_error());
      }
      *solution = out;
   } catch (const std::exception& e) {
      set_last_error(e.what());
      std::fprintf(stderr, "fftsvd_b200 solveSurfaceOperator: %s\n", e.what());
   }
}

extern "C" void generateRHS(double** rhs, struct _SurfaceOperator* pbesurfaceoperator, unsigned int numtotalpanels) {
   if (!rhs) return;
   *rhs = nullptr;
   try {
      FFTSVD_REQUIRE(pbesurfaceoperator && numtotalpanels > 0, "null argument");
      const int n = 2 * (int)numtotalpanels;
      const cudaStream_t stream = dropin_stream();
      DevBuf<double> d(n);
      d.zero(stream);
      rhs_region(reinterpret_cast<const ref::SurfaceOperator*>(pbesurfaceoperator), d.get());
      double* out = static_cast<double*>(std::calloc((size_t)n, sizeof(double)));
      FFTSVD_REQUIRE(out, "host allocation failed");
      const cudaError_t e1 = cudaMemcpyAsync(out, d.get(), sizeof(double) * n, cudaMemcpyDeviceToHost, stream);
      const cudaError_t e2 = e1 == cudaSuccess ? cudaStreamSynchronize(stream) : e1;
      if (e2 != cudaSuccess) {
         std::free(out);
         throw Error(FFTSVD_ERR_CUDA, std::string("generateRHS copy: ") + cudaGetErrorString(e2));
      }
      *rhs = out;
   } catch (const std::exception& e) {
      set_last_error(e.what());
      std::fprintf(stderr, "fftsvd_b200 generateRHS: %s\n", e.what());
   }
}

extern "C" void collectPotentials(struct PDBentry_s* PDBcollectentries, unsigned int numPDBcollectentries,
                                  struct PDBentry_s* PDBinputentries, unsigned int numPDBinputentries,
                                  struct _SurfaceOperator* pbesurfaceoperator, double* solution) {
   constexpr double kKTConversion = 561.0;  // FFTSVDpbeAPI.h:13
   try {
      FFTSVD_REQUIRE(pbesurfaceoperator && solution, "null argument");
      FFTSVD_REQUIRE(numPDBcollectentries == 0 || PDBcollectentries, "null collect entries");
      FFTSVD_REQUIRE(numPDBinputentries == 0 || PDBinputentries, "null input entries");
      const ref::SurfaceOperator* so = reinterpret_cast<const ref::SurfaceOperator*>(pbesurfaceoperator);
      ref::PDBentry* collect = reinterpret_cast<ref::PDBentry*>(PDBcollectentries);
      const ref::PDBentry* input = reinterpret_cast<const ref::PDBentry*>(PDBinputentries);
      double eps_in = 0.0;
      if (const double* g = api_global(&innerdielectric, "innerdielectric")) {
         eps_in = *g;
      } else {
         std::vector<double> eps;
         charge_epsilons(so, eps);
         FFTSVD_REQUIRE(!eps.empty(), "innerdielectric is not defined and no region holds charges");
         for (double e : eps)
            FFTSVD_REQUIRE(e == eps[0], "innerdielectric is not defined and the charged regions differ in epsilon");
         eps_in = eps[0];
      }
      FFTSVD_REQUIRE(eps_in > 0.0, "innerdielectric must be positive");
      const unsigned int* coul = api_global(&addcoulombic, "addcoulombic");
      const size_t nc = numPDBcollectentries;
      std::vector<double> pot(nc, 0.0);
      reaction_regions(so, solution, pot);
      for (size_t a = 0; a < nc; a++) pot[a] = kKTConversion * pot[a] / eps_in;
      if (coul && *coul && nc > 0) {
         std::vector<double> cpos(3 * nc), ipos, iq;
         for (size_t c = 0; c < nc; c++) {
            cpos[3 * c] = collect[c].x;
            cpos[3 * c + 1] = collect[c].y;
            cpos[3 * c + 2] = collect[c].z;
         }
         for (unsigned a = 0; a < numPDBinputentries; a++)
            if (std::toupper((unsigned char)input[a].chain) != 'X') {
               ipos.insert(ipos.end(), {input[a].x, input[a].y, input[a].z});
               iq.push_back(input[a].charge);
            }
         if (!iq.empty()) {
            DevBuf<double> dcpos, dipos, diq, dpot;
            dcpos.upload(cpos);
            dipos.upload(ipos);
            diq.upload(iq);
            dpot.upload(pot);
            const cudaStream_t stream = dropin_stream();
            const int ncol = (int)nc;
            coulomb_kernel<<<(ncol + 127) / 128, 128, 0, stream>>>(ncol, dcpos.get(), (int)iq.size(), dipos.get(),
                                                                    diq.get(), kKTConversion, eps_in, dpot.get());
            FFTSVD_CHECK_LAUNCH();
            FFTSVD_CUDA(cudaMemcpyAsync(pot.data(), dpot.get(), sizeof(double) * nc, cudaMemcpyDeviceToHost, stream));
            FFTSVD_CUDA(cudaStreamSynchronize(stream));
         }
      }
      for (size_t a = 0; a < nc; a++) collect[a].potential = pot[a];
   } catch (const std::exception& e) {
      set_last_error(e.what());
      std::fprintf(stderr, "fftsvd_b200 collectPotentials: %s\n", e.what());
   }
}
