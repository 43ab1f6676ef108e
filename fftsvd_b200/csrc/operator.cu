// FFTSVD matvec on sm_100a: layout construction (host) and the four kernels.
//
// Reference stages (all in the reference are scalar loops over the octree):
//   join          SurfaceOperator_joinpotentials      SurfaceOperator.c:51-65
//   far_forward   Cube_multiplyboth_FFT_PV_VT         Cube.c:1986-2060, FFT.c:66-108
//   far_backward  Cube_multiply_T + Cube_multiply_U_UTI_IFFT   Cube.c:2062-2111, 2156-2225, FFT.c:112-150
//   near          Cube_multiply_D (single and double) Cube.c:1730-1798, plus the inner-surface
//                 jump and the split/join into the global vector   SurfaceOperator.c:78-158
//
// The DFTs are the zero-padded (2n-1)^3 real-data transforms of FFT.c written
// out as separable direct DFTs (the sizes are odd and tiny: 2n-1 = 7..17), with
// the padding offset n/2 folded into the twiddle exponents so only the n^3
// nonzero inputs and the n^3 cropped outputs are touched.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <string>

#include "operator.h"

namespace fftsvd {

// ------------------------------------------------------------------ layout

static int pad2(int v) { return (v + 1) & ~1; }

OperatorLayout build_layout(int num_unknowns, int num_trees, const fftsvd_tree_flat* trees,
                            const fftsvd_region_map* maps) {
   OperatorLayout L;
   FFTSVD_REQUIRE(num_unknowns > 0 && num_trees > 0, "empty operator");
   L.num_unknowns = num_unknowns;
   L.num_trees = num_trees;
   L.tree_panel_off.resize(num_trees + 1);
   L.tree_point_off.resize(num_trees + 1);
   int64_t np = 0, nq = 0;
   for (int t = 0; t < num_trees; t++) {
      FFTSVD_REQUIRE(trees[t].num_panels >= 0 && trees[t].num_points >= 0, "negative tree size");
      FFTSVD_REQUIRE(trees[t].depth >= 1 && trees[t].depth <= FFTSVD_MAX_DEPTH, "tree depth out of range");
      L.tree_panel_off[t] = np;
      L.tree_point_off[t] = nq;
      np += trees[t].num_panels;
      nq += trees[t].num_points;
      L.stage_levels = std::max(L.stage_levels, (int)trees[t].depth);
   }
   L.tree_panel_off[num_trees] = np;
   L.tree_point_off[num_trees] = nq;
   L.total_panels = np + 1;  // last slot stays zero: target of padding columns
   L.total_points = nq;
   const int32_t zero_slot = (int32_t)np;

   L.join_phi_idx.assign(L.total_panels, 0);
   L.join_dphi_idx.assign(L.total_panels, 0);
   L.join_phi_scale.assign(L.total_panels, 0.0);
   L.join_dphi_scale.assign(L.total_panels, 0.0);
   L.point_out.assign(nq, -1);
   L.point_panel.assign(nq, -1);
   L.point_jump.assign(nq, 0.0);
   std::vector<char> row_written(num_unknowns, 0);

   for (int t = 0; t < num_trees; t++) {
      const fftsvd_tree_flat& T = trees[t];
      const fftsvd_region_map& M = maps[t];
      const int64_t po = L.tree_panel_off[t], qo = L.tree_point_off[t];
      for (int k = 0; k < T.num_panels; k++) {
         FFTSVD_REQUIRE(M.phi_index[k] >= 0 && M.phi_index[k] < num_unknowns, "phi_index out of range");
         FFTSVD_REQUIRE(M.dphi_index[k] >= 0 && M.dphi_index[k] < num_unknowns, "dphi_index out of range");
         L.join_phi_idx[po + k] = M.phi_index[k];
         L.join_dphi_idx[po + k] = M.dphi_index[k];
         L.join_phi_scale[po + k] = M.phi_scale[k];
         L.join_dphi_scale[po + k] = M.dphi_scale[k];
      }
      for (int p = 0; p < T.num_points; p++) {
         int o = M.out_index[p];
         FFTSVD_REQUIRE(o >= 0 && o < num_unknowns, "out_index out of range");
         FFTSVD_REQUIRE(!row_written[o], "two tree points write the same unknown row");
         row_written[o] = 1;
         L.point_out[qo + p] = o;
         double j = M.jump ? M.jump[p] : 0.0;
         if (j != 0.0) {
            FFTSVD_REQUIRE(p < T.num_panels, "jump term on a point without a matching panel");
            L.point_jump[qo + p] = j;
            L.point_panel[qo + p] = (int32_t)(po + p);
         }
      }

      // ---- near field
      std::vector<char> covered(T.num_points, 0);
      for (int l = 0; l < T.num_leaves; l++) {
         const int r0 = T.leaf_row_ptr[l], r1 = T.leaf_row_ptr[l + 1];
         const int c0 = T.leaf_col_ptr[l], c1 = T.leaf_col_ptr[l + 1];
         const int nr = r1 - r0, nc = c1 - c0, ncp = pad2(nc);
         FFTSVD_REQUIRE(nr >= 0 && nc >= 0, "bad leaf extents");
         if (nr == 0) continue;
         FFTSVD_REQUIRE(T.leaf_d_ptr[l + 1] - T.leaf_d_ptr[l] == (int64_t)nr * nc, "leaf D size mismatch");
         LeafDesc d;
         d.row_off = (int32_t)L.leaf_rows.size();
         d.nrows = nr;
         d.col_off = (int32_t)L.leaf_cols.size();
         d.ncols = ncp;
         d.d_off = (int64_t)(L.d_pairs.size() / 2);
         for (int r = r0; r < r1; r++) {
            int p = T.leaf_rows[r];
            FFTSVD_REQUIRE(p >= 0 && p < T.num_points, "leaf row out of range");
            FFTSVD_REQUIRE(!covered[p], "point in two leaves");
            covered[p] = 1;
            L.leaf_rows.push_back((int32_t)(qo + p));
         }
         for (int c = c0; c < c1; c++) {
            int k = T.leaf_cols[c];
            FFTSVD_REQUIRE(k >= 0 && k < T.num_panels, "leaf column out of range");
            L.leaf_cols.push_back((int32_t)(po + k));
         }
         for (int c = nc; c < ncp; c++) L.leaf_cols.push_back(zero_slot);
         const int64_t db = T.leaf_d_ptr[l];
         for (int r = 0; r < nr; r++) {
            for (int c = 0; c < nc; c++) {
               L.d_pairs.push_back(T.d_single[db + (int64_t)r * nc + c]);
               L.d_pairs.push_back(T.d_double[db + (int64_t)r * nc + c]);
            }
            for (int c = nc; c < ncp; c++) { L.d_pairs.push_back(0.0); L.d_pairs.push_back(0.0); }
         }
         L.operator_elems += 2LL * nr * nc;
         L.leaves.push_back(d);
      }
      // points of no leaf still receive their far field and jump term
      std::vector<int32_t> rest;
      for (int p = 0; p < T.num_points; p++)
         if (!covered[p]) rest.push_back((int32_t)(qo + p));
      for (size_t i = 0; i < rest.size(); i += 64) {
         LeafDesc d;
         d.row_off = (int32_t)L.leaf_rows.size();
         d.nrows = (int32_t)std::min<size_t>(64, rest.size() - i);
         d.col_off = (int32_t)L.leaf_cols.size();
         d.ncols = 0;
         d.d_off = (int64_t)(L.d_pairs.size() / 2);
         for (int r = 0; r < d.nrows; r++) L.leaf_rows.push_back(rest[i + r]);
         L.leaves.push_back(d);
      }

      // ---- far field
      std::vector<int64_t> spec_of_cube(T.num_cubes, -1);
      const int64_t t_base = (int64_t)(L.t_pairs.size() / 2);
      for (int c = 0; c < T.num_cubes; c++) {
         const int lvl = T.cube_level[c];
         FFTSVD_REQUIRE(lvl >= 0 && lvl < T.depth, "cube level out of range");
         const int n = T.grid[lvl];
         FFTSVD_REQUIRE(n >= 2 && n <= 12, "grid size out of range");
         const int m = T.cube_panel_ptr[c + 1] - T.cube_panel_ptr[c];
         const int r = T.cube_row_rank[c];
         const int ninter = T.inter_ptr[c + 1] - T.inter_ptr[c];
         if (m <= 0 || r <= 0 || ninter <= 0) continue;
         const int n3 = n * n * n, Np = 2 * n - 1, pg = Np * Np * n;
         FFTSVD_REQUIRE(T.cube_vt_ptr[c + 1] - T.cube_vt_ptr[c] == (int64_t)r * m, "VT size mismatch");
         FFTSVD_REQUIRE(T.cube_pv_ptr[c + 1] - T.cube_pv_ptr[c] == (int64_t)r * n3, "PV size mismatch");
         FFTSVD_REQUIRE(r <= 1024, "row rank too large");
         SrcDesc s;
         s.n = n; s.m = m; s.r = r;
         s.panel_off = (int32_t)L.src_panels.size();
         s.vt_off = (int64_t)L.vt.size();
         s.pv_off = (int64_t)(L.pv_pairs.size() / 2);
         s.spec_off = L.spectra_elems;
         spec_of_cube[c] = L.spectra_elems;
         L.spectra_elems += pg;
         for (int i = T.cube_panel_ptr[c]; i < T.cube_panel_ptr[c + 1]; i++) {
            FFTSVD_REQUIRE(T.cube_panels[i] >= 0 && T.cube_panels[i] < T.num_panels, "cube panel out of range");
            L.src_panels.push_back((int32_t)(po + T.cube_panels[i]));
         }
         const int64_t vb = T.cube_vt_ptr[c];
         L.vt.insert(L.vt.end(), T.vt + vb, T.vt + vb + (int64_t)r * m);
         const int64_t pb = T.cube_pv_ptr[c];
         for (int j = 0; j < r; j++)
            for (int p = 0; p < n3; p++) {
               L.pv_pairs.push_back(T.pv_single[pb + (int64_t)p * r + j]);
               L.pv_pairs.push_back(T.pv_double[pb + (int64_t)p * r + j]);
            }
         L.operator_elems += (int64_t)r * m + 2LL * r * n3;
         const int ch = std::min(m, 1024);
         const int H = n;
         int need = 2 * ch + 2 * r + n3 + 2 * Np + 2 * (n * n * H) + 2 * (n * Np * H) + 16;
         L.max_src_smem_elems = std::max(L.max_src_smem_elems, need);
         L.src.push_back(s);
      }
      for (int c = 0; c < T.num_cubes; c++) {
         const int lvl = T.cube_level[c];
         const int n = T.grid[lvl];
         const int p = T.cube_point_ptr[c + 1] - T.cube_point_ptr[c];
         const int r = T.cube_col_rank[c];
         if (p <= 0 || r <= 0) continue;
         const int n3 = n * n * n, Np = 2 * n - 1, pg = Np * Np * n, H = n;
         FFTSVD_REQUIRE(T.cube_uti_ptr[c + 1] - T.cube_uti_ptr[c] == (int64_t)r * n3, "UTI size mismatch");
         FFTSVD_REQUIRE(T.cube_u_ptr[c + 1] - T.cube_u_ptr[c] == (int64_t)r * p, "U size mismatch");
         FFTSVD_REQUIRE(r <= 1024, "column rank too large");
         DstDesc d;
         d.n = n; d.p = p; d.r = r;
         d.point_off = (int32_t)L.dst_points.size();
         d.uti_off = (int64_t)L.uti.size();
         d.u_off = (int64_t)L.u_cm.size();
         d.inter_off = (int32_t)(L.inter_pairs.size() / 2);
         d.stage = lvl;
         d.pad = 0;
         for (int i = T.cube_point_ptr[c]; i < T.cube_point_ptr[c + 1]; i++) {
            FFTSVD_REQUIRE(T.cube_points[i] >= 0 && T.cube_points[i] < T.num_points, "cube point out of range");
            L.dst_points.push_back((int32_t)(qo + T.cube_points[i]));
         }
         const int64_t ub = T.cube_uti_ptr[c];
         L.uti.insert(L.uti.end(), T.uti + ub, T.uti + ub + (int64_t)r * n3);
         const int64_t uub = T.cube_u_ptr[c];
         for (int j = 0; j < r; j++)
            for (int q = 0; q < p; q++) L.u_cm.push_back(T.u[uub + (int64_t)q * r + j]);
         L.operator_elems += (int64_t)r * n3 + (int64_t)p * r;
         int cnt = 0;
         for (int i = T.inter_ptr[c]; i < T.inter_ptr[c + 1]; i++) {
            const int s = T.inter_cubes[i];
            FFTSVD_REQUIRE(s >= 0 && s < T.num_cubes, "interacting cube out of range");
            if (spec_of_cube[s] < 0) continue;  // source without panels or rank: contributes zero
            FFTSVD_REQUIRE(T.cube_level[s] == lvl, "interaction across levels");
            const int dx = T.cube_index[3 * c] - T.cube_index[3 * s];
            const int dy = T.cube_index[3 * c + 1] - T.cube_index[3 * s + 1];
            const int dz = T.cube_index[3 * c + 2] - T.cube_index[3 * s + 2];
            FFTSVD_REQUIRE(std::abs(dx) <= 3 && std::abs(dy) <= 3 && std::abs(dz) <= 3, "interaction offset too large");
            FFTSVD_REQUIRE(std::abs(dx) > 1 || std::abs(dy) > 1 || std::abs(dz) > 1, "local cube in interaction list");
            const int slot = ((dx + 3) * 7 + (dy + 3)) * 7 + (dz + 3);
            const int64_t toff = t_base + T.t_level_ptr[lvl] + (int64_t)slot * pg;
            FFTSVD_REQUIRE(T.t_level_ptr[lvl + 1] - T.t_level_ptr[lvl] == 343LL * pg, "translation table size mismatch");
            L.inter_pairs.push_back(spec_of_cube[s]);
            L.inter_pairs.push_back(toff);
            cnt++;
         }
         d.inter_cnt = cnt;
         int need = 2 * pg + 2 * (n * Np * H) + 2 * (n * n * H) + n3 + r + 2 * Np + 16;
         L.max_dst_smem_elems = std::max(L.max_dst_smem_elems, need);
         if (cnt > 0) L.dst.push_back(d);
         else L.uti.resize(d.uti_off), L.u_cm.resize(d.u_off), L.dst_points.resize(d.point_off);
      }
      // translation operators of this tree (unique tables: 316 non-local offsets per level)
      const int64_t nt = T.t_level_ptr[T.depth];
      L.t_pairs.insert(L.t_pairs.end(), T.t_ops, T.t_ops + 2 * nt);
      for (int lvl = 0; lvl < T.depth; lvl++) {
         const int n = T.grid[lvl], Np = 2 * n - 1;
         L.t_elems += 2LL * 316 * Np * Np * n;
      }
   }
   for (int o = 0; o < num_unknowns; o++)
      if (!row_written[o]) L.full_cover = false;

   // every index a kernel will form stays inside its buffer
   const int64_t npairs_d = (int64_t)L.d_pairs.size() / 2, npv = (int64_t)L.pv_pairs.size() / 2;
   const int64_t nt = (int64_t)L.t_pairs.size() / 2;
   for (const LeafDesc& d : L.leaves) {
      FFTSVD_REQUIRE(d.nrows > 0 && d.ncols >= 0 && d.ncols % 2 == 0 && d.d_off % 2 == 0, "leaf descriptor");
      FFTSVD_REQUIRE(d.row_off + (int64_t)d.nrows <= (int64_t)L.leaf_rows.size(), "leaf rows out of range");
      FFTSVD_REQUIRE(d.col_off + (int64_t)d.ncols <= (int64_t)L.leaf_cols.size(), "leaf cols out of range");
      FFTSVD_REQUIRE(d.d_off + (int64_t)d.nrows * d.ncols <= npairs_d, "leaf block out of range");
   }
   for (int32_t v : L.leaf_rows) FFTSVD_REQUIRE(v >= 0 && v < L.total_points, "leaf row index");
   for (int32_t v : L.leaf_cols) FFTSVD_REQUIRE(v >= 0 && v < L.total_panels, "leaf col index");
   for (const SrcDesc& s : L.src) {
      const int64_t n3 = (int64_t)s.n * s.n * s.n, pg = (int64_t)(2 * s.n - 1) * (2 * s.n - 1) * s.n;
      FFTSVD_REQUIRE(s.panel_off + (int64_t)s.m <= (int64_t)L.src_panels.size(), "source panels out of range");
      FFTSVD_REQUIRE(s.vt_off + (int64_t)s.r * s.m <= (int64_t)L.vt.size(), "VT out of range");
      FFTSVD_REQUIRE(s.pv_off + (int64_t)s.r * n3 <= npv, "PV out of range");
      FFTSVD_REQUIRE(s.spec_off + pg <= L.spectra_elems, "spectrum out of range");
   }
   for (int32_t v : L.src_panels) FFTSVD_REQUIRE(v >= 0 && v < L.total_panels, "source panel index");
   for (const DstDesc& d : L.dst) {
      const int64_t n3 = (int64_t)d.n * d.n * d.n, pg = (int64_t)(2 * d.n - 1) * (2 * d.n - 1) * d.n;
      FFTSVD_REQUIRE(d.point_off + (int64_t)d.p <= (int64_t)L.dst_points.size(), "destination points out of range");
      FFTSVD_REQUIRE(d.uti_off + (int64_t)d.r * n3 <= (int64_t)L.uti.size(), "UTI out of range");
      FFTSVD_REQUIRE(d.u_off + (int64_t)d.r * d.p <= (int64_t)L.u_cm.size(), "U out of range");
      FFTSVD_REQUIRE(d.stage >= 0 && d.stage < L.stage_levels, "staging level out of range");
      FFTSVD_REQUIRE(2LL * (d.inter_off + (int64_t)d.inter_cnt) <= (int64_t)L.inter_pairs.size(), "interactions out of range");
      for (int q = 0; q < d.inter_cnt; q++) {
         const int64_t so = L.inter_pairs[2 * (d.inter_off + q)], to = L.inter_pairs[2 * (d.inter_off + q) + 1];
         FFTSVD_REQUIRE(so >= 0 && so + pg <= L.spectra_elems, "interaction spectrum out of range");
         FFTSVD_REQUIRE(to >= 0 && to + pg <= nt, "translation operator out of range");
      }
   }
   for (int32_t v : L.dst_points) FFTSVD_REQUIRE(v >= 0 && v < L.total_points, "destination point index");
   for (int64_t k = 0; k < (int64_t)L.point_out.size(); k++) {
      FFTSVD_REQUIRE(L.point_out[k] >= 0 && L.point_out[k] < num_unknowns, "point without an output row");
      FFTSVD_REQUIRE(L.point_panel[k] >= -1 && L.point_panel[k] < L.total_panels - 1, "jump panel index");
   }
   // algorithmic bytes per kernel (each operator element, spectrum and vector entry counted once)
   {
      KernelBytes& kb = L.kernel_bytes;
      const double np = (double)(L.total_panels - 1), nq = (double)L.total_points;
      kb.fixed[0] = np * (8.0 + 2 * 4.0 + 2 * 8.0);  // x reads, two indices, two scales
      kb.elems[0] = 2.0 * np;                         // {xs, xd} writes
      double vt = 0, pv = 0, spec = 0, uti = 0, u = 0, dpairs = 0, lcols = 0, lrows = 0;
      for (const SrcDesc& sd : L.src) {
         vt += (double)sd.r * sd.m;
         pv += 2.0 * sd.r * sd.n * sd.n * sd.n;
         spec += 2.0 * (2 * sd.n - 1) * (2 * sd.n - 1) * sd.n;
      }
      for (const DstDesc& dd : L.dst) {
         uti += (double)dd.r * dd.n * dd.n * dd.n;
         u += (double)dd.r * dd.p;
      }
      for (const LeafDesc& ld : L.leaves) {
         dpairs += 2.0 * ld.nrows * ld.ncols;
         lcols += ld.ncols;
         lrows += ld.nrows;
      }
      kb.elems[1] = vt + pv + spec + 2.0 * (double)L.src_panels.size();  // + gathered {xs, xd}
      kb.fixed[1] = 4.0 * (double)L.src_panels.size();
      kb.elems[2] = spec + (double)L.t_elems + uti + u + nq;              // spectra, T, UTI, U, staging writes
      kb.fixed[2] = 4.0 * (double)L.dst_points.size() + 16.0 * (double)(L.inter_pairs.size() / 2);
      kb.elems[3] = dpairs + 2.0 * lcols + (double)L.stage_levels * nq;   // D, gathered x, staged far field
      kb.fixed[3] = 4.0 * (lcols + lrows) + nq * (8.0 + 4.0 + 4.0 + 8.0); // indices, y, maps, jump
   }
   // group by grid size (largest first), heavy cubes first within a group so the
   // long blocks start early; each group is one launch with its own shared memory
   std::stable_sort(L.src.begin(), L.src.end(), [](const SrcDesc& a, const SrcDesc& b) {
      if (a.n != b.n) return a.n > b.n;
      return (int64_t)a.r * a.m > (int64_t)b.r * b.m;
   });
   std::stable_sort(L.dst.begin(), L.dst.end(), [](const DstDesc& a, const DstDesc& b) {
      if (a.n != b.n) return a.n > b.n;
      return (int64_t)a.inter_cnt * a.r > (int64_t)b.inter_cnt * b.r;
   });
   auto src_need = [](const SrcDesc& s) {
      const int n = s.n, Np = 2 * n - 1, H = n, ch = std::min(s.m, 1024);
      return 2 * ch + 2 * s.r + n * n * n + 2 * Np + 2 * (n * n * H) + 2 * (n * Np * H) + 16;
   };
   auto dst_need = [](const DstDesc& d) {
      const int n = d.n, Np = 2 * n - 1, H = n, pg = Np * Np * H;
      return 2 * pg + 2 * (n * Np * H) + 2 * (n * n * H) + n * n * n + d.r + 2 * Np + 16;
   };
   for (int i = 0; i < (int)L.src.size(); i++) {
      if (L.src_groups.empty() || L.src_groups.back().n != L.src[i].n) L.src_groups.push_back({L.src[i].n, i, 0, 0});
      LaunchGroup& g = L.src_groups.back();
      g.count++;
      g.smem_elems = std::max(g.smem_elems, src_need(L.src[i]));
   }
   for (int i = 0; i < (int)L.dst.size(); i++) {
      if (L.dst_groups.empty() || L.dst_groups.back().n != L.dst[i].n) L.dst_groups.push_back({L.dst[i].n, i, 0, 0});
      LaunchGroup& g = L.dst_groups.back();
      g.count++;
      g.smem_elems = std::max(g.smem_elems, dst_need(L.dst[i]));
   }
   return L;
}

// ------------------------------------------------------------------ device helpers

template <typename T> struct Cx;
template <> struct Cx<float> {
   using T2 = float2;
   __device__ static inline T2 mul(T2 a, T2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
   __device__ static inline T2 fma(T2 a, T2 b, T2 c) {  // a*b + c
      return make_float2(fmaf(a.x, b.x, fmaf(-a.y, b.y, c.x)), fmaf(a.x, b.y, fmaf(a.y, b.x, c.y)));
   }
   __device__ static inline T2 make(float x, float y) { return make_float2(x, y); }
   __device__ static inline void cis(int m, int N, float* c, float* s) {  // exp(+2 pi i m / N)
      sincospif(2.0f * (float)m / (float)N, s, c);
   }
};
template <> struct Cx<double> {
   using T2 = double2;
   __device__ static inline T2 mul(T2 a, T2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
   __device__ static inline T2 fma(T2 a, T2 b, T2 c) {
      return make_double2(::fma(a.x, b.x, ::fma(-a.y, b.y, c.x)), ::fma(a.x, b.y, ::fma(a.y, b.x, c.y)));
   }
   __device__ static inline T2 make(double x, double y) { return make_double2(x, y); }
   __device__ static inline void cis(int m, int N, double* c, double* s) {
      sincospi(2.0 * (double)m / (double)N, s, c);
   }
};

template <typename T>
__device__ inline T warp_sum(T v) {
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
   return v;
}

template <typename T>
__device__ inline T* carve(char*& p, int count) {
   uintptr_t a = reinterpret_cast<uintptr_t>(p);
   a = (a + 15) & ~uintptr_t(15);
   T* out = reinterpret_cast<T*>(a);
   p = reinterpret_cast<char*>(a + sizeof(T) * (size_t)count);
   return out;
}

// ------------------------------------------------------------------ kernels

// xsd[k] = {dphi_scale[k] * x[dphi_index[k]], phi_scale[k] * x[phi_index[k]]}
template <typename T>
__global__ void join_kernel(int64_t total, const int32_t* __restrict__ phi_idx, const double* __restrict__ phi_scale,
                            const int32_t* __restrict__ dphi_idx, const double* __restrict__ dphi_scale,
                            const double* __restrict__ x, typename Vec2<T>::type* __restrict__ xsd) {
   using T2 = typename Vec2<T>::type;
   for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
      T2 v;
      v.x = (T)(dphi_scale[k] * x[dphi_idx[k]]);
      v.y = (T)(phi_scale[k] * x[phi_idx[k]]);
      xsd[k] = v;
   }
}

constexpr int kFarThreads = 128;
constexpr int kChunk = 1024;

// One block per source cube: a = VT x (both layers), g = PV_s a_s + PV_d a_d on
// the n^3 grid, F = r2c DFT of g placed at offset n/2 in the (2n-1)^3 box.
template <typename T>
__global__ void __launch_bounds__(kFarThreads) far_forward_kernel(
    const SrcDesc* __restrict__ cubes, const int32_t* __restrict__ src_panels,
    const typename Vec2<T>::type* __restrict__ xsd, const T* __restrict__ vt,
    const typename Vec2<T>::type* __restrict__ pv, typename Vec2<T>::type* __restrict__ spectra) {
   using T2 = typename Vec2<T>::type;
   extern __shared__ __align__(16) char smem_raw[];
   const SrcDesc c = cubes[blockIdx.x];
   const int n = c.n, Np = 2 * n - 1, H = n, off = n / 2, n3 = n * n * n;
   const int m = c.m, r = c.r;
   const int ch = min(m, kChunk);
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;

   char* p = smem_raw;
   T* xs = carve<T>(p, ch);
   T* xd = carve<T>(p, ch);
   T* as = carve<T>(p, r);
   T* ad = carve<T>(p, r);
   T* g = carve<T>(p, n3);
   T2* tw = carve<T2>(p, Np);
   T2* A = carve<T2>(p, n * n * H);
   T2* B = carve<T2>(p, n * Np * H);

   for (int j = tid; j < r; j += blockDim.x) { as[j] = T(0); ad[j] = T(0); }
   for (int k = tid; k < Np; k += blockDim.x) {  // exp(-2 pi i k / Np)
      T cs, sn;
      Cx<T>::cis(k, Np, &cs, &sn);
      tw[k] = Cx<T>::make(cs, -sn);
   }
   // VT x, streamed over panel chunks; each row is owned by one warp
   for (int base = 0; base < m; base += ch) {
      const int cnt = min(ch, m - base);
      __syncthreads();
      for (int i = tid; i < cnt; i += blockDim.x) {
         T2 v = xsd[src_panels[c.panel_off + base + i]];
         xs[i] = v.x;
         xd[i] = v.y;
      }
      __syncthreads();
      for (int j = warp; j < r; j += nwarps) {
         const T* row = vt + c.vt_off + (int64_t)j * m + base;
         T s = T(0), d = T(0);
         for (int i = lane; i < cnt; i += 32) {
            T v = row[i];
            s += v * xs[i];
            d += v * xd[i];
         }
         s = warp_sum(s);
         d = warp_sum(d);
         if (lane == 0) { as[j] += s; ad[j] += d; }
      }
   }
   __syncthreads();
   // grid charges
   for (int q = tid; q < n3; q += blockDim.x) {
      const T2* col = pv + c.pv_off + q;
      T acc = T(0);
      for (int j = 0; j < r; j++) {
         T2 w = col[(int64_t)j * n3];
         acc += w.x * as[j] + w.y * ad[j];
      }
      g[q] = acc;
   }
   __syncthreads();
   // DFT along k (input index k + off), half spectrum kf < H
   for (int idx = tid; idx < n * n * H; idx += blockDim.x) {
      const int kf = idx % H, ij = idx / H;
      const T* line = g + ij * n;
      T2 acc = Cx<T>::make(T(0), T(0));
      for (int k = 0; k < n; k++) {
         T2 w = tw[((k + off) * kf) % Np];
         acc.x += line[k] * w.x;
         acc.y += line[k] * w.y;
      }
      A[idx] = acc;
   }
   __syncthreads();
   // along j
   for (int idx = tid; idx < n * Np * H; idx += blockDim.x) {
      const int kf = idx % H, jf = (idx / H) % Np, i = idx / (H * Np);
      T2 acc = Cx<T>::make(T(0), T(0));
      for (int j = 0; j < n; j++) acc = Cx<T>::fma(A[(i * n + j) * H + kf], tw[((j + off) * jf) % Np], acc);
      B[idx] = acc;
   }
   __syncthreads();
   // along i, straight to global
   T2* out = spectra + c.spec_off;
   for (int idx = tid; idx < Np * Np * H; idx += blockDim.x) {
      const int kf = idx % H, jf = (idx / H) % Np, fi = idx / (H * Np);
      T2 acc = Cx<T>::make(T(0), T(0));
      for (int i = 0; i < n; i++) acc = Cx<T>::fma(B[(i * Np + jf) * H + kf], tw[((i + off) * fi) % Np], acc);
      out[idx] = acc;
   }
}

// One block per destination cube: S = sum over interacting sources of
// T[offset] .* F_source, c2r DFT cropped at offset n/2 and scaled by 1/(2n-1)^3,
// u = UTI g, values U u written to this level's staging row of each point.
template <typename T>
__global__ void __launch_bounds__(kFarThreads) far_backward_kernel(
    const DstDesc* __restrict__ cubes, const int32_t* __restrict__ dst_points, const longlong2* __restrict__ inter,
    const typename Vec2<T>::type* __restrict__ tops, const typename Vec2<T>::type* __restrict__ spectra,
    const T* __restrict__ uti, const T* __restrict__ ucm, T* __restrict__ staging, int64_t total_points) {
   using T2 = typename Vec2<T>::type;
   extern __shared__ __align__(16) char smem_raw[];
   const DstDesc c = cubes[blockIdx.x];
   const int n = c.n, Np = 2 * n - 1, H = n, off = n / 2, n3 = n * n * n, pg = Np * Np * H;
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;

   char* p = smem_raw;
   T2* S = carve<T2>(p, pg);
   T2* P1 = carve<T2>(p, n * Np * H);
   T2* P2 = carve<T2>(p, n * n * H);
   T* g = carve<T>(p, n3);
   T* u = carve<T>(p, c.r);
   T2* tw = carve<T2>(p, Np);

   for (int k = tid; k < Np; k += blockDim.x) {  // exp(+2 pi i k / Np)
      T cs, sn;
      Cx<T>::cis(k, Np, &cs, &sn);
      tw[k] = Cx<T>::make(cs, sn);
   }
   // translation: accumulate over sources, frequencies across threads
   for (int f = tid; f < pg; f += blockDim.x) {
      T2 acc = Cx<T>::make(T(0), T(0));
      for (int q = 0; q < c.inter_cnt; q++) {
         const longlong2 pr = inter[c.inter_off + q];
         acc = Cx<T>::fma(tops[pr.y + f], spectra[pr.x + f], acc);
      }
      S[f] = acc;
   }
   __syncthreads();
   // inverse along i (output i < n only)
   for (int idx = tid; idx < n * Np * H; idx += blockDim.x) {
      const int kf = idx % H, jf = (idx / H) % Np, i = idx / (H * Np);
      T2 acc = Cx<T>::make(T(0), T(0));
      for (int fi = 0; fi < Np; fi++) acc = Cx<T>::fma(S[(fi * Np + jf) * H + kf], tw[((i + off) * fi) % Np], acc);
      P1[idx] = acc;
   }
   __syncthreads();
   // inverse along j (output j < n only)
   for (int idx = tid; idx < n * n * H; idx += blockDim.x) {
      const int kf = idx % H, j = (idx / H) % n, i = idx / (H * n);
      T2 acc = Cx<T>::make(T(0), T(0));
      for (int jf = 0; jf < Np; jf++) acc = Cx<T>::fma(P1[(i * Np + jf) * H + kf], tw[((j + off) * jf) % Np], acc);
      P2[idx] = acc;
   }
   __syncthreads();
   // Hermitian half along k -> real, cropped, scaled
   const T scale = T(1) / (T)(Np * Np * Np);
   for (int q = tid; q < n3; q += blockDim.x) {
      const int k = q % n, ij = q / n;
      const T2* line = P2 + ij * H;
      T acc = line[0].x;
      for (int kf = 1; kf < H; kf++) {
         T2 w = tw[((k + off) * kf) % Np];
         acc += T(2) * (line[kf].x * w.x - line[kf].y * w.y);
      }
      g[q] = acc * scale;
   }
   __syncthreads();
   // u = UTI g
   for (int j = warp; j < c.r; j += nwarps) {
      const T* row = uti + c.uti_off + (int64_t)j * n3;
      T s = T(0);
      for (int q = lane; q < n3; q += 32) s += row[q] * g[q];
      s = warp_sum(s);
      if (lane == 0) u[j] = s;
   }
   __syncthreads();
   // U u -> staging (each point belongs to exactly one cube of this level)
   T* stage = staging + (int64_t)c.stage * total_points;
   for (int q = tid; q < c.p; q += blockDim.x) {
      const T* col = ucm + c.u_off + q;
      T acc = T(0);
      for (int j = 0; j < c.r; j++) acc += col[(int64_t)j * c.p] * u[j];
      stage[dst_points[c.point_off + q]] = acc;
   }
}

constexpr int kNearThreads = 128;

template <typename T> struct NearLoad;
template <> struct NearLoad<float> {
   // two columns {Ds, Dd, Ds, Dd} in one 16-byte load
   __device__ static inline float dot2(const float2* row, int c, const float2* x) {
      float4 v = *reinterpret_cast<const float4*>(row + c);
      float2 a = x[c], b = x[c + 1];
      return v.x * a.x + v.y * a.y + v.z * b.x + v.w * b.y;
   }
};
template <> struct NearLoad<double> {
   __device__ static inline double dot2(const double2* row, int c, const double2* x) {
      double2 v0 = row[c], v1 = row[c + 1];
      double2 a = x[c], b = x[c + 1];
      return v0.x * a.x + v0.y * a.y + v1.x * b.x + v1.y * b.y;
   }
};

// One block per leaf: y[out(p)] = (D_s xs + D_d xd)[p] + sum_levels staging[p] + jump(p) xd(p).
template <typename T>
__global__ void __launch_bounds__(kNearThreads) near_kernel(
    const LeafDesc* __restrict__ leaves, const int32_t* __restrict__ rows, const int32_t* __restrict__ cols,
    const typename Vec2<T>::type* __restrict__ d, const typename Vec2<T>::type* __restrict__ xsd,
    const T* __restrict__ staging, int stage_levels, int64_t total_points, const int32_t* __restrict__ point_out,
    const int32_t* __restrict__ point_panel, const double* __restrict__ point_jump,
    const int32_t* __restrict__ phi_idx, const double* __restrict__ phi_scale, const double* __restrict__ x,
    double* __restrict__ y) {
   using T2 = typename Vec2<T>::type;
   extern __shared__ __align__(16) char smem_raw[];
   const LeafDesc L = leaves[blockIdx.x];
   T2* xl = reinterpret_cast<T2*>(smem_raw);
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
   for (int i = tid; i < L.ncols; i += blockDim.x) xl[i] = xsd[cols[L.col_off + i]];
   __syncthreads();
   for (int rr = warp; rr < L.nrows; rr += nwarps) {
      const T2* row = d + L.d_off + (int64_t)rr * L.ncols;
      T acc = T(0);
      for (int c = 2 * lane; c < L.ncols; c += 64) acc += NearLoad<T>::dot2(row, c, xl);
      acc = warp_sum(acc);
      if (lane == 0) {
         const int pnt = rows[L.row_off + rr];
         double v = (double)acc;
         for (int l = 0; l < stage_levels; l++) v += (double)staging[(int64_t)l * total_points + pnt];
         const int k = point_panel[pnt];
         if (k >= 0) v += point_jump[pnt] * (phi_scale[k] * x[phi_idx[k]]);
         y[point_out[pnt]] = v;
      }
   }
}

// ------------------------------------------------------------------ host side

template <typename T>
static void upload_cast(DevBuf<T>& dst, const std::vector<double>& src) {
   std::vector<T> tmp(src.begin(), src.end());
   dst.upload(tmp);
}

template <typename T>
static void upload_pairs(DevBuf<typename Vec2<T>::type>& dst, const std::vector<double>& src) {
   using T2 = typename Vec2<T>::type;
   std::vector<T2> tmp(src.size() / 2);
   for (size_t i = 0; i < tmp.size(); i++) {
      tmp[i].x = (T)src[2 * i];
      tmp[i].y = (T)src[2 * i + 1];
   }
   dst.upload(tmp);
}

template <typename T>
void DeviceOperator<T>::upload(const OperatorLayout& L) {
   num_unknowns_ = L.num_unknowns;
   total_panels_ = L.total_panels;
   total_points_ = L.total_points;
   stage_levels_ = L.stage_levels;
   full_cover_ = L.full_cover;
   n_src_ = (int)L.src.size();
   n_dst_ = (int)L.dst.size();
   n_leaf_ = (int)L.leaves.size();
   join_phi_idx_.upload(L.join_phi_idx);
   join_dphi_idx_.upload(L.join_dphi_idx);
   join_phi_scale_.upload(L.join_phi_scale);
   join_dphi_scale_.upload(L.join_dphi_scale);
   xsd_.alloc(L.total_panels);
   xsd_.zero();
   point_out_.upload(L.point_out);
   point_panel_.upload(L.point_panel);
   point_jump_.upload(L.point_jump);
   leaves_.upload(L.leaves);
   leaf_rows_.upload(L.leaf_rows);
   leaf_cols_.upload(L.leaf_cols);
   upload_pairs<T>(d_, L.d_pairs);
   src_.upload(L.src);
   src_panels_.upload(L.src_panels);
   upload_cast<T>(vt_, L.vt);
   upload_pairs<T>(pv_, L.pv_pairs);
   dst_.upload(L.dst);
   dst_points_.upload(L.dst_points);
   upload_cast<T>(uti_, L.uti);
   upload_cast<T>(u_, L.u_cm);
   {
      std::vector<longlong2> ip(L.inter_pairs.size() / 2);
      for (size_t i = 0; i < ip.size(); i++) { ip[i].x = L.inter_pairs[2 * i]; ip[i].y = L.inter_pairs[2 * i + 1]; }
      inter_.upload(ip);
   }
   upload_pairs<T>(t_, L.t_pairs);
   spectra_.alloc(std::max<int64_t>(L.spectra_elems, 1));
   staging_.alloc(std::max<int64_t>((int64_t)L.stage_levels * L.total_points, 1));
   staging_.zero();
   // entries of the zero slot and staging rows nobody writes must stay zero
   src_groups_ = L.src_groups;
   dst_groups_ = L.dst_groups;
   src_smem_ = 0;
   dst_smem_ = 0;
   for (const LaunchGroup& g : src_groups_) src_smem_ = std::max(src_smem_, (int)(g.smem_elems * sizeof(T) + 128));
   for (const LaunchGroup& g : dst_groups_) dst_smem_ = std::max(dst_smem_, (int)(g.smem_elems * sizeof(T) + 128));
   int maxcols = 0;
   for (const auto& l : L.leaves) maxcols = std::max(maxcols, l.ncols);
   leaf_smem_max_ = (int)(maxcols * sizeof(T2) + 16);
   int dev = 0, optin = 0;
   FFTSVD_CUDA(cudaGetDevice(&dev));
   FFTSVD_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
   if (src_smem_ > optin || dst_smem_ > optin || leaf_smem_max_ > optin)
      throw Error(FFTSVD_ERR_UNSUPPORTED, "operator block needs more shared memory than the device offers");
   FFTSVD_CUDA(cudaFuncSetAttribute(far_forward_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, src_smem_));
   FFTSVD_CUDA(cudaFuncSetAttribute(far_backward_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, dst_smem_));
   FFTSVD_CUDA(cudaFuncSetAttribute(near_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, leaf_smem_max_));
   FFTSVD_CUDA(cudaDeviceSynchronize());
}

template <typename T>
void DeviceOperator<T>::enable_timing(bool on) {
   if (on && !ev_[0])
      for (auto& e : ev_) FFTSVD_CUDA(cudaEventCreate(&e));
   timing_ = on;
}

template <typename T>
void DeviceOperator<T>::stage_ms(float* join_ms, float* fwd_ms, float* bwd_ms, float* near_ms) const {
   *join_ms = *near_ms = *fwd_ms = *bwd_ms = 0.f;
   if (!ev_[0]) return;
   FFTSVD_CUDA(cudaEventSynchronize(ev_[4]));
   FFTSVD_CUDA(cudaEventElapsedTime(join_ms, ev_[0], ev_[1]));
   FFTSVD_CUDA(cudaEventElapsedTime(fwd_ms, ev_[1], ev_[2]));
   FFTSVD_CUDA(cudaEventElapsedTime(bwd_ms, ev_[2], ev_[3]));
   FFTSVD_CUDA(cudaEventElapsedTime(near_ms, ev_[3], ev_[4]));
}

template <typename T>
void DeviceOperator<T>::apply(const double* x, double* y, cudaStream_t stream) {
   if (timing_) FFTSVD_CUDA(cudaEventRecord(ev_[0], stream));
   if (!full_cover_) FFTSVD_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * num_unknowns_, stream));
   {
      const int64_t total = total_panels_ - 1;  // the zero slot is never written
      int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
      if (blocks < 1) blocks = 1;
      join_kernel<T><<<blocks, 256, 0, stream>>>(total, join_phi_idx_.get(), join_phi_scale_.get(),
                                                 join_dphi_idx_.get(), join_dphi_scale_.get(), x, xsd_.get());
      FFTSVD_CHECK_LAUNCH();
   }
   if (timing_) FFTSVD_CUDA(cudaEventRecord(ev_[1], stream));
   for (const LaunchGroup& g : src_groups_) {
      const int smem = (int)(g.smem_elems * sizeof(T) + 128);
      far_forward_kernel<T><<<g.count, kFarThreads, smem, stream>>>(src_.get() + g.begin, src_panels_.get(),
                                                                    xsd_.get(), vt_.get(), pv_.get(), spectra_.get());
      FFTSVD_CHECK_LAUNCH();
   }
   if (timing_) FFTSVD_CUDA(cudaEventRecord(ev_[2], stream));
   for (const LaunchGroup& g : dst_groups_) {
      const int smem = (int)(g.smem_elems * sizeof(T) + 128);
      far_backward_kernel<T><<<g.count, kFarThreads, smem, stream>>>(
          dst_.get() + g.begin, dst_points_.get(), inter_.get(), t_.get(), spectra_.get(), uti_.get(), u_.get(),
          staging_.get(), total_points_);
      FFTSVD_CHECK_LAUNCH();
   }
   if (timing_) FFTSVD_CUDA(cudaEventRecord(ev_[3], stream));
   if (n_leaf_ > 0) {
      near_kernel<T><<<n_leaf_, kNearThreads, leaf_smem_max_, stream>>>(
          leaves_.get(), leaf_rows_.get(), leaf_cols_.get(), d_.get(), xsd_.get(), staging_.get(), stage_levels_,
          total_points_, point_out_.get(), point_panel_.get(), point_jump_.get(), join_phi_idx_.get(),
          join_phi_scale_.get(), x, y);
      FFTSVD_CHECK_LAUNCH();
   }
   if (timing_) FFTSVD_CUDA(cudaEventRecord(ev_[4], stream));
}

template <typename T>
size_t DeviceOperator<T>::device_bytes() const {
   return join_phi_idx_.bytes() + join_dphi_idx_.bytes() + join_phi_scale_.bytes() + join_dphi_scale_.bytes() +
          xsd_.bytes() + point_out_.bytes() + point_panel_.bytes() + point_jump_.bytes() + leaves_.bytes() +
          leaf_rows_.bytes() + leaf_cols_.bytes() + d_.bytes() + src_.bytes() + src_panels_.bytes() +
          vt_.bytes() + pv_.bytes() + dst_.bytes() + dst_points_.bytes() + uti_.bytes() + u_.bytes() +
          inter_.bytes() + t_.bytes() + spectra_.bytes() + staging_.bytes();
}

template class DeviceOperator<float>;
template class DeviceOperator<double>;

}  // namespace fftsvd
