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
#include <cstdlib>
#include <cstring>
#include <array>
#include <map>
#include <mutex>
#include <unordered_map>
#include <exception>
#include <type_traits>
#include <numeric>
#include <string>

#include "operator.h"

namespace fftsvd {

// ------------------------------------------------------------------ layout

static int pad2(int v) { return (v + 1) & ~1; }
static int pad16(int v) { return (v + 15) & ~15; }

void TileProblem::add_output(int k, uint64_t code, int64_t tb, int pgp, int64_t out) {
   key.push_back(k);
   morton.push_back(code);
   t_base.push_back(tb);
   pg.push_back(pgp);
   out_off.push_back(out);
   ptr.push_back(ptr.back());
}

void TileProblem::add_pair(int64_t in, int s) {
   in_off.push_back(in);
   slot.push_back(s);
   ptr.back()++;
}

// Cube coordinates from a Morton code (bit 3b + k of the code is bit b of coordinate k).
static void morton_decode(uint64_t code, int c[3]) {
   c[0] = c[1] = c[2] = 0;
   for (int b = 0; b < 21; b++)
      for (int k = 0; k < 3; k++) c[k] |= (int)((code >> (3 * b + k)) & 1) << b;
}

namespace {
// Sibling outputs sharing one list of sources: per source its base slot (the slot of
// member 0) and the mask of the members that interact with it.
struct MemberGroup {
   std::vector<int> members;   // output ids
   std::vector<int> delta;     // slot of member j = base + delta[j]
   std::vector<int64_t> src;   // input offsets, first-seen order
   std::vector<uint32_t> mask;
   std::vector<int> base;
};

constexpr int kCenterSlot = 171;  // offset (0, 0, 0)

int slot_of(const int v[3]) { return ((v[0] + 3) * 7 + (v[1] + 3)) * 7 + (v[2] + 3); }

// Members [first, last) of ids (siblings in Morton order) as one group.  Returns false
// when the shared source list would not be exact for every member: each member's
// offset to each source of the union must lie in [-3, 3]^3, and a member that does not
// interact with a source must be its neighbour (its slot is then one of the zeroed
// local-offset rows).
bool make_group(const TileProblem& P, const std::vector<int>& ids, size_t first, size_t last, MemberGroup& G) {
   G = MemberGroup();
   std::vector<std::array<int, 3>> pos;
   for (size_t i = first; i < last; i++) {
      int c[3];
      morton_decode(P.morton[ids[i]], c);
      pos.push_back({c[0], c[1], c[2]});
   }
   std::unordered_map<int64_t, int> where;
   where.reserve(256);
   std::vector<std::array<int, 3>> v0;  // offset of member 0 to each source
   for (size_t m = 0; m < pos.size(); m++) {
      const int o = ids[first + m];
      const int dp[3] = {pos[m][0] - pos[0][0], pos[m][1] - pos[0][1], pos[m][2] - pos[0][2]};
      G.members.push_back(o);
      G.delta.push_back(dp[0] * 49 + dp[1] * 7 + dp[2]);
      for (int64_t q = P.ptr[o]; q < P.ptr[o + 1]; q++) {
         const int s = P.slot[q];
         FFTSVD_REQUIRE(s >= 0 && s < 343, "translation slot");
         const std::array<int, 3> v = {s / 49 - 3 - dp[0], (s / 7) % 7 - 3 - dp[1], s % 7 - 3 - dp[2]};
         auto it = where.find(P.in_off[q]);
         if (it == where.end()) {
            it = where.emplace(P.in_off[q], (int)G.src.size()).first;
            G.src.push_back(P.in_off[q]);
            G.mask.push_back(0);
            v0.push_back(v);
         }
         const int e = it->second;
         if (v0[e] != v) return false;
         FFTSVD_REQUIRE(!((G.mask[e] >> m) & 1u), "repeated interaction");
         G.mask[e] |= 1u << m;
      }
   }
   for (size_t e = 0; e < G.src.size(); e++) {
      for (size_t m = 0; m < pos.size(); m++) {
         int v[3], far = 0;
         for (int k = 0; k < 3; k++) {
            v[k] = v0[e][k] + pos[m][k] - pos[0][k];
            if (v[k] < -3 || v[k] > 3) return false;
            far |= (v[k] < -1 || v[k] > 1);
         }
         if (!((G.mask[e] >> m) & 1u) && far) return false;
      }
      G.base.push_back(slot_of(v0[e].data()));
   }
   return true;
}
}  // namespace

// Tiling: outputs of one key in Morton order form member groups (runs of at most
// kGroupMax siblings, or single outputs where a shared list would not be exact);
// consecutive groups form a tile while its groups, halo inputs and padded entries fit
// the limits; tiles grouped by frequency count.  The groups and the order of every
// group's entries do not depend on the limits, so neither does any sum the
// translation forms: the limits change the speed only.
static void build_tiles(const TileProblem& P, const TileLimits& lim, TileSet& S) {
   std::map<int, std::vector<int>> by_key;
   for (int i = 0; i < (int)P.key.size(); i++)
      if (P.ptr[i + 1] > P.ptr[i]) by_key[P.key[i]].push_back(i);
   for (auto& kv : by_key) {
      std::vector<int>& ids = kv.second;
      std::stable_sort(ids.begin(), ids.end(), [&](int a, int b) { return P.morton[a] < P.morton[b]; });
      // runs of at most kGroupMax siblings, each made into one group (or single outputs)
      // in parallel and concatenated in run order
      std::vector<std::pair<size_t, size_t>> runs;
      for (size_t i = 0; i < ids.size();) {
         size_t last = i + 1;
         while (last < ids.size() && (int)(last - i) < kGroupMax && (P.morton[ids[last]] >> 3) == (P.morton[ids[i]] >> 3))
            last++;
         runs.push_back({i, last});
         i = last;
      }
      std::vector<std::vector<MemberGroup>> made(runs.size());
      std::exception_ptr err;
#pragma omp parallel for schedule(dynamic, 64)
      for (int64_t r = 0; r < (int64_t)runs.size(); r++) {
         try {
            const size_t first = runs[r].first, last = runs[r].second;
            MemberGroup G;
            if (make_group(P, ids, first, last, G)) {
               made[r].push_back(std::move(G));
            } else {
               for (size_t k = first; k < last; k++) {
                  FFTSVD_REQUIRE(make_group(P, ids, k, k + 1, G), "interaction outside the 7x7x7 offset range");
                  made[r].push_back(std::move(G));
               }
            }
         } catch (...) {
#pragma omp critical(fftsvd_tile_groups)
            if (!err) err = std::current_exception();
         }
      }
      if (err) std::rethrow_exception(err);
      std::vector<MemberGroup> groups;
      for (auto& v : made)
         for (auto& g : v) groups.push_back(std::move(g));
      size_t pos = 0;
      while (pos < groups.size()) {
         TileDesc tile;
         tile.ngroups = tile.nsrc = tile.nentries = tile.nmembers = 0;
         tile.pad = 0;
         tile.pg = P.pg[groups[pos].members[0]];
         tile.t_off = P.t_base[groups[pos].members[0]];
         tile.grp_off = (int64_t)S.tile_grp.size();
         tile.mem_off = (int64_t)S.tile_dst.size();
         tile.src_off = (int64_t)S.tile_src.size();
         tile.ent_off = (int64_t)S.tile_entries.size();
         std::unordered_map<int64_t, int> halo;
         halo.reserve(2 * kTileMaxSrc);
         std::vector<int> tg;
         while (pos < groups.size()) {
            const MemberGroup& G = groups[pos];
            int fresh = 0;
            for (int64_t in : G.src)
               if (!halo.count(in)) fresh++;
            const int padded = ((int)G.src.size() + 3) & ~3;
            if (!tg.empty() && ((int)tg.size() + 1 > lim.max_groups || tile.nsrc + fresh > lim.max_src ||
                                tile.nentries + padded > lim.max_entries))
               break;
            FFTSVD_REQUIRE(fresh <= kTileMaxSrc && padded <= kTileMaxEntries, "interaction list too long");
            for (int64_t in : G.src)
               if (!halo.count(in)) {
                  halo[in] = tile.nsrc++;
                  S.tile_src.push_back(in);
               }
            tile.nentries += padded;
            tg.push_back((int)pos);
            pos++;
         }
         // one warp per group: groups by decreasing cost (entries times members plus the
         // entry overhead), which the kernel deals to its warps in a snake order
         auto cost = [&](int gi) { return (groups[gi].src.size() + 3) / 4 * (2 + groups[gi].members.size()); };
         std::stable_sort(tg.begin(), tg.end(), [&](int a, int b) { return cost(a) > cost(b); });
         int ent = 0;
         for (int gi : tg) {
            const MemberGroup& G = groups[gi];
            const int nm = (int)G.members.size(), ne = ((int)G.src.size() + 3) & ~3;
            S.tile_grp.push_back(make_int4(ent, ne, tile.nmembers, nm));
            for (int j = 0; j < nm; j++) {
               S.tile_dst.push_back(P.out_off[G.members[j]]);
               S.tile_delta.push_back(G.delta[j] - kEntryBaseBias);
            }
            for (size_t e = 0; e < G.src.size(); e++)
               S.tile_entries.push_back(((uint32_t)halo.at(G.src[e]) << 17) | (G.mask[e] << 9) |
                                        (uint32_t)(G.base[e] + kEntryBaseBias));
            // padding: halo row 0 through each member's own (zeroed) offset
            for (int e = (int)G.src.size(); e < ne; e++)
               S.tile_entries.push_back((uint32_t)(kCenterSlot + kEntryBaseBias));
            ent += ne;
            tile.nmembers += nm;
            tile.ngroups++;
         }
         S.tiles.push_back(tile);
      }
   }
   std::stable_sort(S.tiles.begin(), S.tiles.end(), [](const TileDesc& a, const TileDesc& b) { return a.pg > b.pg; });
   for (int i = 0; i < (int)S.tiles.size(); i++) {
      const TileDesc& t = S.tiles[i];
      if (S.tile_groups.empty() || S.tile_groups.back().pg != t.pg) {
         TileGroup g;
         g.pg = t.pg;
         g.begin = i;
         S.tile_groups.push_back(g);
      }
      TileGroup& g = S.tile_groups.back();
      g.count++;
      g.max_src = std::max(g.max_src, t.nsrc);
      g.max_entries = std::max(g.max_entries, t.nentries);
      g.max_groups = std::max(g.max_groups, t.ngroups);
      g.max_members = std::max(g.max_members, t.nmembers);
   }
}

// Every index the translation kernel forms stays inside its buffers: table rows, the
// in_elems input spectra and the out_elems output spectra, and the shared-memory rows.
static void check_tiles(const TileSet& S, int64_t nt, int64_t in_elems, int64_t out_elems) {
   // tiles are checked independently on all host threads; the first failure is rethrown
   std::exception_ptr err;
#pragma omp parallel for schedule(dynamic, 16)
   for (int64_t ti = 0; ti < (int64_t)S.tiles.size(); ti++) {
      try {
         const TileDesc& t = S.tiles[ti];
         FFTSVD_REQUIRE(t.ngroups > 0 && t.ngroups <= kTileMaxGroups && t.nsrc > 0 && t.nsrc <= kTileMaxSrc &&
                            t.nentries > 0 && t.nentries <= kTileMaxEntries && t.nentries % 4 == 0 &&
                            t.nmembers > 0 && t.nmembers <= kTileMaxGroups * kGroupMax && t.pg > 0 && t.pg % 16 == 0,
                        "tile descriptor");
         FFTSVD_REQUIRE(t.grp_off + t.ngroups <= (int64_t)S.tile_grp.size(), "tile groups out of range");
         FFTSVD_REQUIRE(t.mem_off + t.nmembers <= (int64_t)S.tile_dst.size() &&
                            t.mem_off + t.nmembers <= (int64_t)S.tile_delta.size(),
                        "tile members out of range");
         FFTSVD_REQUIRE(t.src_off + t.nsrc <= (int64_t)S.tile_src.size(), "tile sources out of range");
         FFTSVD_REQUIRE(t.ent_off + t.nentries <= (int64_t)S.tile_entries.size(), "tile entries out of range");
         FFTSVD_REQUIRE(t.t_off >= 0 && t.t_off + 343LL * t.pg <= nt, "tile translation table out of range");
         for (int i = 0; i < t.nmembers; i++) {
            const int64_t so = S.tile_dst[t.mem_off + i];
            FFTSVD_REQUIRE(so >= 0 && so + t.pg <= out_elems, "tile destination spectrum out of range");
         }
         for (int i = 0; i < t.nsrc; i++) {
            const int64_t so = S.tile_src[t.src_off + i];
            FFTSVD_REQUIRE(so >= 0 && so + t.pg <= in_elems, "tile source spectrum out of range");
         }
         for (int g = 0; g < t.ngroups; g++) {
            const int4 gi = S.tile_grp[t.grp_off + g];
            FFTSVD_REQUIRE(gi.x >= 0 && gi.x % 4 == 0 && gi.y > 0 && gi.y % 4 == 0 && gi.x + gi.y <= t.nentries &&
                               gi.z >= 0 && gi.w >= 1 && gi.w <= kGroupMax && gi.z + gi.w <= t.nmembers,
                           "tile group out of range");
            for (int e = gi.x; e < gi.x + gi.y; e++) {
               const uint32_t w = S.tile_entries[t.ent_off + e];
               const int halo = (int)(w >> 17), base = (int)(w & 0x1ffu) - kEntryBaseBias;
               const uint32_t mask = (w >> 9) & 0xffu;
               // the kernel reads slot base + delta_j for every member j of the warp's largest
               // group (delta 0 beyond this group's members): all of them must be table rows
               FFTSVD_REQUIRE(halo < t.nsrc && (mask >> gi.w) == 0 && base >= 0 && base < 343, "tile entry out of range");
               for (int j = 0; j < gi.w; j++) {
                  const int slot = base + S.tile_delta[t.mem_off + gi.z + j] + kEntryBaseBias;
                  FFTSVD_REQUIRE(slot >= 0 && slot < 343, "tile entry slot out of range");
                  const int dx = slot / 49 - 3, dy = (slot / 7) % 7 - 3, dz = slot % 7 - 3;
                  const bool local = std::abs(dx) <= 1 && std::abs(dy) <= 1 && std::abs(dz) <= 1;
                  FFTSVD_REQUIRE(local != (((mask >> j) & 1u) != 0), "tile entry reaches a non-interacting member");
               }
            }
         }
      } catch (...) {
#pragma omp critical(fftsvd_tile_check)
         if (!err) err = std::current_exception();
      }
   }
   if (err) std::rethrow_exception(err);
}

void make_tiles(const TileProblems& P, const TileLimits& lim, TileSet& fwd, TileSet& adj) {
   FFTSVD_REQUIRE(lim.max_groups >= 1 && lim.max_groups <= kTileMaxGroups && lim.max_src >= 1 &&
                      lim.max_src <= kTileMaxSrc && lim.max_entries >= 4 && lim.max_entries <= kTileMaxEntries,
                  "tile limits out of range");
   fwd = TileSet();
   adj = TileSet();
   // the two directions one after the other, each building its member groups on all
   // host threads (an exception in either is carried out and rethrown here)
   std::exception_ptr err[2];
   for (int d = 0; d < 2; d++) {
      try {
         if (d == 0) {
            build_tiles(P.fwd, lim, fwd);
            check_tiles(fwd, P.nt, P.spectra_elems, P.translated_elems);  // spectra -> translated
         } else {
            build_tiles(P.adj, lim, adj);
            check_tiles(adj, P.nt, P.translated_elems, P.spectra_elems);  // transposed: translated -> spectra
         }
      } catch (...) {
         err[d] = std::current_exception();
      }
   }
   for (auto& e : err)
      if (e) std::rethrow_exception(e);
}

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
   // room for every tree's arrays at once (bounds from the trees' own totals), so that no
   // tree's growth reallocates and copies the arrays of the trees before it
   {
      size_t rows = 0, cols = 0, dp = 0, sp = 0, vt = 0, pv = 0, pts = 0, uti = 0, u = 0, ip = 0, tp = 0, cubes = 0;
      size_t leaves = 0;
      for (int t = 0; t < num_trees; t++) {
         const fftsvd_tree_flat& T = trees[t];
         const int nl = std::max(T.num_leaves, 0), nc = std::max(T.num_cubes, 0);
         leaves += nl;
         cubes += nc;
         if (nl > 0) {
            rows += (size_t)std::max(T.leaf_row_ptr[nl], 0);
            cols += (size_t)std::max(T.leaf_col_ptr[nl], 0) + nl;  // columns padded to even counts
            dp += 2 * ((size_t)std::max<int64_t>(T.leaf_d_ptr[nl], 0) + (size_t)std::max(T.leaf_row_ptr[nl], 0));
         }
         if (nc > 0) {
            sp += (size_t)std::max(T.cube_panel_ptr[nc], 0);
            vt += (size_t)std::max<int64_t>(T.cube_vt_ptr[nc], 0);
            pv += 2 * (size_t)std::max<int64_t>(T.cube_pv_ptr[nc], 0);
            pts += (size_t)std::max(T.cube_point_ptr[nc], 0);
            uti += (size_t)std::max<int64_t>(T.cube_uti_ptr[nc], 0);
            u += (size_t)std::max<int64_t>(T.cube_u_ptr[nc], 0);
            ip += 2 * (size_t)std::max(T.inter_ptr[nc], 0);
         }
         for (int l = 0; l < (int)std::min<int64_t>(T.depth, FFTSVD_MAX_DEPTH); l++) {
            const int n = T.grid[l], Npl = 2 * n - 1;
            if (n >= 2 && n <= 12) tp += 2 * 343 * (size_t)pad16(Npl * Npl * n);
         }
      }
      L.leaves.reserve(leaves);
      L.leaf_rows.reserve(rows);
      L.leaf_cols.reserve(cols);
      L.d_pairs.reserve(dp);
      L.src.reserve(cubes);
      L.src_panels.reserve(sp);
      L.vt.reserve(vt);
      L.pv_pairs.reserve(pv);
      L.dst.reserve(cubes);
      L.dst_points.reserve(pts);
      L.uti.reserve(uti);
      L.u_cm.reserve(u);
      L.inter_pairs.reserve(ip);
      L.t_pairs.reserve(tp);
   }
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
   struct DstExtra {
      int key;        // tree * 64 + level
      uint64_t morton;
      int64_t t_base; // translation table of slot 0 of the cube's tree and level
      int pg;
   };
   std::vector<DstExtra> dst_extra;  // parallel to L.dst until the tiles are built
   std::vector<DstExtra> src_extra;  // parallel to L.src

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

      // ---- near field: a serial pass checks every leaf and places it, then the rows,
      // columns and {D_single, D_double} pairs are filled in parallel
      std::vector<char> covered(T.num_points, 0);
      std::vector<int> near_leaf;  // leaves with rows, in order
      const size_t lr0 = L.leaf_rows.size(), lc0 = L.leaf_cols.size(), ld0 = L.leaves.size();
      const size_t dp0 = L.d_pairs.size();
      size_t nrows_all = 0, ncols_all = 0, npairs_all = 0;
      for (int l = 0; l < T.num_leaves; l++) {
         const int r0 = T.leaf_row_ptr[l], r1 = T.leaf_row_ptr[l + 1];
         const int c0 = T.leaf_col_ptr[l], c1 = T.leaf_col_ptr[l + 1];
         const int nr = r1 - r0, nc = c1 - c0, ncp = pad2(nc);
         FFTSVD_REQUIRE(nr >= 0 && nc >= 0, "bad leaf extents");
         if (nr == 0) continue;
         FFTSVD_REQUIRE(T.leaf_d_ptr[l + 1] - T.leaf_d_ptr[l] == (int64_t)nr * nc, "leaf D size mismatch");
         for (int r = r0; r < r1; r++) {
            const int pt = T.leaf_rows[r];
            FFTSVD_REQUIRE(pt >= 0 && pt < T.num_points, "leaf row out of range");
            FFTSVD_REQUIRE(!covered[pt], "point in two leaves");
            covered[pt] = 1;
         }
         for (int c = c0; c < c1; c++)
            FFTSVD_REQUIRE(T.leaf_cols[c] >= 0 && T.leaf_cols[c] < T.num_panels, "leaf column out of range");
         LeafDesc d;
         d.row_off = (int32_t)(lr0 + nrows_all);
         d.nrows = nr;
         d.col_off = (int32_t)(lc0 + ncols_all);
         d.ncols = ncp;
         d.d_off = (int64_t)((dp0 / 2) + npairs_all);
         nrows_all += nr;
         ncols_all += ncp;
         npairs_all += (size_t)nr * ncp;
         L.operator_elems += 2LL * nr * nc;
         L.leaves.push_back(d);
         near_leaf.push_back(l);
      }
      L.leaf_rows.resize(lr0 + nrows_all);
      L.leaf_cols.resize(lc0 + ncols_all);
      L.d_pairs.resize(dp0 + 2 * npairs_all);
      const int nleaf_here = (int)near_leaf.size();
#pragma omp parallel for schedule(dynamic, 16)
      for (int i = 0; i < nleaf_here; i++) {
         const int l = near_leaf[i];
         const LeafDesc& d = L.leaves[ld0 + i];
         const int r0 = T.leaf_row_ptr[l], c0 = T.leaf_col_ptr[l];
         const int nr = d.nrows, nc = T.leaf_col_ptr[l + 1] - c0, ncp = d.ncols;
         for (int r = 0; r < nr; r++) L.leaf_rows[d.row_off + r] = (int32_t)(qo + T.leaf_rows[r0 + r]);
         for (int c = 0; c < nc; c++) L.leaf_cols[d.col_off + c] = (int32_t)(po + T.leaf_cols[c0 + c]);
         for (int c = nc; c < ncp; c++) L.leaf_cols[d.col_off + c] = zero_slot;
         const int64_t db = T.leaf_d_ptr[l];
         double* out = &L.d_pairs[2 * (size_t)d.d_off];
         for (int r = 0; r < nr; r++) {
            for (int c = 0; c < nc; c++) {
               *out++ = T.d_single[db + (int64_t)r * nc + c];
               *out++ = T.d_double[db + (int64_t)r * nc + c];
            }
            for (int c = nc; c < ncp; c++) {
               *out++ = 0.0;
               *out++ = 0.0;
            }
         }
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
      // translation tables of this tree, each slot padded to a multiple of 16 complex values
      std::vector<int64_t> tlev(T.depth + 1);
      tlev[0] = (int64_t)(L.t_pairs.size() / 2);
      for (int l = 0; l < T.depth; l++) {
         const int nl = T.grid[l], Npl = 2 * nl - 1;
         FFTSVD_REQUIRE(nl >= 2 && nl <= 12, "grid size out of range");
         tlev[l + 1] = tlev[l] + 343LL * pad16(Npl * Npl * nl);
      }
      // source cubes: a serial pass checks and places them, the panel lists, VT and the
      // transposed {PV_single, PV_double} pairs are copied in parallel
      std::vector<int> src_cube;  // parallel to the SrcDesc appended for this tree
      const size_t s0 = L.src.size(), sp0 = L.src_panels.size(), vt0 = L.vt.size(), pv0 = L.pv_pairs.size();
      size_t sp_all = 0, vt_all = 0, pv_all = 0;
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
         for (int i = T.cube_panel_ptr[c]; i < T.cube_panel_ptr[c + 1]; i++)
            FFTSVD_REQUIRE(T.cube_panels[i] >= 0 && T.cube_panels[i] < T.num_panels, "cube panel out of range");
         SrcDesc sd;
         sd.n = n; sd.m = m; sd.r = r;
         sd.panel_off = (int32_t)(sp0 + sp_all);
         sd.vt_off = (int64_t)(vt0 + vt_all);
         sd.pv_off = (int64_t)((pv0 / 2) + pv_all / 2);
         sd.spec_off = L.spectra_elems;
         spec_of_cube[c] = L.spectra_elems;
         L.spectra_elems += pad16(pg);
         sp_all += m;
         vt_all += (size_t)r * m;
         pv_all += 2 * (size_t)r * n3;
         L.operator_elems += (int64_t)r * m + 2LL * r * n3;
         const int ch = std::min(m, 1024);
         const int H = n;
         int need = 2 * ch + 2 * r + n3 + 2 * Np + 2 * (n * n * H) + 2 * (n * Np * H) + 16;
         L.max_src_smem_elems = std::max(L.max_src_smem_elems, need);
         sd.level = lvl;
         sd.pad = 0;
         L.src.push_back(sd);
         src_cube.push_back(c);
         {
            const int32_t* ci = &T.cube_index[3 * c];
            uint64_t code = 0;  // Morton order of the cube coordinates
            for (int bb = 0; bb < 21; bb++)
               for (int k = 0; k < 3; k++) code |= (uint64_t)((ci[k] >> bb) & 1) << (3 * bb + k);
            src_extra.push_back({t * 64 + lvl, code, tlev[lvl], pad16(pg)});
         }
      }
      L.src_panels.resize(sp0 + sp_all);
      L.vt.resize(vt0 + vt_all);
      L.pv_pairs.resize(pv0 + pv_all);
      const int nsrc_here = (int)src_cube.size();
#pragma omp parallel for schedule(dynamic, 16)
      for (int i = 0; i < nsrc_here; i++) {
         const int c = src_cube[i];
         const SrcDesc& sd = L.src[s0 + i];
         const int m = sd.m, r = sd.r, n3 = sd.n * sd.n * sd.n;
         for (int k = 0; k < m; k++) L.src_panels[sd.panel_off + k] = (int32_t)(po + T.cube_panels[T.cube_panel_ptr[c] + k]);
         std::copy(T.vt + T.cube_vt_ptr[c], T.vt + T.cube_vt_ptr[c] + (int64_t)r * m, L.vt.begin() + sd.vt_off);
         const int64_t pb = T.cube_pv_ptr[c];
         double* out = &L.pv_pairs[2 * (size_t)sd.pv_off];
         for (int j = 0; j < r; j++)
            for (int q = 0; q < n3; q++) {
               *out++ = T.pv_single[pb + (int64_t)q * r + j];
               *out++ = T.pv_double[pb + (int64_t)q * r + j];
            }
      }
      // destination cubes: a serial pass checks them, counts their interactions with
      // source spectra and places them, then points, UTI, the transposed U and the
      // interaction pairs are filled in parallel
      std::vector<int> dst_cube;
      const size_t d0 = L.dst.size(), dp_0 = L.dst_points.size(), uti0 = L.uti.size(), u0 = L.u_cm.size();
      const size_t ip0 = L.inter_pairs.size();
      size_t dp_all = 0, uti_all = 0, u_all = 0, ip_all = 0;
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
         for (int i = T.cube_point_ptr[c]; i < T.cube_point_ptr[c + 1]; i++)
            FFTSVD_REQUIRE(T.cube_points[i] >= 0 && T.cube_points[i] < T.num_points, "cube point out of range");
         int cnt = 0;
         for (int i = T.inter_ptr[c]; i < T.inter_ptr[c + 1]; i++) {
            const int sc = T.inter_cubes[i];
            FFTSVD_REQUIRE(sc >= 0 && sc < T.num_cubes, "interacting cube out of range");
            if (spec_of_cube[sc] < 0) continue;  // source without panels or rank: contributes zero
            FFTSVD_REQUIRE(T.cube_level[sc] == lvl, "interaction across levels");
            const int dx = T.cube_index[3 * c] - T.cube_index[3 * sc];
            const int dy = T.cube_index[3 * c + 1] - T.cube_index[3 * sc + 1];
            const int dz = T.cube_index[3 * c + 2] - T.cube_index[3 * sc + 2];
            FFTSVD_REQUIRE(std::abs(dx) <= 3 && std::abs(dy) <= 3 && std::abs(dz) <= 3, "interaction offset too large");
            FFTSVD_REQUIRE(std::abs(dx) > 1 || std::abs(dy) > 1 || std::abs(dz) > 1, "local cube in interaction list");
            FFTSVD_REQUIRE(T.t_level_ptr[lvl + 1] - T.t_level_ptr[lvl] == 343LL * pg, "translation table size mismatch");
            cnt++;
         }
         L.operator_elems += (int64_t)r * n3 + (int64_t)p * r;
         int need = 2 * pg + 2 * (n * Np * H) + 2 * (n * n * H) + n3 + r + 2 * Np + 16;
         L.max_dst_smem_elems = std::max(L.max_dst_smem_elems, need);
         if (cnt == 0) continue;  // no interaction with any source spectrum: no far field to add
         DstDesc dd;
         dd.n = n; dd.p = p; dd.r = r;
         dd.point_off = (int32_t)(dp_0 + dp_all);
         dd.uti_off = (int64_t)(uti0 + uti_all);
         dd.u_off = (int64_t)(u0 + u_all);
         dd.inter_off = (int32_t)((ip0 + ip_all) / 2);
         dd.inter_cnt = cnt;
         dd.stage = lvl;
         dd.pad = 0;
         dd.s_off = L.translated_elems;
         L.translated_elems += pad16(pg);
         dp_all += p;
         uti_all += (size_t)r * n3;
         u_all += (size_t)r * p;
         ip_all += 2 * (size_t)cnt;
         L.dst.push_back(dd);
         dst_cube.push_back(c);
         const int32_t* ci = &T.cube_index[3 * c];
         uint64_t code = 0;  // Morton order of the cube coordinates
         for (int bb = 0; bb < 21; bb++)
            for (int k = 0; k < 3; k++) code |= (uint64_t)((ci[k] >> bb) & 1) << (3 * bb + k);
         dst_extra.push_back({t * 64 + lvl, code, tlev[lvl], pad16(pg)});
      }
      L.dst_points.resize(dp_0 + dp_all);
      L.uti.resize(uti0 + uti_all);
      L.u_cm.resize(u0 + u_all);
      L.inter_pairs.resize(ip0 + ip_all);
      const int ndst_here = (int)dst_cube.size();
#pragma omp parallel for schedule(dynamic, 16)
      for (int i = 0; i < ndst_here; i++) {
         const int c = dst_cube[i];
         const DstDesc& dd = L.dst[d0 + i];
         const int p = dd.p, r = dd.r, n = dd.n, n3 = n * n * n, pg = (2 * n - 1) * (2 * n - 1) * n;
         const int lvl = T.cube_level[c];
         for (int k = 0; k < p; k++)
            L.dst_points[dd.point_off + k] = (int32_t)(qo + T.cube_points[T.cube_point_ptr[c] + k]);
         std::copy(T.uti + T.cube_uti_ptr[c], T.uti + T.cube_uti_ptr[c] + (int64_t)r * n3, L.uti.begin() + dd.uti_off);
         const int64_t uub = T.cube_u_ptr[c];
         double* uo = &L.u_cm[dd.u_off];
         for (int j = 0; j < r; j++)
            for (int q = 0; q < p; q++) *uo++ = T.u[uub + (int64_t)q * r + j];
         int64_t* io = &L.inter_pairs[2 * (size_t)dd.inter_off];
         for (int ii = T.inter_ptr[c]; ii < T.inter_ptr[c + 1]; ii++) {
            const int sc = T.inter_cubes[ii];
            if (spec_of_cube[sc] < 0) continue;
            const int dx = T.cube_index[3 * c] - T.cube_index[3 * sc];
            const int dy = T.cube_index[3 * c + 1] - T.cube_index[3 * sc + 1];
            const int dz = T.cube_index[3 * c + 2] - T.cube_index[3 * sc + 2];
            const int slot = ((dx + 3) * 7 + (dy + 3)) * 7 + (dz + 3);
            *io++ = spec_of_cube[sc];
            *io++ = tlev[lvl] + (int64_t)slot * pad16(pg);
         }
      }
      // translation operators of this tree (unique tables: 316 non-local offsets per level),
      // every slot padded with zeros to a multiple of 16 complex values
      FFTSVD_REQUIRE((int64_t)(L.t_pairs.size() / 2) == tlev[0], "translation table offset");
      for (int lvl = 0; lvl < T.depth; lvl++) {
         const int n = T.grid[lvl], Np = 2 * n - 1, pg = Np * Np * n, pgp = pad16(pg);
         FFTSVD_REQUIRE(T.t_level_ptr[lvl + 1] - T.t_level_ptr[lvl] == 343LL * pg, "translation table size mismatch");
         for (int slot = 0; slot < 343; slot++) {
            // the 27 local offsets (|d| <= 1 on every axis) never interact: zero rows, which the
            // translation reads for sibling members that do not interact with a shared source
            const int dx = slot / 49 - 3, dy = (slot / 7) % 7 - 3, dz = slot % 7 - 3;
            if (std::abs(dx) <= 1 && std::abs(dy) <= 1 && std::abs(dz) <= 1) {
               L.t_pairs.insert(L.t_pairs.end(), 2 * (size_t)pgp, 0.0);
               continue;
            }
            const double* src = T.t_ops + 2 * (T.t_level_ptr[lvl] + (int64_t)slot * pg);
            L.t_pairs.insert(L.t_pairs.end(), src, src + 2 * pg);
            L.t_pairs.insert(L.t_pairs.end(), 2 * (size_t)(pgp - pg), 0.0);
         }
         L.t_elems += 2LL * 316 * pg;
      }
      FFTSVD_REQUIRE((int64_t)(L.t_pairs.size() / 2) == tlev[T.depth], "translation table size");
   }
   for (int o = 0; o < num_unknowns; o++)
      if (!row_written[o]) L.full_cover = false;

   // ---- translation tiles: destinations of one tree and level in Morton order, greedily
   // grouped while the tile's destinations, halo sources and interactions fit the limits.
   // The transposed operator translates the other way: every source cube gathers from the
   // destinations whose lists hold it, through the table slot of the opposite offset
   // (the grid-to-grid kernel of a symmetric Green's function satisfies G_DS^T = G_SD).
   L.problems = std::make_shared<TileProblems>();
   {
      TileProblem& fwd = L.problems->fwd;
      TileProblem& adj = L.problems->adj;
      // source index of each spectrum (spectra start at distinct multiples of 16)
      std::vector<int32_t> src_of_spec((size_t)(L.spectra_elems / 16) + 1, -1);
      for (int i = 0; i < (int)L.src.size(); i++) {
         FFTSVD_REQUIRE(L.src[i].spec_off % 16 == 0, "spectrum offset");
         src_of_spec[(size_t)(L.src[i].spec_off / 16)] = i;
      }
      auto source_of = [&](int64_t so) {
         const int i = so >= 0 && so < L.spectra_elems && so % 16 == 0 ? src_of_spec[(size_t)(so / 16)] : -1;
         FFTSVD_REQUIRE(i >= 0, "interaction with an unknown source spectrum");
         return i;
      };
      const int64_t npairs = (int64_t)L.inter_pairs.size() / 2;
      fwd.in_off.reserve(npairs);
      fwd.slot.reserve(npairs);
      adj.in_off.reserve(npairs);
      adj.slot.reserve(npairs);
      // the transposed lists in compressed form: per source, its destinations in the order
      // of the destinations and their interactions
      std::vector<int64_t> adj_ptr(L.src.size() + 1, 0);
      for (int i = 0; i < (int)L.dst.size(); i++) {
         const DstDesc& d = L.dst[i];
         for (int q = 0; q < d.inter_cnt; q++) adj_ptr[source_of(L.inter_pairs[2 * (d.inter_off + q)]) + 1]++;
      }
      for (size_t i = 0; i < L.src.size(); i++) adj_ptr[i + 1] += adj_ptr[i];
      std::vector<int64_t> adj_out((size_t)adj_ptr.back());
      std::vector<int> adj_slot((size_t)adj_ptr.back());
      std::vector<int64_t> fill(adj_ptr.begin(), adj_ptr.end() - 1);
      for (int i = 0; i < (int)L.dst.size(); i++) {
         const DstDesc& d = L.dst[i];
         const DstExtra& e = dst_extra[i];
         fwd.add_output(e.key, e.morton, e.t_base, e.pg, d.s_off);
         for (int q = 0; q < d.inter_cnt; q++) {
            const int64_t so = L.inter_pairs[2 * (d.inter_off + q)];
            const int64_t to = L.inter_pairs[2 * (d.inter_off + q) + 1];
            const int64_t slot = (to - e.t_base) / e.pg;
            FFTSVD_REQUIRE(slot >= 0 && slot < 343 && (to - e.t_base) % e.pg == 0, "translation slot");
            fwd.add_pair(so, (int)slot);
            const int64_t at = fill[source_of(so)]++;
            adj_out[at] = d.s_off;
            adj_slot[at] = 342 - (int)slot;
         }
      }
      for (int i = 0; i < (int)L.src.size(); i++) {
         const DstExtra& e = src_extra[i];
         adj.add_output(e.key, e.morton, e.t_base, e.pg, L.src[i].spec_off);
         for (int64_t k = adj_ptr[i]; k < adj_ptr[i + 1]; k++) adj.add_pair(adj_out[k], adj_slot[k]);
      }
   }

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
   for (const DstDesc& d : L.dst) {
      const int64_t pg = (int64_t)(2 * d.n - 1) * (2 * d.n - 1) * d.n;
      FFTSVD_REQUIRE(d.s_off >= 0 && d.s_off + pg <= L.translated_elems, "translated spectrum out of range");
   }
   L.problems->nt = nt;
   L.problems->spectra_elems = L.spectra_elems;
   L.problems->translated_elems = L.translated_elems;
   make_tiles(*L.problems, TileLimits(), L.fwd, L.adj);
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
      const double sbuf = 2.0 * (double)L.translated_elems;
      kb.elems[2] = spec + (double)L.t_elems + sbuf;                      // spectra, T, translated writes
      kb.fixed[2] = 4.0 * (double)(L.fwd.tile_entries.size() + L.fwd.tile_delta.size()) + 16.0 * (double)L.fwd.tile_grp.size() +
                 8.0 * (double)(L.fwd.tile_src.size() + L.fwd.tile_dst.size());
      kb.elems[3] = sbuf + uti + u + nq;                                  // translated, UTI, U, staging writes
      kb.fixed[3] = 4.0 * (double)L.dst_points.size();
      kb.elems[4] = dpairs + 2.0 * lcols + (double)L.stage_levels * nq;   // D, gathered x, staged far field
      kb.fixed[4] = 4.0 * (lcols + lrows) + nq * (8.0 + 4.0 + 4.0 + 8.0); // indices, y, maps, jump
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
      if (L.src_groups.empty() || L.src_groups.back().n != L.src[i].n) L.src_groups.push_back({L.src[i].n, i, 0, 0, 0});
      LaunchGroup& g = L.src_groups.back();
      g.count++;
      g.smem_elems = std::max(g.smem_elems, src_need(L.src[i]));
      g.max_rank = std::max(g.max_rank, L.src[i].r);
      g.units += L.src[i].m;
      const int n = L.src[i].n, Np = 2 * n - 1;
      g.batch_shared = std::max(g.batch_shared, 2 * std::min(L.src[i].m, 1024) + 2 * Np);
      g.batch_per_rhs = std::max(g.batch_per_rhs, 2 * L.src[i].r + n * n * n + 2 * n * n * n + 2 * n * Np * n);
   }
   for (int i = 0; i < (int)L.dst.size(); i++) {
      if (L.dst_groups.empty() || L.dst_groups.back().n != L.dst[i].n) L.dst_groups.push_back({L.dst[i].n, i, 0, 0, 0});
      LaunchGroup& g = L.dst_groups.back();
      g.count++;
      g.smem_elems = std::max(g.smem_elems, dst_need(L.dst[i]));
      g.max_rank = std::max(g.max_rank, L.dst[i].r);
      g.units += L.dst[i].p;
      const int n = L.dst[i].n, Np = 2 * n - 1;
      g.batch_shared = std::max(g.batch_shared, 2 * Np);
      g.batch_per_rhs = std::max(g.batch_per_rhs, 2 * Np * Np * n + 2 * n * Np * n + 2 * n * n * n + n * n * n +
                                                      L.dst[i].r);
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
                            const double* __restrict__ x, typename Vec2<T>::type* __restrict__ xsd, BatchStrides bs) {
   using T2 = typename Vec2<T>::type;
   x += blockIdx.y * bs.n;
   xsd += blockIdx.y * bs.panels;
   for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
      T2 v;
      v.x = (T)(dphi_scale[k] * x[dphi_idx[k]]);
      v.y = (T)(phi_scale[k] * x[phi_idx[k]]);
      xsd[k] = v;
   }
}

constexpr int kFarThreads = 512;  // upper bound; each launch group picks its own block size

// block size of a block-per-cube launch: enough threads for the spectrum of one cube
static int far_threads(int n) {
   const int pg = (2 * n - 1) * (2 * n - 1) * n;
   return pg <= 256 ? 128 : pg <= 512 ? 256 : 512;
}
// Block size of a group's block-per-cube launch: a power of two from 64 to 512 covering a
// quarter of the spectrum and half of the cube's mean panel (or point) count.  Measured on the
// B200: on the 81 920-panel blob the 6^3 grid (156 panels per cube) ran the mixed solve 2 %
// faster on 256 threads than on 512; on the 327 680-panel blob, whose coarse cubes hold
// 284 to 5 851 panels, halving the blocks made the solve 1.6 % slower.
static int far_threads(const LaunchGroup& g) {
   const int pg = (2 * g.n - 1) * (2 * g.n - 1) * g.n;
   const int64_t mean = g.count > 0 ? g.units / g.count : 0;
   const int64_t want = std::max<int64_t>(pg / 4, mean / 2);
   int t = 64;
   while (t < want && t < kFarThreads) t *= 2;
   return t;
}
constexpr int kChunk = 1024;

// right-hand sides per block of the batched far-field kernels
template <typename T>
constexpr int far_rb() { return sizeof(T) == 4 ? 8 : 4; }
// dynamic shared memory of a block of g serving rb right-hand sides (16-byte carve padding included)
static int far_batch_smem(const LaunchGroup& g, int rb, size_t elem) {
   return (int)((g.batch_shared + (size_t)rb * g.batch_per_rhs) * elem + 256);
}

// One block per source cube and RB right-hand sides: a = VT x (both layers), g = PV_s a_s +
// PV_d a_d on the n^3 grid, F = r2c DFT of g placed at offset n/2 in the (2n-1)^3 box.
// Every right-hand side goes through the arithmetic of RB = 1 (same loops, chunks and
// reduction order); RB > 1 reads each PV row and twiddle once for RB right-hand sides and
// runs the transform stages over all of them between barriers.
template <typename T, int RB>
__global__ void __launch_bounds__(kFarThreads) far_forward_kernel(
    const SrcDesc* __restrict__ cubes, const int32_t* __restrict__ src_panels,
    const typename Vec2<T>::type* __restrict__ xsd, const T* __restrict__ vt,
    const typename Vec2<T>::type* __restrict__ pv, typename Vec2<T>::type* __restrict__ spectra, BatchStrides bs) {
   using T2 = typename Vec2<T>::type;
   const int ngrp = bs.nrhs / RB;
   const int rhs0 = (blockIdx.x % ngrp) * RB, unit = blockIdx.x / ngrp;  // right-hand sides fastest
   extern __shared__ __align__(16) char smem_raw[];
   const SrcDesc c = cubes[unit];
   const int n = c.n, Np = 2 * n - 1, H = n, off = n / 2, n3 = n * n * n;
   const int NA = n * n * H, NB = n * Np * H, PG = Np * Np * H;
   const int m = c.m, r = c.r;
   const int ch = min(m, kChunk);
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;

   char* p = smem_raw;
   T* xs = carve<T>(p, ch);
   T* xd = carve<T>(p, ch);
   T* as = carve<T>(p, RB * r);
   T* ad = carve<T>(p, RB * r);
   T* g = carve<T>(p, RB * n3);
   T2* tw = carve<T2>(p, Np);
   T2* A = carve<T2>(p, RB * NA);
   T2* B = carve<T2>(p, RB * NB);

   for (int j = tid; j < RB * r; j += blockDim.x) { as[j] = T(0); ad[j] = T(0); }
   for (int k = tid; k < Np; k += blockDim.x) {  // exp(-2 pi i k / Np)
      T cs, sn;
      Cx<T>::cis(k, Np, &cs, &sn);
      tw[k] = Cx<T>::make(cs, -sn);
   }
   // VT x, streamed over panel chunks; each row is owned by one warp
   for (int rb = 0; rb < RB; rb++) {
      const T2* x = xsd + (int64_t)(rhs0 + rb) * bs.panels;
      T* asr = as + rb * r;
      T* adr = ad + rb * r;
      for (int base = 0; base < m; base += ch) {
         const int cnt = min(ch, m - base);
         __syncthreads();
         for (int i = tid; i < cnt; i += blockDim.x) {
            T2 v = x[src_panels[c.panel_off + base + i]];
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
            if (lane == 0) { asr[j] += s; adr[j] += d; }
         }
      }
   }
   __syncthreads();
   // grid charges
   for (int q = tid; q < n3; q += blockDim.x) {
      const T2* col = pv + c.pv_off + q;
      T acc[RB];
#pragma unroll
      for (int rb = 0; rb < RB; rb++) acc[rb] = T(0);
      for (int j = 0; j < r; j++) {
         T2 w = col[(int64_t)j * n3];
#pragma unroll
         for (int rb = 0; rb < RB; rb++) acc[rb] += w.x * as[rb * r + j] + w.y * ad[rb * r + j];
      }
#pragma unroll
      for (int rb = 0; rb < RB; rb++) g[rb * n3 + q] = acc[rb];
   }
   __syncthreads();
   // DFT along k (input index k + off), half spectrum kf < H
   for (int idx = tid; idx < RB * NA; idx += blockDim.x) {
      const int rb = idx / NA, e = idx - rb * NA;
      const int kf = e % H, ij = e / H;
      const T* line = g + rb * n3 + ij * n;
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
   for (int idx = tid; idx < RB * NB; idx += blockDim.x) {
      const int rb = idx / NB, e = idx - rb * NB;
      const int kf = e % H, jf = (e / H) % Np, i = e / (H * Np);
      const T2* Ar = A + rb * NA;
      T2 acc = Cx<T>::make(T(0), T(0));
      for (int j = 0; j < n; j++) acc = Cx<T>::fma(Ar[(i * n + j) * H + kf], tw[((j + off) * jf) % Np], acc);
      B[idx] = acc;
   }
   __syncthreads();
   // along i, straight to global
   for (int idx = tid; idx < RB * PG; idx += blockDim.x) {
      const int rb = idx / PG, e = idx - rb * PG;
      const int kf = e % H, jf = (e / H) % Np, fi = e / (H * Np);
      const T2* Br = B + rb * NB;
      T2 acc = Cx<T>::make(T(0), T(0));
      for (int i = 0; i < n; i++) acc = Cx<T>::fma(Br[(i * Np + jf) * H + kf], tw[((i + off) * fi) % Np], acc);
      spectra[(int64_t)(rhs0 + rb) * bs.spectra + c.spec_off + e] = acc;
   }
}

constexpr int kTileRowBytes = 128;                         // shared-memory row per slot/source and chunk
constexpr int kTileUnits = kTileRowBytes / 16;             // 16-byte units per row: threads per member group
constexpr int kTranslateThreads = kTileMaxGroups * kTileUnits;

__device__ inline void cp_async16(void* smem, const void* gmem) {
   const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
   asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ inline void cp_async_wait() {
   asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// 16 bytes of spectrum: two FP32 complex values or one FP64 complex value
template <typename T> struct Pack16;
template <> struct Pack16<float> {
   using V = float4;
   __device__ static inline V zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
   __device__ static inline void add(V& a, const V& b) {
      a.x += b.x;
      a.y += b.y;
      a.z += b.z;
      a.w += b.w;
   }
   __device__ static inline V shfl_xor(const V& a, int m) {
      return make_float4(__shfl_xor_sync(0xffffffffu, a.x, m), __shfl_xor_sync(0xffffffffu, a.y, m),
                         __shfl_xor_sync(0xffffffffu, a.z, m), __shfl_xor_sync(0xffffffffu, a.w, m));
   }
   __device__ static inline void fma(V& acc, const V& a, const V& b) {  // acc += a * b, two complex
      acc.x = fmaf(a.x, b.x, fmaf(-a.y, b.y, acc.x));
      acc.y = fmaf(a.x, b.y, fmaf(a.y, b.x, acc.y));
      acc.z = fmaf(a.z, b.z, fmaf(-a.w, b.w, acc.z));
      acc.w = fmaf(a.z, b.w, fmaf(a.w, b.z, acc.w));
   }
};
template <> struct Pack16<double> {
   using V = double2;
   __device__ static inline V zero() { return make_double2(0.0, 0.0); }
   __device__ static inline void add(V& a, const V& b) {
      a.x += b.x;
      a.y += b.y;
   }
   __device__ static inline V shfl_xor(const V& a, int m) {
      return make_double2(__shfl_xor_sync(0xffffffffu, a.x, m), __shfl_xor_sync(0xffffffffu, a.y, m));
   }
   __device__ static inline void fma(V& acc, const V& a, const V& b) {
      acc.x = ::fma(a.x, b.x, ::fma(-a.y, b.y, acc.x));
      acc.y = ::fma(a.x, b.y, ::fma(a.y, b.x, acc.y));
   }
};

// One member group's part of one frequency chunk, one warp per group: lane = (entry
// phase p = lane / 8, 16-byte unit u = lane % 8).  Phase p takes the entry pairs
// p, p + 4, p + 8, ... of the group's list; for each entry it reads the source unit
// from shared memory once and applies it to all NM members of the group.  Members are
// siblings, so every source of the group lies within three cubes of each member and
// base + delta_j is always a table row; for a member that does not interact with the
// source it is one of the 27 local-offset rows, which hold zeros.  Padding entries
// point at the zero row of each member's own offset.  The loop therefore has no
// branches.  Shared entry word: bits 20-31 halo row in 16-byte units, bits 0-11
// (base slot + bias) in 16-byte units; dj[j] is member j's (delta - bias) in bytes.
// The four phase partials are summed with shuffles in a fixed order.
template <typename T, int NM>
__device__ __forceinline__ void translate_group(uint32_t tsu, uint32_t fsu, uint32_t es, int npairs, int phase,
                                                const int (&dj)[kGroupMax], typename Pack16<T>::V (&acc)[kGroupMax]) {
   using V = typename Pack16<T>::V;
   extern __shared__ __align__(16) char smem_raw[];
   for (int q = phase; q < npairs; q += 4) {
      const uint2 w2 = *reinterpret_cast<const uint2*>(smem_raw + es + (uint32_t)q * 8u);
      const uint32_t ws[2] = {w2.x, w2.y};
#pragma unroll
      for (int e = 0; e < 2; e++) {
         const uint32_t w = ws[e];
         const V f = *reinterpret_cast<const V*>(smem_raw + fsu + ((w >> 16) & 0xfff0u));
         const uint32_t tb = tsu + ((w << 4) & 0xfff0u);
#pragma unroll
         for (int j = 0; j < NM; j++)
            Pack16<T>::fma(acc[j], *reinterpret_cast<const V*>(smem_raw + (tb + (uint32_t)dj[j])), f);
      }
   }
#pragma unroll
   for (int j = 0; j < NM; j++) {
      Pack16<T>::add(acc[j], Pack16<T>::shfl_xor(acc[j], 8));
      Pack16<T>::add(acc[j], Pack16<T>::shfl_xor(acc[j], 16));
   }
}

// One block per (tile, range of frequency chunks): S[d][f] = sum over the
// interactions of destination d of T[slot][f] * F[source][f] (Cube_multiply_T,
// Cube.c:2062-2111).  The chunk of all 343 translation slots of the tile's tree and
// level and the chunk of every halo source spectrum are copied to shared memory with
// cp.async, so each table entry and spectrum crosses L2 once per tile instead of
// once per interaction; two blocks per SM overlap one's copies with the other's
// arithmetic.  Rows are padded to a multiple of 16 complex values, so every copy is
// a full aligned 16 bytes.  Each warp takes member groups of the tile in turn: the
// groups are ordered by cost and dealt to the warps in a snake order, so the warps of
// a block finish together.  A warp keeps one accumulator per member, so each source
// unit read from shared memory serves every sibling of the group.
//
// Single right-hand side: a row is kTileRowBytes of consecutive frequencies of
// one spectrum (8 units); the slot rows are as wide.
// Batch (BATCH, blockIdx.z = group of 8 right-hand sides in planar buffers): a
// row is one 16-byte unit (2 FP32 or 1 FP64 frequency) of each of the 8
// right-hand sides, and a slot row is the single unit of those frequencies, read
// once and applied to all 8.
template <typename T, bool BATCH>
__global__ void __launch_bounds__(kTranslateThreads, 2) translate_kernel(
    const TileDesc* __restrict__ tiles, const int64_t* __restrict__ tile_src, const int64_t* __restrict__ tile_dst,
    const int32_t* __restrict__ tile_delta, const int4* __restrict__ tile_grp,
    const uint32_t* __restrict__ tile_entries, const typename Vec2<T>::type* __restrict__ tops,
    const typename Vec2<T>::type* __restrict__ spectra, typename Vec2<T>::type* __restrict__ S,
    int chunks_per_block, BatchStrides bs) {
   using T2 = typename Vec2<T>::type;
   using V = typename Pack16<T>::V;
   constexpr int U = kTileUnits;                                  // 16-byte units per row
   constexpr int PER16 = 16 / (int)sizeof(T2);                    // complex values per unit
   constexpr int CH = BATCH ? PER16 : kTileRowBytes / (int)sizeof(T2);  // frequencies per chunk
   constexpr int TU = BATCH ? 1 : U;                              // units per slot row
   extern __shared__ __align__(16) char smem_raw[];
   if (BATCH) {
      spectra += (int64_t)blockIdx.z * U * bs.spectra;  // first right-hand side of this group
      S += (int64_t)blockIdx.z * U * bs.translated;
   }
   const TileDesc t = tiles[blockIdx.x];
   const int nchunks = t.pg / CH;
   const int kbeg = blockIdx.y * chunks_per_block;
   if (kbeg >= nchunks) return;
   const int kend = min(nchunks, kbeg + chunks_per_block);
   char* p = smem_raw;
   // batch: two buffers (the table rows are one unit wide, so both fit beside a second block
   // per SM): the next chunk is copied while this one is multiplied
   constexpr bool DB = BATCH;
   V* const Tb0 = carve<V>(p, 343 * TU);
   V* const Fb0 = carve<V>(p, t.nsrc * U);
   V* const Tb1 = DB ? carve<V>(p, 343 * TU) : Tb0;
   V* const Fb1 = DB ? carve<V>(p, t.nsrc * U) : Fb0;
   uint32_t* ent = carve<uint32_t>(p, t.nentries);
   int4* grp = carve<int4>(p, t.ngroups);
   int64_t* dstoff = carve<int64_t>(p, t.nmembers);
   int* delta = carve<int>(p, t.nmembers);
   int64_t* srcoff = carve<int64_t>(p, t.nsrc);
   // entries re-encoded with row offsets in 16-byte units (halo <= 319 rows of U units,
   // base + bias <= 511 rows of TU units: both below 4096)
   for (int i = threadIdx.x; i < t.nentries; i += blockDim.x) {
      const uint32_t w = tile_entries[t.ent_off + i];
      ent[i] = (((w >> 17) * (uint32_t)U) << 20) | ((w & 0x1ffu) * (uint32_t)TU);
   }
   for (int i = threadIdx.x; i < t.ngroups; i += blockDim.x) grp[i] = tile_grp[t.grp_off + i];
   for (int i = threadIdx.x; i < t.nmembers; i += blockDim.x) {
      dstoff[i] = tile_dst[t.mem_off + i];
      delta[i] = tile_delta[t.mem_off + i] * TU * 16;
   }
   for (int i = threadIdx.x; i < t.nsrc; i += blockDim.x) srcoff[i] = tile_src[t.src_off + i];
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
   const int u = lane & (U - 1), phase = lane / U;
   // all shared accesses below are smem_raw plus a byte offset, so they compile to
   // shared-window loads
   const uint32_t es0 = (uint32_t)((const char*)ent - smem_raw);
   auto stage = [&](int k, int b) {
      const int f0 = k * CH;
      V* const Tb = b ? Tb1 : Tb0;
      V* const Fb = b ? Fb1 : Fb0;
      for (int i = threadIdx.x; i < 343 * TU; i += blockDim.x) {
         const int s = i / TU, uu = i % TU;
         cp_async16(&Tb[i], &tops[t.t_off + (int64_t)s * t.pg + f0 + uu * PER16]);
      }
      for (int i = threadIdx.x; i < t.nsrc * U; i += blockDim.x) {
         const int s = i / U, uu = i % U;
         if (BATCH)
            cp_async16(&Fb[i], &spectra[uu * bs.spectra + srcoff[s] + f0]);
         else
            cp_async16(&Fb[i], &spectra[srcoff[s] + f0 + uu * PER16]);
      }
      cp_async_commit();
   };
   __syncthreads();  // metadata written
   if (DB) stage(kbeg, 0);
   for (int k = kbeg; k < kend; k++) {
      const int f0 = k * CH;
      const int b = DB ? (k - kbeg) & 1 : 0;
      if (DB) {
         if (k + 1 < kend) {
            stage(k + 1, b ^ 1);
            cp_async_wait<1>();
         } else {
            cp_async_wait<0>();
         }
      } else {
         if (k > kbeg) __syncthreads();  // the previous chunk's rows consumed
         stage(k, 0);
         cp_async_wait<0>();
      }
      __syncthreads();
      // all shared accesses below are smem_raw plus a byte offset, so they compile to
      // shared-window loads
      const uint32_t tsu = (uint32_t)((const char*)(b ? Tb1 : Tb0) - smem_raw) + (BATCH ? 0u : (uint32_t)u * 16u);
      const uint32_t fsu = (uint32_t)((const char*)(b ? Fb1 : Fb0) - smem_raw) + (uint32_t)u * 16u;
      // groups in cost order, dealt to the warps in a snake order
      for (int r = 0;; r++) {
         const int gidx = r * nwarps + ((r & 1) ? nwarps - 1 - warp : warp);
         if (gidx >= t.ngroups) break;
         const int4 gi = grp[gidx];
         int dj[kGroupMax];
#pragma unroll
         for (int j = 0; j < kGroupMax; j++) dj[j] = j < gi.w ? delta[gi.z + j] : 0;
         V acc[kGroupMax];
#pragma unroll
         for (int j = 0; j < kGroupMax; j++) acc[j] = Pack16<T>::zero();
         const uint32_t es = es0 + (uint32_t)gi.x * 4u;
         const int np = gi.y >> 1;
         switch (gi.w) {
            case 1: translate_group<T, 1>(tsu, fsu, es, np, phase, dj, acc); break;
            case 2: translate_group<T, 2>(tsu, fsu, es, np, phase, dj, acc); break;
            case 3: translate_group<T, 3>(tsu, fsu, es, np, phase, dj, acc); break;
            case 4: translate_group<T, 4>(tsu, fsu, es, np, phase, dj, acc); break;
            case 5: translate_group<T, 5>(tsu, fsu, es, np, phase, dj, acc); break;
            case 6: translate_group<T, 6>(tsu, fsu, es, np, phase, dj, acc); break;
            case 7: translate_group<T, 7>(tsu, fsu, es, np, phase, dj, acc); break;
            default: translate_group<T, 8>(tsu, fsu, es, np, phase, dj, acc); break;
         }
         // phase p writes the members j = p, p + 4 (every lane holds the sums)
#pragma unroll
         for (int j = 0; j < kGroupMax; j++)
            if (j < gi.w && (j & 3) == phase) {
               const int64_t o = dstoff[gi.z + j];
               if (BATCH)
                  *reinterpret_cast<V*>(&S[u * bs.translated + o + f0]) = acc[j];
               else
                  *reinterpret_cast<V*>(&S[o + f0 + u * PER16]) = acc[j];
            }
      }
      if (DB) __syncthreads();  // buffer b is refilled by the copies issued in the next iteration
   }
}

// One block per destination cube and RB right-hand sides: the translated spectrum S, c2r
// DFT cropped at offset n/2 and scaled by 1/(2n-1)^3, u = UTI g, values U u written to
// this level's staging row of each point (Cube_multiply_U_UTI_IFFT, Cube.c:2156-2225).
// Every right-hand side goes through the arithmetic of RB = 1 (same loops and reduction
// order); RB > 1 reads each UTI and U row once for RB right-hand sides.
template <typename T, int RB>
__global__ void __launch_bounds__(kFarThreads) far_backward_kernel(
    const DstDesc* __restrict__ cubes, const int32_t* __restrict__ dst_points,
    const typename Vec2<T>::type* __restrict__ translated, const T* __restrict__ uti, const T* __restrict__ ucm,
    T* __restrict__ staging, int64_t total_points, BatchStrides bs) {
   using T2 = typename Vec2<T>::type;
   const int ngrp = bs.nrhs / RB;
   const int rhs0 = (blockIdx.x % ngrp) * RB, unit = blockIdx.x / ngrp;  // right-hand sides fastest
   extern __shared__ __align__(16) char smem_raw[];
   const DstDesc c = cubes[unit];
   const int n = c.n, Np = 2 * n - 1, H = n, off = n / 2, n3 = n * n * n, pg = Np * Np * H;
   const int NA = n * n * H, NB = n * Np * H, r = c.r;
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;

   char* p = smem_raw;
   T2* S = carve<T2>(p, RB * pg);
   T2* P1 = carve<T2>(p, RB * NB);
   T2* P2 = carve<T2>(p, RB * NA);
   T* g = carve<T>(p, RB * n3);
   T* u = carve<T>(p, RB * r);
   T2* tw = carve<T2>(p, Np);

   for (int k = tid; k < Np; k += blockDim.x) {  // exp(+2 pi i k / Np)
      T cs, sn;
      Cx<T>::cis(k, Np, &cs, &sn);
      tw[k] = Cx<T>::make(cs, sn);
   }
   for (int f = tid; f < RB * pg; f += blockDim.x) {
      const int rb = f / pg;
      S[f] = translated[(int64_t)(rhs0 + rb) * bs.translated + c.s_off + (f - rb * pg)];
   }
   __syncthreads();
   // inverse along i (output i < n only)
   for (int idx = tid; idx < RB * NB; idx += blockDim.x) {
      const int rb = idx / NB, e = idx - rb * NB;
      const int kf = e % H, jf = (e / H) % Np, i = e / (H * Np);
      const T2* Sr = S + rb * pg;
      T2 acc = Cx<T>::make(T(0), T(0));
      for (int fi = 0; fi < Np; fi++) acc = Cx<T>::fma(Sr[(fi * Np + jf) * H + kf], tw[((i + off) * fi) % Np], acc);
      P1[idx] = acc;
   }
   __syncthreads();
   // inverse along j (output j < n only)
   for (int idx = tid; idx < RB * NA; idx += blockDim.x) {
      const int rb = idx / NA, e = idx - rb * NA;
      const int kf = e % H, j = (e / H) % n, i = e / (H * n);
      const T2* P1r = P1 + rb * NB;
      T2 acc = Cx<T>::make(T(0), T(0));
      for (int jf = 0; jf < Np; jf++) acc = Cx<T>::fma(P1r[(i * Np + jf) * H + kf], tw[((j + off) * jf) % Np], acc);
      P2[idx] = acc;
   }
   __syncthreads();
   // Hermitian half along k -> real, cropped, scaled
   const T scale = T(1) / (T)(Np * Np * Np);
   for (int q = tid; q < RB * n3; q += blockDim.x) {
      const int rb = q / n3, e = q - rb * n3;
      const int k = e % n, ij = e / n;
      const T2* line = P2 + rb * NA + ij * H;
      T acc = line[0].x;
      for (int kf = 1; kf < H; kf++) {
         T2 w = tw[((k + off) * kf) % Np];
         acc += T(2) * (line[kf].x * w.x - line[kf].y * w.y);
      }
      g[q] = acc * scale;
   }
   __syncthreads();
   // u = UTI g
   for (int j = warp; j < r; j += nwarps) {
      const T* row = uti + c.uti_off + (int64_t)j * n3;
      T s[RB];
#pragma unroll
      for (int rb = 0; rb < RB; rb++) s[rb] = T(0);
      for (int q = lane; q < n3; q += 32) {
         const T v = row[q];
#pragma unroll
         for (int rb = 0; rb < RB; rb++) s[rb] += v * g[rb * n3 + q];
      }
#pragma unroll
      for (int rb = 0; rb < RB; rb++) {
         const T t = warp_sum(s[rb]);
         if (lane == 0) u[rb * r + j] = t;
      }
   }
   __syncthreads();
   // U u -> staging (each point belongs to exactly one cube of this level)
   for (int q = tid; q < c.p; q += blockDim.x) {
      const T* col = ucm + c.u_off + q;
      T acc[RB];
#pragma unroll
      for (int rb = 0; rb < RB; rb++) acc[rb] = T(0);
      for (int j = 0; j < r; j++) {
         const T v = col[(int64_t)j * c.p];
#pragma unroll
         for (int rb = 0; rb < RB; rb++) acc[rb] += v * u[rb * r + j];
      }
      const int32_t pt = dst_points[c.point_off + q];
#pragma unroll
      for (int rb = 0; rb < RB; rb++)
         staging[(int64_t)(rhs0 + rb) * bs.staging + (int64_t)c.stage * total_points + pt] = acc[rb];
   }
}

constexpr int kWarpCubes = 2;  // cubes (warps) per block (B200: 0.5 % faster solves than 4)
constexpr int kWarpThreads = 32 * kWarpCubes;

// ---- transposed operator (y = A^T x), for the adjoint solve
//
// A = sum over trees of Out^T (S Gs + D Gd + J Gd), with Gs/Gd the scaled gathers of the
// join, S/D the single/double-layer operators (near blocks plus far field) and J the
// jump.  A^T x: gather z = x[out(p)] per tree point, form S^T z and D^T z per tree panel,
// then scatter-add them scaled to the rows the join read.  The far field runs the
// forward pipeline backwards: per destination cube U^T, UTI^T and the forward DFT; the
// translation with the opposite-offset slots (transposed tiles); per source cube the
// inverse DFT, PV_s^T / PV_d^T and VT^T into one staging row per level.  Blocks of one
// cube per block; the DFTs are those of the forward kernels.

// zt[p] = x[out(p)] for every tree point
template <typename T>
__global__ void gather_points_kernel(int64_t total, const int32_t* __restrict__ point_out, const double* __restrict__ x,
                                     T* __restrict__ zt) {
   for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x)
      zt[k] = (T)x[point_out[k]];
}

// per destination cube: a = U^T z (U is p x r), g = UTI^T a on the n^3 grid, F = r2c DFT of
// g at offset n/2, written to the cube's translated-spectrum slot
template <typename T>
__global__ void __launch_bounds__(kFarThreads) far_backward_t_kernel(
    const DstDesc* __restrict__ cubes, const int32_t* __restrict__ dst_points, const T* __restrict__ zt,
    const T* __restrict__ uti, const T* __restrict__ ucm, typename Vec2<T>::type* __restrict__ out_spectra) {
   using T2 = typename Vec2<T>::type;
   extern __shared__ __align__(16) char smem_raw[];
   const DstDesc c = cubes[blockIdx.x];
   const int n = c.n, Np = 2 * n - 1, H = n, off = n / 2, n3 = n * n * n;
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
   char* p = smem_raw;
   T* a = carve<T>(p, c.r);
   T* g = carve<T>(p, n3);
   T2* tw = carve<T2>(p, Np);
   T2* A = carve<T2>(p, n * n * H);
   T2* B = carve<T2>(p, n * Np * H);
   for (int k = tid; k < Np; k += blockDim.x) {  // exp(-2 pi i k / Np)
      T cs, sn;
      Cx<T>::cis(k, Np, &cs, &sn);
      tw[k] = Cx<T>::make(cs, -sn);
   }
   // a_j = sum_q U[q][j] z[q]; U stored r x p (row j contiguous over the points)
   for (int j = warp; j < c.r; j += nwarps) {
      const T* row = ucm + c.u_off + (int64_t)j * c.p;
      T s = T(0);
      for (int q = lane; q < c.p; q += 32) s += row[q] * zt[dst_points[c.point_off + q]];
      s = warp_sum(s);
      if (lane == 0) a[j] = s;
   }
   __syncthreads();
   for (int x = tid; x < n3; x += blockDim.x) {
      T s = T(0);
      for (int j = 0; j < c.r; j++) s += uti[c.uti_off + (int64_t)j * n3 + x] * a[j];
      g[x] = s;
   }
   __syncthreads();
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
   for (int idx = tid; idx < n * Np * H; idx += blockDim.x) {
      const int kf = idx % H, jf = (idx / H) % Np, i = idx / (H * Np);
      T2 acc = Cx<T>::make(T(0), T(0));
      for (int j = 0; j < n; j++) acc = Cx<T>::fma(A[(i * n + j) * H + kf], tw[((j + off) * jf) % Np], acc);
      B[idx] = acc;
   }
   __syncthreads();
   T2* out = out_spectra + c.s_off;
   for (int idx = tid; idx < Np * Np * H; idx += blockDim.x) {
      const int kf = idx % H, jf = (idx / H) % Np, fi = idx / (H * Np);
      T2 acc = Cx<T>::make(T(0), T(0));
      for (int i = 0; i < n; i++) acc = Cx<T>::fma(B[(i * Np + jf) * H + kf], tw[((i + off) * fi) % Np], acc);
      out[idx] = acc;
   }
}

// per source cube: g = c2r DFT of the translated spectrum (cropped at n/2, scaled),
// a_s = PV_s^T g, a_d = PV_d^T g, and per panel {VT^T a_s, VT^T a_d} into the level's
// staging row (each panel belongs to one source cube per level)
template <typename T>
__global__ void __launch_bounds__(kFarThreads) far_forward_t_kernel(
    const SrcDesc* __restrict__ cubes, const int32_t* __restrict__ src_panels,
    const typename Vec2<T>::type* __restrict__ in_spectra, const T* __restrict__ vt,
    const typename Vec2<T>::type* __restrict__ pv, typename Vec2<T>::type* __restrict__ staging,
    int64_t total_panels) {
   using T2 = typename Vec2<T>::type;
   extern __shared__ __align__(16) char smem_raw[];
   const SrcDesc c = cubes[blockIdx.x];
   const int n = c.n, Np = 2 * n - 1, H = n, off = n / 2, n3 = n * n * n, pg = Np * Np * H;
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5;
   char* p = smem_raw;
   T2* S = carve<T2>(p, pg);
   T2* P1 = carve<T2>(p, n * Np * H);
   T2* P2 = carve<T2>(p, n * n * H);
   T* g = carve<T>(p, n3);
   T2* a = carve<T2>(p, c.r);
   T2* tw = carve<T2>(p, Np);
   for (int k = tid; k < Np; k += blockDim.x) {  // exp(+2 pi i k / Np)
      T cs, sn;
      Cx<T>::cis(k, Np, &cs, &sn);
      tw[k] = Cx<T>::make(cs, sn);
   }
   for (int f = tid; f < pg; f += blockDim.x) S[f] = in_spectra[c.spec_off + f];
   __syncthreads();
   for (int idx = tid; idx < n * Np * H; idx += blockDim.x) {
      const int kf = idx % H, jf = (idx / H) % Np, i = idx / (H * Np);
      T2 acc = Cx<T>::make(T(0), T(0));
      for (int fi = 0; fi < Np; fi++) acc = Cx<T>::fma(S[(fi * Np + jf) * H + kf], tw[((i + off) * fi) % Np], acc);
      P1[idx] = acc;
   }
   __syncthreads();
   for (int idx = tid; idx < n * n * H; idx += blockDim.x) {
      const int kf = idx % H, j = (idx / H) % n, i = idx / (H * n);
      T2 acc = Cx<T>::make(T(0), T(0));
      for (int jf = 0; jf < Np; jf++) acc = Cx<T>::fma(P1[(i * Np + jf) * H + kf], tw[((j + off) * jf) % Np], acc);
      P2[idx] = acc;
   }
   __syncthreads();
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
   // a_j = {sum_x PV_s[j][x] g[x], sum_x PV_d[j][x] g[x]}; pv stored r x n^3 of pairs
   for (int j = warp; j < c.r; j += nwarps) {
      const T2* row = pv + c.pv_off + (int64_t)j * n3;
      T s = T(0), d = T(0);
      for (int x = lane; x < n3; x += 32) {
         const T2 w = row[x];
         s += w.x * g[x];
         d += w.y * g[x];
      }
      s = warp_sum(s);
      d = warp_sum(d);
      if (lane == 0) a[j] = Cx<T>::make(s, d);
   }
   __syncthreads();
   T2* stage = staging + (int64_t)c.level * total_panels;
   for (int i = tid; i < c.m; i += blockDim.x) {
      T s = T(0), d = T(0);
      for (int j = 0; j < c.r; j++) {
         const T v = vt[c.vt_off + (int64_t)j * c.m + i];
         s += v * a[j].x;
         d += v * a[j].y;
      }
      stage[src_panels[c.panel_off + i]] = Cx<T>::make(s, d);
   }
}

// dynamic shared memory of the transposed far-field kernels (their carve order, 16-byte aligned)
template <typename T>
static int far_backward_t_smem(int n, int r) {
   const int Np = 2 * n - 1, H = n, T2s = 2 * (int)sizeof(T);
   return 16 * 6 + r * (int)sizeof(T) + n * n * n * (int)sizeof(T) + Np * T2s + n * n * H * T2s + n * Np * H * T2s;
}
template <typename T>
static int far_forward_t_smem(int n, int r) {
   const int Np = 2 * n - 1, H = n, T2s = 2 * (int)sizeof(T);
   return 16 * 7 + Np * Np * H * T2s + n * Np * H * T2s + n * n * H * T2s + n * n * n * (int)sizeof(T) + r * T2s +
          Np * T2s;
}

// per leaf (one warp): column sums of the near-field blocks against the leaf's gathered
// rows, {sum_r Ds[r][c] z[r], sum_r Dd[r][c] z[r]}, added to the column's panel
template <typename T>
__global__ void __launch_bounds__(kWarpThreads) near_t_kernel(const LeafDesc* __restrict__ leaves, int n_leaf,
                                                              const int32_t* __restrict__ rows,
                                                              const int32_t* __restrict__ cols,
                                                              const typename Vec2<T>::type* __restrict__ d,
                                                              const T* __restrict__ zt, double2* __restrict__ ut,
                                                              int32_t zero_slot) {
   using T2 = typename Vec2<T>::type;
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   const int leaf = blockIdx.x * kWarpCubes + warp;
   if (leaf >= n_leaf) return;
   const LeafDesc L = leaves[leaf];
   for (int c = lane; c < L.ncols; c += 32) {
      const int k = cols[L.col_off + c];
      if (k == zero_slot) continue;  // padding column
      double s = 0.0, dd = 0.0;
      for (int r = 0; r < L.nrows; r++) {
         const T2 v = d[L.d_off + (int64_t)r * L.ncols + c];
         const double z = (double)zt[rows[L.row_off + r]];
         s += (double)v.x * z;
         dd += (double)v.y * z;
      }
      atomicAdd(&ut[k].x, s);
      atomicAdd(&ut[k].y, dd);
   }
}

// per tree panel k: single-layer and double-layer sums (near, far levels, jump), added
// scaled to the rows its join read: y[dphi(k)] += dphi_scale s, y[phi(k)] += phi_scale d
template <typename T>
__global__ void scatter_panels_kernel(int64_t np, const double2* __restrict__ ut,
                                      const typename Vec2<T>::type* __restrict__ staging, int levels,
                                      int64_t total_panels, const double* __restrict__ panel_jump,
                                      const int32_t* __restrict__ panel_point, const T* __restrict__ zt,
                                      const int32_t* __restrict__ phi_idx, const double* __restrict__ phi_scale,
                                      const int32_t* __restrict__ dphi_idx, const double* __restrict__ dphi_scale,
                                      double* __restrict__ y) {
   for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < np; k += (int64_t)gridDim.x * blockDim.x) {
      double s = ut[k].x, d = ut[k].y;
      for (int l = 0; l < levels; l++) {
         const auto v = staging[(int64_t)l * total_panels + k];
         s += (double)v.x;
         d += (double)v.y;
      }
      const int q = panel_point[k];
      if (q >= 0) d += panel_jump[k] * (double)zt[q];
      atomicAdd(&y[dphi_idx[k]], dphi_scale[k] * s);
      atomicAdd(&y[phi_idx[k]], phi_scale[k] * d);
   }
}

// ---- one warp per cube for the small grids of the fine levels
//
// Most cubes sit on the finest levels, where the grid is 4^3 and a cube holds a
// few panels: a whole block per cube spends its time on launch and barrier
// latency.  These kernels give each cube one warp (several cubes per block),
// replace barriers by __syncwarp, and fix the grid edge at compile time.  The
// arithmetic is the block kernels' (same DFT factorisation and twiddles).


template <int N>
struct SmallGrid {
   static constexpr int Np = 2 * N - 1, H = N, OFF = N / 2, N3 = N * N * N;
   static constexpr int NA = N * N * H, NB = N * Np * H, PG = Np * Np * H;
   static constexpr int kFwdElems = NA + NB + (N3 + 1) / 2;  // A, B and the real grid g, in complex units
   static constexpr int kBwdElems = PG + NB;                 // S (later P2, u) and P1 (later g)
};

template <typename T, int N>
__global__ void __launch_bounds__(kWarpThreads, 24) far_forward_warp_kernel(
    const SrcDesc* __restrict__ cubes, int count, const int32_t* __restrict__ src_panels,
    const typename Vec2<T>::type* __restrict__ xsd, const T* __restrict__ vt,
    const typename Vec2<T>::type* __restrict__ pv, typename Vec2<T>::type* __restrict__ spectra, BatchStrides bs) {
   using T2 = typename Vec2<T>::type;
   const int rhs = blockIdx.x % bs.nrhs, unit = blockIdx.x / bs.nrhs;  // right-hand side fastest
   xsd += rhs * bs.panels;
   spectra += rhs * bs.spectra;
   using G = SmallGrid<N>;
   constexpr int Np = G::Np, H = G::H, OFF = G::OFF, N3 = G::N3;
   constexpr unsigned kAll = 0xffffffffu;
   __shared__ T2 tw[Np];
   __shared__ __align__(16) T2 work[kWarpCubes][G::kFwdElems];
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   if (threadIdx.x < Np) {  // exp(-2 pi i k / Np)
      T cs, sn;
      Cx<T>::cis(threadIdx.x, Np, &cs, &sn);
      tw[threadIdx.x] = Cx<T>::make(cs, -sn);
   }
   __syncthreads();
   const int cube = unit * kWarpCubes + warp;
   if (cube >= count) return;
   const SrcDesc c = cubes[cube];
   T2* A = work[warp];
   T2* B = A + G::NA;
   T* g = reinterpret_cast<T*>(B + G::NB);
   const int m = c.m, r = c.r;  // r <= 32: lane j owns row j of VT
   // a = VT x, panels broadcast from the lane that loaded them, 32 at a time
   T as = T(0), ad = T(0);
   const T* row = vt + c.vt_off + (int64_t)min(lane, r - 1) * m;
   for (int base = 0; base < m; base += 32) {
      T2 xv = Cx<T>::make(T(0), T(0));
      if (base + lane < m) xv = xsd[src_panels[c.panel_off + base + lane]];
      const int cnt = min(32, m - base);
#pragma unroll 8
      for (int i = 0; i < cnt; i++) {
         const T xs = __shfl_sync(kAll, xv.x, i), xd = __shfl_sync(kAll, xv.y, i);
         if (lane < r) {
            const T v = row[base + i];
            as += v * xs;
            ad += v * xd;
         }
      }
   }
   // grid charges g = PV_s a_s + PV_d a_d, lanes over grid points
   constexpr int QT = (N3 + 31) / 32;
   T acc[QT];
#pragma unroll
   for (int t = 0; t < QT; t++) acc[t] = T(0);
   const T2* pvc = pv + c.pv_off;
#pragma unroll 4
   for (int j = 0; j < r; j++) {
      const T s = __shfl_sync(kAll, as, j), d = __shfl_sync(kAll, ad, j);
#pragma unroll
      for (int t = 0; t < QT; t++) {
         const int q = lane + 32 * t;
         if (q < N3) {
            const T2 w = pvc[(int64_t)j * N3 + q];
            acc[t] += w.x * s + w.y * d;
         }
      }
   }
#pragma unroll
   for (int t = 0; t < QT; t++)
      if (lane + 32 * t < N3) g[lane + 32 * t] = acc[t];
   __syncwarp();
   // DFT along k (input index k + OFF), half spectrum kf < H
   for (int idx = lane; idx < G::NA; idx += 32) {
      const int kf = idx % H, ij = idx / H;
      const T* line = g + ij * N;
      T2 a = Cx<T>::make(T(0), T(0));
#pragma unroll
      for (int k = 0; k < N; k++) {
         const T2 w = tw[((k + OFF) * kf) % Np];
         a.x += line[k] * w.x;
         a.y += line[k] * w.y;
      }
      A[idx] = a;
   }
   __syncwarp();
   // along j
   for (int idx = lane; idx < G::NB; idx += 32) {
      const int kf = idx % H, jf = (idx / H) % Np, i = idx / (H * Np);
      T2 a = Cx<T>::make(T(0), T(0));
#pragma unroll
      for (int j = 0; j < N; j++) a = Cx<T>::fma(A[(i * N + j) * H + kf], tw[((j + OFF) * jf) % Np], a);
      B[idx] = a;
   }
   __syncwarp();
   // along i, straight to global
   T2* out = spectra + c.spec_off;
   for (int idx = lane; idx < G::PG; idx += 32) {
      const int kf = idx % H, jf = (idx / H) % Np, fi = idx / (H * Np);
      T2 a = Cx<T>::make(T(0), T(0));
#pragma unroll
      for (int i = 0; i < N; i++) a = Cx<T>::fma(B[(i * Np + jf) * H + kf], tw[((i + OFF) * fi) % Np], a);
      out[idx] = a;
   }
}

template <typename T, int N>
__global__ void __launch_bounds__(kWarpThreads) far_backward_warp_kernel(
    const DstDesc* __restrict__ cubes, int count, const int32_t* __restrict__ dst_points,
    const typename Vec2<T>::type* __restrict__ translated, const T* __restrict__ uti, const T* __restrict__ ucm,
    T* __restrict__ staging, int64_t total_points, BatchStrides bs) {
   using T2 = typename Vec2<T>::type;
   const int rhs = blockIdx.x % bs.nrhs, unit = blockIdx.x / bs.nrhs;  // right-hand side fastest
   translated += rhs * bs.translated;
   staging += rhs * bs.staging;
   using G = SmallGrid<N>;
   constexpr int Np = G::Np, H = G::H, OFF = G::OFF, N3 = G::N3;
   constexpr unsigned kAll = 0xffffffffu;
   __shared__ T2 tw[Np];
   __shared__ __align__(16) T2 work[kWarpCubes][G::kBwdElems];
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   if (threadIdx.x < Np) {  // exp(+2 pi i k / Np)
      T cs, sn;
      Cx<T>::cis(threadIdx.x, Np, &cs, &sn);
      tw[threadIdx.x] = Cx<T>::make(cs, sn);
   }
   __syncthreads();
   const int cube = unit * kWarpCubes + warp;
   if (cube >= count) return;
   const DstDesc c = cubes[cube];
   T2* S = work[warp];
   T2* P1 = S + G::PG;
   for (int f = lane; f < G::PG; f += 32) S[f] = translated[c.s_off + f];
   __syncwarp();
   // inverse along i (output i < N only)
   for (int idx = lane; idx < G::NB; idx += 32) {
      const int kf = idx % H, jf = (idx / H) % Np, i = idx / (H * Np);
      T2 a = Cx<T>::make(T(0), T(0));
#pragma unroll
      for (int fi = 0; fi < Np; fi++) a = Cx<T>::fma(S[(fi * Np + jf) * H + kf], tw[((i + OFF) * fi) % Np], a);
      P1[idx] = a;
   }
   __syncwarp();
   // inverse along j (output j < N only), into the space of S
   T2* P2 = S;
   for (int idx = lane; idx < G::NA; idx += 32) {
      const int kf = idx % H, j = (idx / H) % N, i = idx / (H * N);
      T2 a = Cx<T>::make(T(0), T(0));
#pragma unroll
      for (int jf = 0; jf < Np; jf++) a = Cx<T>::fma(P1[(i * Np + jf) * H + kf], tw[((j + OFF) * jf) % Np], a);
      P2[idx] = a;
   }
   __syncwarp();
   // Hermitian half along k -> real, cropped, scaled; into the space of P1
   T* g = reinterpret_cast<T*>(P1);
   const T scale = T(1) / (T)(Np * Np * Np);
   for (int q = lane; q < N3; q += 32) {
      const int k = q % N, ij = q / N;
      const T2* line = P2 + ij * H;
      T a = line[0].x;
#pragma unroll
      for (int kf = 1; kf < H; kf++) {
         const T2 w = tw[((k + OFF) * kf) % Np];
         a += T(2) * (line[kf].x * w.x - line[kf].y * w.y);
      }
      g[q] = a * scale;
   }
   __syncwarp();
   // u = UTI g: four lanes per row, eight rows per pass; u into the space of S
   T* u = reinterpret_cast<T*>(S);
   const int r = c.r, quarter = lane & 3;
   for (int j0 = 0; j0 < r; j0 += 8) {
      const int j = j0 + (lane >> 2);
      T s = T(0);
      if (j < r) {
         const T* urow = uti + c.uti_off + (int64_t)j * N3;
#pragma unroll 8
         for (int q = quarter; q < N3; q += 4) s += urow[q] * g[q];
      }
      s += __shfl_xor_sync(kAll, s, 1);
      s += __shfl_xor_sync(kAll, s, 2);
      if (quarter == 0 && j < r) u[j] = s;
   }
   __syncwarp();
   // U u -> staging (each point belongs to exactly one cube of this level)
   T* stage = staging + (int64_t)c.stage * total_points;
   const T* ucol = ucm + c.u_off;
   for (int q = lane; q < c.p; q += 32) {
      T a = T(0);
#pragma unroll 4
      for (int j = 0; j < r; j++) a += ucol[(int64_t)j * c.p + q] * u[j];
      stage[dst_points[c.point_off + q]] = a;
   }
}

// ---- the 4^3 grid (7 x 7 x 4 half spectrum) with the DFT held in registers
//
// Lane L = 16 hi + 4 jp + kq and register h address grid point q = L + 32 h, i.e.
// (i, j, k) = (2 h + hi, jp, kq).  Each separable DFT stage gathers its inputs
// with shuffles from the lanes that hold them, and every twiddle is either a
// compile-time entry of the 7-point table or precomputed per lane, so the
// stages run without index arithmetic.  Spectrum row fi (28 complex values,
// (jf, kf) = (jp + 4 hi, kq)) is written or read by lanes 0..27 as one
// contiguous segment.  Same factorisation and twiddles as the generic kernels.

template <typename T>
__device__ inline typename Vec2<T>::type shfl_c(typename Vec2<T>::type v, int src) {
   v.x = __shfl_sync(0xffffffffu, v.x, src);
   v.y = __shfl_sync(0xffffffffu, v.y, src);
   return v;
}

// Bulk asynchronous prefetch (the TMA engine's cp.async.bulk.prefetch.L2) of bytes
// [off, off + len) of a buffer of buf_bytes into L2: 16-byte aligned pieces of at most
// 32 KiB that stay inside the buffer.  A prefetch only warms L2: it writes nothing, and
// nothing waits for it.
__device__ inline void prefetch_l2(const void* base, int64_t buf_bytes, int64_t off, int64_t len) {
   int64_t a = off & ~int64_t(15);
   const int64_t e = min((off + len + 15) & ~int64_t(15), buf_bytes & ~int64_t(15));
   const char* p = static_cast<const char*>(base);
   while (a < e) {
      const unsigned n = (unsigned)min(e - a, int64_t(32768));
      asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p + a), "r"(n) : "memory");
      a += n;
   }
}

// Bytes of the operator buffers the streaming kernels prefetch from, and how far ahead:
// a warp about to work on unit u (a cube, or a leaf) prefetches the blocks of unit
// u + ahead, the unit the same warp slot of the next wave of resident blocks will take
// (ahead = resident warps of the launch; 0 disables the prefetch).
struct Prefetch {
   int64_t ahead = 0;
   int64_t a_bytes = 0, b_bytes = 0, c_bytes = 0;  // VT, PV | UTI, U, translated | D
};

template <typename T>
__global__ void __launch_bounds__(kWarpThreads, sizeof(T) == 4 ? 16 : 8) far_forward_n4_kernel(
    const SrcDesc* __restrict__ cubes, int count, const int32_t* __restrict__ src_panels,
    const typename Vec2<T>::type* __restrict__ xsd, const T* __restrict__ vt,
    const typename Vec2<T>::type* __restrict__ pv, typename Vec2<T>::type* __restrict__ spectra, BatchStrides bs,
    Prefetch pre) {
   using T2 = typename Vec2<T>::type;
   const int rhs = blockIdx.x % bs.nrhs, unit = blockIdx.x / bs.nrhs;  // right-hand side fastest
   xsd += rhs * bs.panels;
   spectra += rhs * bs.spectra;
   constexpr int N = 4, Np = 7, OFF = 2, N3 = 64, ROW = Np * N;  // ROW: complex values per fi
   constexpr unsigned kAll = 0xffffffffu;
   __shared__ T2 tw[Np];
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   if (threadIdx.x < Np) {  // exp(-2 pi i k / 7)
      T cs, sn;
      Cx<T>::cis(threadIdx.x, Np, &cs, &sn);
      tw[threadIdx.x] = Cx<T>::make(cs, -sn);
   }
   __syncthreads();
   const int cube = unit * kWarpCubes + warp;
   if (cube >= count) return;
   const SrcDesc c = cubes[cube];
   if (pre.ahead > 0 && rhs == 0 && lane == 0 && cube + pre.ahead < count) {
      const SrcDesc nc = cubes[cube + pre.ahead];
      prefetch_l2(vt, pre.a_bytes, nc.vt_off * (int64_t)sizeof(T), (int64_t)nc.r * nc.m * (int64_t)sizeof(T));
      prefetch_l2(pv, pre.b_bytes, nc.pv_off * (int64_t)sizeof(T2), (int64_t)nc.r * 64 * (int64_t)sizeof(T2));
   }
   const int m = c.m, r = c.r;  // r <= 32: lane j owns row j of VT
   const int kq = lane & 3, jp = (lane >> 2) & 3, hi = lane >> 4;
   // per-lane twiddles: stage k (kf = kq) and stage j (jf = jp, jp + 4)
   T2 w1[N], w2[2][N], W[Np];
#pragma unroll
   for (int k = 0; k < N; k++) w1[k] = tw[((k + OFF) * kq) % Np];
#pragma unroll
   for (int sl = 0; sl < 2; sl++)
#pragma unroll
      for (int j = 0; j < N; j++) w2[sl][j] = tw[((j + OFF) * (jp + 4 * sl)) % Np];
#pragma unroll
   for (int q = 0; q < Np; q++) W[q] = tw[q];
   // FP64: the first PF rows of PV (they depend only on the cube) are in flight during
   // VT x (FP32 keeps its registers for occupancy instead)
   constexpr int PF = sizeof(T) == 8 ? 4 : 0;
   const T2* pvc = pv + c.pv_off + lane;
   T2 pf0[PF > 0 ? PF : 1], pf1[PF > 0 ? PF : 1];
#pragma unroll
   for (int j = 0; j < PF; j++) {
      pf0[j] = pf1[j] = Cx<T>::make(T(0), T(0));
      if (j < r) {
         pf0[j] = pvc[(int64_t)j * N3];
         pf1[j] = pvc[(int64_t)j * N3 + 32];
      }
   }
   // a = VT x
   T as = T(0), ad = T(0);
   const T* row = vt + c.vt_off + (int64_t)min(lane, r - 1) * m;
   for (int base = 0; base < m; base += 32) {
      T2 xv = Cx<T>::make(T(0), T(0));
      if (base + lane < m) xv = xsd[src_panels[c.panel_off + base + lane]];
      const int cnt = min(32, m - base);
#pragma unroll 8
      for (int i = 0; i < cnt; i++) {
         const T xs = __shfl_sync(kAll, xv.x, i), xd = __shfl_sync(kAll, xv.y, i);
         if (lane < r) {
            const T v = row[base + i];
            as += v * xs;
            ad += v * xd;
         }
      }
   }
   // grid charges at q = lane and lane + 32
   T g0 = T(0), g1 = T(0);
#pragma unroll
   for (int j = 0; j < PF; j++)
      if (j < r) {
         const T s = __shfl_sync(kAll, as, j), d = __shfl_sync(kAll, ad, j);
         g0 += pf0[j].x * s + pf0[j].y * d;
         g1 += pf1[j].x * s + pf1[j].y * d;
      }
#pragma unroll 4
   for (int j = PF; j < r; j++) {
      const T s = __shfl_sync(kAll, as, j), d = __shfl_sync(kAll, ad, j);
      const T2 w0 = pvc[(int64_t)j * N3], w1v = pvc[(int64_t)j * N3 + 32];
      g0 += w0.x * s + w0.y * d;
      g1 += w1v.x * s + w1v.y * d;
   }
   // along k: lane computes kf = kq of line (i, jp) from the four lanes of its quad
   T2 A[2];
#pragma unroll
   for (int h = 0; h < 2; h++) {
      const T g = h ? g1 : g0;
      T2 a = Cx<T>::make(T(0), T(0));
#pragma unroll
      for (int k = 0; k < N; k++) {
         const T gk = __shfl_sync(kAll, g, (lane & ~3) | k);
         a.x += gk * w1[k].x;
         a.y += gk * w1[k].y;
      }
      A[h] = a;
   }
   // along j: lane computes jf = jp and jp + 4 of column (i, kq)
   T2 B[2][2];
#pragma unroll
   for (int h = 0; h < 2; h++) {
      T2 Aj[N];
#pragma unroll
      for (int j = 0; j < N; j++) Aj[j] = shfl_c<T>(A[h], (lane & ~12) | (j << 2));
#pragma unroll
      for (int sl = 0; sl < 2; sl++) {
         T2 b = Cx<T>::make(T(0), T(0));
#pragma unroll
         for (int j = 0; j < N; j++) b = Cx<T>::fma(Aj[j], w2[sl][j], b);
         B[h][sl] = b;
      }
   }
   // along i: lanes hi = 0 finish jf = jp, lanes hi = 1 jf = jp + 4, exchanging
   // with lane ^ 16 the two values of i (2 h + hi) that the partner needs
   T2 Bi[N];
#pragma unroll
   for (int h = 0; h < 2; h++) {
      const T2 mine = hi ? B[h][1] : B[h][0];
      const T2 recv = shfl_c<T>(hi ? B[h][0] : B[h][1], lane ^ 16);
      Bi[2 * h] = hi ? recv : mine;
      Bi[2 * h + 1] = hi ? mine : recv;
   }
   T2* out = spectra + c.spec_off + lane;
   if (lane < ROW) {
#pragma unroll
      for (int fi = 0; fi < Np; fi++) {
         T2 o = Cx<T>::make(T(0), T(0));
#pragma unroll
         for (int i = 0; i < N; i++) o = Cx<T>::fma(Bi[i], W[((i + OFF) * fi) % Np], o);
         out[fi * ROW] = o;
      }
   }
}

template <typename T>
__global__ void __launch_bounds__(kWarpThreads, sizeof(T) == 4 ? 16 : 8) far_backward_n4_kernel(
    const DstDesc* __restrict__ cubes, int count, const int32_t* __restrict__ dst_points,
    const typename Vec2<T>::type* __restrict__ translated, const T* __restrict__ uti, const T* __restrict__ ucm,
    T* __restrict__ staging, int64_t total_points, BatchStrides bs, Prefetch pre) {
   using T2 = typename Vec2<T>::type;
   const int rhs = blockIdx.x % bs.nrhs, unit = blockIdx.x / bs.nrhs;  // right-hand side fastest
   translated += rhs * bs.translated;
   staging += rhs * bs.staging;
   constexpr int N = 4, Np = 7, OFF = 2, N3 = 64, ROW = Np * N;
   constexpr unsigned kAll = 0xffffffffu;
   __shared__ T2 tw[Np];
   __shared__ __align__(16) T2 work[kWarpCubes][N * ROW];  // P1 [i][jf][kf], later g and u
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   if (threadIdx.x < Np) {  // exp(+2 pi i k / 7)
      T cs, sn;
      Cx<T>::cis(threadIdx.x, Np, &cs, &sn);
      tw[threadIdx.x] = Cx<T>::make(cs, sn);
   }
   __syncthreads();
   const int cube = unit * kWarpCubes + warp;
   if (cube >= count) return;
   const DstDesc c = cubes[cube];
   if (pre.ahead > 0 && rhs == 0 && lane == 0 && cube + pre.ahead < count) {
      const DstDesc nc = cubes[cube + pre.ahead];
      prefetch_l2(uti, pre.a_bytes, nc.uti_off * (int64_t)sizeof(T), (int64_t)nc.r * N3 * (int64_t)sizeof(T));
      prefetch_l2(ucm, pre.b_bytes, nc.u_off * (int64_t)sizeof(T), (int64_t)nc.r * nc.p * (int64_t)sizeof(T));
   }
   const int kq = lane & 3, jp = (lane >> 2) & 3;
   T2 W[Np], w2[Np], w3[N];
#pragma unroll
   for (int q = 0; q < Np; q++) W[q] = tw[q];
#pragma unroll
   for (int jf = 0; jf < Np; jf++) w2[jf] = tw[((jp + OFF) * jf) % Np];
#pragma unroll
   for (int kf = 0; kf < N; kf++) w3[kf] = tw[((kq + OFF) * kf) % Np];
   T2* P1 = work[warp];
   // inverse along i (i < 4) of column (jf, kf) = (jp + 4 hi, kq), straight from global
   if (lane < ROW) {
      T2 S[Np];
      const T2* in = translated + c.s_off + lane;
#pragma unroll
      for (int fi = 0; fi < Np; fi++) S[fi] = in[fi * ROW];
#pragma unroll
      for (int i = 0; i < N; i++) {
         T2 a = Cx<T>::make(T(0), T(0));
#pragma unroll
         for (int fi = 0; fi < Np; fi++) a = Cx<T>::fma(S[fi], W[((i + OFF) * fi) % Np], a);
         P1[i * ROW + lane] = a;
      }
   }
   __syncwarp();
   // inverse along j (j = jp < 4) for i = 2 h + hi, kf = kq
   T2 P2[2];
#pragma unroll
   for (int h = 0; h < 2; h++) {
      const int i = 2 * h + (lane >> 4);
      T2 a = Cx<T>::make(T(0), T(0));
#pragma unroll
      for (int jf = 0; jf < Np; jf++) a = Cx<T>::fma(P1[i * ROW + jf * N + kq], w2[jf], a);
      P2[h] = a;
   }
   // Hermitian half along k -> real grid value (i, jp, k = kq), cropped and scaled
   const T scale = T(1) / (T)(Np * Np * Np);
   T g[2];
#pragma unroll
   for (int h = 0; h < 2; h++) {
      const T2 p0 = shfl_c<T>(P2[h], lane & ~3);
      T a = p0.x;
#pragma unroll
      for (int kf = 1; kf < N; kf++) {
         const T2 pk = shfl_c<T>(P2[h], (lane & ~3) | kf);
         a += T(2) * (pk.x * w3[kf].x - pk.y * w3[kf].y);
      }
      g[h] = a * scale;
   }
   __syncwarp();  // P1 is reused for g and u
   T* gs = reinterpret_cast<T*>(P1);
   gs[lane] = g[0];
   gs[lane + 32] = g[1];
   T* u = gs + N3;
   __syncwarp();
   // u = UTI g: four lanes per row, eight rows per pass
   const int r = c.r, quarter = lane & 3;
   for (int j0 = 0; j0 < r; j0 += 8) {
      const int j = j0 + (lane >> 2);
      T sum = T(0);
      if (j < r) {
         const T* urow = uti + c.uti_off + (int64_t)j * N3;
#pragma unroll
         for (int q = quarter; q < N3; q += 4) sum += urow[q] * gs[q];
      }
      sum += __shfl_xor_sync(kAll, sum, 1);
      sum += __shfl_xor_sync(kAll, sum, 2);
      if (quarter == 0 && j < r) u[j] = sum;
   }
   __syncwarp();
   // U u -> staging (each point belongs to exactly one cube of this level)
   T* stage = staging + (int64_t)c.stage * total_points;
   const T* ucol = ucm + c.u_off;
   for (int q = lane; q < c.p; q += 32) {
      T a = T(0);
#pragma unroll 4
      for (int j = 0; j < r; j++) a += ucol[(int64_t)j * c.p + q] * u[j];
      stage[dst_points[c.point_off + q]] = a;
   }
}

// ---- the transposed 4^3 transforms, one cube per warp with the DFT in registers
// (lane and register layout of far_forward_n4_kernel / far_backward_n4_kernel: grid
// point q = lane + 32 h)

// per destination cube: a = U^T z (lane j accumulates row j, the points broadcast 32 at
// a time), g = UTI^T a at q = lane and lane + 32, F = r2c DFT of g into the cube's
// translated-spectrum slot
template <typename T>
__global__ void __launch_bounds__(kWarpThreads, sizeof(T) == 4 ? 16 : 8) far_backward_t_n4_kernel(
    const DstDesc* __restrict__ cubes, int count, const int32_t* __restrict__ dst_points, const T* __restrict__ zt,
    const T* __restrict__ uti, const T* __restrict__ ucm, typename Vec2<T>::type* __restrict__ out_spectra) {
   using T2 = typename Vec2<T>::type;
   constexpr int N = 4, Np = 7, OFF = 2, N3 = 64, ROW = Np * N;
   constexpr unsigned kAll = 0xffffffffu;
   __shared__ T2 tw[Np];
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   if (threadIdx.x < Np) {  // exp(-2 pi i k / 7)
      T cs, sn;
      Cx<T>::cis(threadIdx.x, Np, &cs, &sn);
      tw[threadIdx.x] = Cx<T>::make(cs, -sn);
   }
   __syncthreads();
   const int cube = blockIdx.x * kWarpCubes + warp;
   if (cube >= count) return;
   const DstDesc c = cubes[cube];
   const int p = c.p, r = c.r;  // r <= 32: lane j owns row j of U^T
   T a = T(0);
   const T* urow = ucm + c.u_off + (int64_t)min(lane, r - 1) * p;
   for (int base = 0; base < p; base += 32) {
      const T zv = base + lane < p ? zt[dst_points[c.point_off + base + lane]] : T(0);
      const int cnt = min(32, p - base);
#pragma unroll 8
      for (int i = 0; i < cnt; i++) {
         const T zi = __shfl_sync(kAll, zv, i);
         if (lane < r) a += urow[base + i] * zi;
      }
   }
   T g0 = T(0), g1 = T(0);
   const T* uc = uti + c.uti_off + lane;
#pragma unroll 4
   for (int j = 0; j < r; j++) {
      const T aj = __shfl_sync(kAll, a, j);
      g0 += uc[(int64_t)j * N3] * aj;
      g1 += uc[(int64_t)j * N3 + 32] * aj;
   }
   // r2c DFT of g: stage k, stage j, stage i (as far_forward_n4_kernel)
   const int kq = lane & 3, jp = (lane >> 2) & 3, hi = lane >> 4;
   T2 w1[N], w2[2][N], W[Np];
#pragma unroll
   for (int k = 0; k < N; k++) w1[k] = tw[((k + OFF) * kq) % Np];
#pragma unroll
   for (int sl = 0; sl < 2; sl++)
#pragma unroll
      for (int j = 0; j < N; j++) w2[sl][j] = tw[((j + OFF) * (jp + 4 * sl)) % Np];
#pragma unroll
   for (int q = 0; q < Np; q++) W[q] = tw[q];
   T2 A[2];
#pragma unroll
   for (int h = 0; h < 2; h++) {
      const T gv = h ? g1 : g0;
      T2 s = Cx<T>::make(T(0), T(0));
#pragma unroll
      for (int k = 0; k < N; k++) {
         const T gk = __shfl_sync(kAll, gv, (lane & ~3) | k);
         s.x += gk * w1[k].x;
         s.y += gk * w1[k].y;
      }
      A[h] = s;
   }
   T2 B[2][2];
#pragma unroll
   for (int h = 0; h < 2; h++) {
      T2 Aj[N];
#pragma unroll
      for (int j = 0; j < N; j++) Aj[j] = shfl_c<T>(A[h], (lane & ~12) | (j << 2));
#pragma unroll
      for (int sl = 0; sl < 2; sl++) {
         T2 s = Cx<T>::make(T(0), T(0));
#pragma unroll
         for (int j = 0; j < N; j++) s = Cx<T>::fma(Aj[j], w2[sl][j], s);
         B[h][sl] = s;
      }
   }
   T2 Bi[N];
#pragma unroll
   for (int h = 0; h < 2; h++) {
      const T2 mine = hi ? B[h][1] : B[h][0];
      const T2 recv = shfl_c<T>(hi ? B[h][0] : B[h][1], lane ^ 16);
      Bi[2 * h] = hi ? recv : mine;
      Bi[2 * h + 1] = hi ? mine : recv;
   }
   T2* out = out_spectra + c.s_off + lane;
   if (lane < ROW) {
#pragma unroll
      for (int fi = 0; fi < Np; fi++) {
         T2 o = Cx<T>::make(T(0), T(0));
#pragma unroll
         for (int i = 0; i < N; i++) o = Cx<T>::fma(Bi[i], W[((i + OFF) * fi) % Np], o);
         out[fi * ROW] = o;
      }
   }
}

// per source cube: g = c2r DFT of the spectrum (cropped at offset 2, scaled by 1/343),
// a_j = {PV_s[j] . g, PV_d[j] . g}, and per panel {VT^T a_s, VT^T a_d} into the level's
// staging row
template <typename T>
__global__ void __launch_bounds__(kWarpThreads, sizeof(T) == 4 ? 16 : 8) far_forward_t_n4_kernel(
    const SrcDesc* __restrict__ cubes, int count, const int32_t* __restrict__ src_panels,
    const typename Vec2<T>::type* __restrict__ in_spectra, const T* __restrict__ vt,
    const typename Vec2<T>::type* __restrict__ pv, typename Vec2<T>::type* __restrict__ staging,
    int64_t total_panels) {
   using T2 = typename Vec2<T>::type;
   constexpr int N = 4, Np = 7, OFF = 2, N3 = 64, ROW = Np * N;
   constexpr unsigned kAll = 0xffffffffu;
   __shared__ T2 tw[Np];
   __shared__ __align__(16) T2 work[kWarpCubes][N * ROW];  // P1 [i][jf][kf], later a
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   if (threadIdx.x < Np) {  // exp(+2 pi i k / 7)
      T cs, sn;
      Cx<T>::cis(threadIdx.x, Np, &cs, &sn);
      tw[threadIdx.x] = Cx<T>::make(cs, sn);
   }
   __syncthreads();
   const int cube = blockIdx.x * kWarpCubes + warp;
   if (cube >= count) return;
   const SrcDesc c = cubes[cube];
   const int kq = lane & 3, jp = (lane >> 2) & 3;
   T2 W[Np], w2[Np], w3[N];
#pragma unroll
   for (int q = 0; q < Np; q++) W[q] = tw[q];
#pragma unroll
   for (int jf = 0; jf < Np; jf++) w2[jf] = tw[((jp + OFF) * jf) % Np];
#pragma unroll
   for (int kf = 0; kf < N; kf++) w3[kf] = tw[((kq + OFF) * kf) % Np];
   T2* P1 = work[warp];
   // inverse along i (i < 4) of column (jf, kf) = (jp + 4 hi, kq), straight from global
   if (lane < ROW) {
      T2 S[Np];
      const T2* in = in_spectra + c.spec_off + lane;
#pragma unroll
      for (int fi = 0; fi < Np; fi++) S[fi] = in[fi * ROW];
#pragma unroll
      for (int i = 0; i < N; i++) {
         T2 s = Cx<T>::make(T(0), T(0));
#pragma unroll
         for (int fi = 0; fi < Np; fi++) s = Cx<T>::fma(S[fi], W[((i + OFF) * fi) % Np], s);
         P1[i * ROW + lane] = s;
      }
   }
   __syncwarp();
   // inverse along j (j = jp) for i = 2 h + hi, kf = kq
   T2 P2[2];
#pragma unroll
   for (int h = 0; h < 2; h++) {
      const int i = 2 * h + (lane >> 4);
      T2 s = Cx<T>::make(T(0), T(0));
#pragma unroll
      for (int jf = 0; jf < Np; jf++) s = Cx<T>::fma(P1[i * ROW + jf * N + kq], w2[jf], s);
      P2[h] = s;
   }
   // Hermitian half along k -> real grid value at q = lane + 32 h, cropped and scaled
   const T scale = T(1) / (T)(Np * Np * Np);
   T g[2];
#pragma unroll
   for (int h = 0; h < 2; h++) {
      const T2 p0 = shfl_c<T>(P2[h], lane & ~3);
      T s = p0.x;
#pragma unroll
      for (int kf = 1; kf < N; kf++) {
         const T2 pk = shfl_c<T>(P2[h], (lane & ~3) | kf);
         s += T(2) * (pk.x * w3[kf].x - pk.y * w3[kf].y);
      }
      g[h] = s * scale;
   }
   __syncwarp();  // P1 is reused for a
   T2* a = P1;
   const int r = c.r, m = c.m;  // r <= 32
   const T2* pvc = pv + c.pv_off + lane;
   for (int j = 0; j < r; j++) {
      const T2 w0 = pvc[(int64_t)j * N3], w1v = pvc[(int64_t)j * N3 + 32];
      T s = w0.x * g[0] + w1v.x * g[1];
      T d = w0.y * g[0] + w1v.y * g[1];
      s = warp_sum(s);
      d = warp_sum(d);
      if (lane == 0) a[j] = Cx<T>::make(s, d);
   }
   __syncwarp();
   T2* stage = staging + (int64_t)c.level * total_panels;
   for (int i = lane; i < m; i += 32) {
      T s = T(0), d = T(0);
#pragma unroll 4
      for (int j = 0; j < r; j++) {
         const T v = vt[c.vt_off + (int64_t)j * m + i];
         s += v * a[j].x;
         d += v * a[j].y;
      }
      stage[src_panels[c.panel_off + i]] = Cx<T>::make(s, d);
   }
}

constexpr int kNearThreads = 64;  // two leaves per block (B200: 0.1-0.4 % faster solves than four)

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

// One warp per leaf, blockDim.x / 32 leaves per block, each warp with xl_stride
// complex values of shared memory for its gathered panel values:
// y[out(p)] = (D_s xs + D_d xd)[p] + jump(p) xd(p).  The far field is added
// afterwards by far_add_kernel, so this kernel does not wait for it.
template <typename T>
__global__ void __launch_bounds__(kNearThreads) near_kernel(
    const LeafDesc* __restrict__ leaves, int n_leaf, int xl_stride, const int32_t* __restrict__ rows,
    const int32_t* __restrict__ cols, const typename Vec2<T>::type* __restrict__ d,
    const typename Vec2<T>::type* __restrict__ xsd, const int32_t* __restrict__ point_out,
    const int32_t* __restrict__ point_panel, const double* __restrict__ point_jump,
    const int32_t* __restrict__ phi_idx, const double* __restrict__ phi_scale, const double* __restrict__ x,
    double* __restrict__ y, BatchStrides bs, Prefetch pre) {
   using T2 = typename Vec2<T>::type;
   extern __shared__ __align__(16) char smem_raw[];
   const int rhs = blockIdx.x % bs.nrhs, unit = blockIdx.x / bs.nrhs;  // right-hand side fastest
   xsd += rhs * bs.panels;
   x += rhs * bs.n;
   y += rhs * bs.n;
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   const int leaf = unit * (blockDim.x >> 5) + warp;
   if (leaf >= n_leaf) return;
   const LeafDesc L = leaves[leaf];
   if (pre.ahead > 0 && rhs == 0 && lane == 0 && leaf + pre.ahead < n_leaf) {
      const LeafDesc nl = leaves[leaf + pre.ahead];
      prefetch_l2(d, pre.c_bytes, nl.d_off * (int64_t)sizeof(T2), (int64_t)nl.nrows * nl.ncols * (int64_t)sizeof(T2));
   }
   T2* xl = reinterpret_cast<T2*>(smem_raw) + (size_t)warp * xl_stride;
   for (int i = lane; i < L.ncols; i += 32) xl[i] = xsd[cols[L.col_off + i]];
   __syncwarp();
   for (int r0 = 0; r0 < L.nrows; r0 += 32) {
      const int rend = min(32, L.nrows - r0);
      // row sums; lane rr keeps the sum of row r0 + rr
      T mine = T(0);
      int rr = 0;
      // eight rows at a time: eight independent loads in flight per lane, and the eight warp
      // sums in one transposing butterfly (nine shuffles instead of forty): after it lane
      // 4 q holds the sum of row rr + q, which lane rr + q takes for the epilogue
      for (; rr + 7 < rend; rr += 8) {
         const T2* row0 = d + L.d_off + (int64_t)(r0 + rr) * L.ncols;
         T a[8];
#pragma unroll
         for (int q = 0; q < 8; q++) a[q] = T(0);
         for (int c = 2 * lane; c < L.ncols; c += 64) {
#pragma unroll
            for (int q = 0; q < 8; q++) a[q] += NearLoad<T>::dot2(row0 + (int64_t)q * L.ncols, c, xl);
         }
         // each level keeps half of the rows (chosen by one lane bit) and adds the partner's half
         const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
         T k4[4];
#pragma unroll
         for (int q = 0; q < 4; q++) {
            const T give = b4 ? a[q] : a[q + 4], keep = b4 ? a[q + 4] : a[q];
            k4[q] = keep + __shfl_xor_sync(0xffffffffu, give, 16);
         }
         T k2[2];
#pragma unroll
         for (int q = 0; q < 2; q++) {
            const T give = b3 ? k4[q] : k4[q + 2], keep = b3 ? k4[q + 2] : k4[q];
            k2[q] = keep + __shfl_xor_sync(0xffffffffu, give, 8);
         }
         const T give = b2 ? k2[0] : k2[1], keep = b2 ? k2[1] : k2[0];
         T k1 = keep + __shfl_xor_sync(0xffffffffu, give, 4);
         k1 += __shfl_xor_sync(0xffffffffu, k1, 2);
         k1 += __shfl_xor_sync(0xffffffffu, k1, 1);
         const T got = __shfl_sync(0xffffffffu, k1, 4 * ((lane - rr) & 7));
         if (lane >= rr && lane < rr + 8) mine = got;
      }
      for (; rr + 1 < rend; rr += 2) {
         const T2* row0 = d + L.d_off + (int64_t)(r0 + rr) * L.ncols;
         const T2* row1 = row0 + L.ncols;
         T a0 = T(0), a1 = T(0);
         for (int c = 2 * lane; c < L.ncols; c += 64) {
            a0 += NearLoad<T>::dot2(row0, c, xl);
            a1 += NearLoad<T>::dot2(row1, c, xl);
         }
         a0 = warp_sum(a0);
         a1 = warp_sum(a1);
         if (lane == rr) mine = a0;
         if (lane == rr + 1) mine = a1;
      }
      if (rr < rend) {
         const T2* row0 = d + L.d_off + (int64_t)(r0 + rr) * L.ncols;
         T a0 = T(0);
         for (int c = 2 * lane; c < L.ncols; c += 64) a0 += NearLoad<T>::dot2(row0, c, xl);
         a0 = warp_sum(a0);
         if (lane == rr) mine = a0;
      }
      if (lane < rend) {
         const int pnt = rows[L.row_off + r0 + lane];
         double v = (double)mine;
         const int k = point_panel[pnt];
         if (k >= 0) v += point_jump[pnt] * (phi_scale[k] * x[phi_idx[k]]);
         y[point_out[pnt]] = v;
      }
   }
}

// y[out(p)] += sum over levels of staging[level][p], for every leaf row p (each
// output row has exactly one leaf row, so every element has one writer).
template <typename T>
__global__ void far_add_kernel(int64_t nrows, const int32_t* __restrict__ rows, const T* __restrict__ staging,
                               int stage_levels, int64_t total_points, const int32_t* __restrict__ point_out,
                               double* __restrict__ y, BatchStrides bs) {
   staging += blockIdx.y * bs.staging;  // right-hand side blockIdx.y of a batch
   y += blockIdx.y * bs.n;
   for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nrows; i += (int64_t)gridDim.x * blockDim.x) {
      const int pnt = rows[i];
      double v = 0.0;
      for (int l = 0; l < stage_levels; l++) v += (double)staging[(int64_t)l * total_points + pnt];
      y[point_out[pnt]] += v;
   }
}

// ------------------------------------------------------------------ host side

// FP64 uploads go straight from the layout's arrays; FP32 ones through a converted copy
template <typename T, typename Vec>
static void upload_cast(DevBuf<T>& dst, const Vec& src) {
   if constexpr (std::is_same<T, double>::value) {
      dst.upload(src.data(), src.size());
      return;
   }
   std::vector<T, FillLater<T>> tmp(src.size());
   const int64_t n = (int64_t)tmp.size();
#pragma omp parallel for schedule(static)
   for (int64_t i = 0; i < n; i++) tmp[i] = (T)src[i];
   dst.upload(tmp.data(), tmp.size());
}

template <typename T, typename Vec>
static void upload_pairs(DevBuf<typename Vec2<T>::type>& dst, const Vec& src) {
   using T2 = typename Vec2<T>::type;
   if constexpr (std::is_same<T, double>::value) {  // {re, im} pairs are double2 in memory
      dst.upload(reinterpret_cast<const T2*>(src.data()), src.size() / 2);
      return;
   }
   std::vector<T2, FillLater<T2>> tmp(src.size() / 2);
   const int64_t np = (int64_t)tmp.size();
#pragma omp parallel for schedule(static)
   for (int64_t i = 0; i < np; i++) {
      tmp[i].x = (T)src[2 * i];
      tmp[i].y = (T)src[2 * i + 1];
   }
   dst.upload(tmp.data(), tmp.size());
}

// The dynamic shared-memory limit of a kernel is one device-wide setting shared by
// every surface: raise it to what this surface needs, never lower it (a smaller
// surface set up later must not break the launches of a larger one).
static std::mutex g_smem_limit_mutex;
template <typename K>
static void raise_smem_limit(K* kernel, int bytes) {
   std::lock_guard<std::mutex> lock(g_smem_limit_mutex);
   cudaFuncAttributes a;
   FFTSVD_CUDA(cudaFuncGetAttributes(&a, kernel));
   if (a.maxDynamicSharedSizeBytes < bytes)
      FFTSVD_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
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
   n_rows_ = (int64_t)L.leaf_rows.size();
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
   upload_pairs<T>(t_, L.t_pairs);
   fwd_.upload(L.fwd);
   adj_.upload(L.adj);
   // transposed operator: gathered points, per-panel sums, per-level far-field rows, and
   // for each panel the point whose jump term it takes (a point and its panel share an index)
   zt_.alloc(std::max<int64_t>(L.total_points, 1));
   ut_.alloc(L.total_panels);
   staget_.alloc(std::max<int64_t>((int64_t)L.stage_levels * L.total_panels, 1));
   staget_.zero();  // rows no source cube of a level writes stay zero
   {
      std::vector<double> pj(L.total_panels, 0.0);
      std::vector<int32_t> pp(L.total_panels, -1);
      for (int64_t q = 0; q < L.total_points; q++)
         if (L.point_panel[q] >= 0) {
            FFTSVD_REQUIRE(pp[L.point_panel[q]] < 0, "two jump points on one panel");
            pp[L.point_panel[q]] = (int32_t)q;
            pj[L.point_panel[q]] = L.point_jump[q];
         }
      panel_jump_.upload(pj);
      panel_point_.upload(pp);
   }
   translated_.alloc(std::max<int64_t>(L.translated_elems, 1));
   spectra_.alloc(std::max<int64_t>(L.spectra_elems, 1));
   spectra_.zero();      // row padding is read by the translation and must stay zero
   translated_.zero();
   staging_.alloc(std::max<int64_t>((int64_t)L.stage_levels * L.total_points, 1));
   staging_.zero();
   // entries of the zero slot and staging rows nobody writes must stay zero
   src_groups_ = L.src_groups;
   dst_groups_ = L.dst_groups;
   src_smem_ = 0;
   dst_smem_ = 0;
   for (const LaunchGroup& g : src_groups_) src_smem_ = std::max(src_smem_, (int)(g.smem_elems * sizeof(T) + 128));
   for (const LaunchGroup& g : dst_groups_) dst_smem_ = std::max(dst_smem_, (int)(g.smem_elems * sizeof(T) + 128));
   src_smem_t_ = dst_smem_t_ = 0;
   for (const SrcDesc& c : L.src) src_smem_t_ = std::max(src_smem_t_, far_forward_t_smem<T>(c.n, c.r));
   for (const DstDesc& c : L.dst) dst_smem_t_ = std::max(dst_smem_t_, far_backward_t_smem<T>(c.n, c.r));
   int maxcols = 2;
   for (const auto& l : L.leaves) maxcols = std::max(maxcols, l.ncols);
   int dev = 0, optin = 0;
   FFTSVD_CUDA(cudaGetDevice(&dev));
   FFTSVD_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
   FFTSVD_CUDA(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, dev));
   sm_count_ = std::max(sm_count_, 1);
   // one warp per leaf; as many leaves per block (up to four) as the gathered columns allow
   near_stride_ = maxcols;
   near_warps_ = (int)std::max<size_t>(1, std::min<size_t>(kNearThreads / 32, (size_t)optin / (maxcols * sizeof(T2))));
   leaf_smem_max_ = (int)(near_warps_ * maxcols * sizeof(T2));
   if (src_smem_ > optin || dst_smem_ > optin || leaf_smem_max_ > optin || src_smem_t_ > optin ||
       dst_smem_t_ > optin)
      throw Error(FFTSVD_ERR_UNSUPPORTED, "operator block needs more shared memory than the device offers");
   raise_translate_smem(optin);
   // FFTSVD_B200_WARP_MIN_CUBES overrides the cube count from which small grids run
   // one cube per warp (tests set 0 to cover those kernels on small surfaces)
   warp_min_cubes_ = kWarpMinCubes;
   if (const char* e = std::getenv("FFTSVD_B200_WARP_MIN_CUBES")) warp_min_cubes_ = std::max(0, std::atoi(e));
   spectra_elems_ = std::max<int64_t>(L.spectra_elems, 1);
   translated_elems_ = std::max<int64_t>(L.translated_elems, 1);
   batch_capacity_ = 0;
   raise_smem_limit(far_forward_kernel<T, 1>, src_smem_);
   raise_smem_limit(far_backward_kernel<T, 1>, dst_smem_);
   smem_optin_ = optin;
   int src_b = 1, dst_b = 1;
   for (const LaunchGroup& g : src_groups_) {
      const int b = far_batch_smem(g, far_rb<T>(), sizeof(T));
      if (b <= optin) src_b = std::max(src_b, b);
   }
   for (const LaunchGroup& g : dst_groups_) {
      const int b = far_batch_smem(g, far_rb<T>(), sizeof(T));
      if (b <= optin) dst_b = std::max(dst_b, b);
   }
   raise_smem_limit(far_forward_kernel<T, far_rb<T>()>, src_b);
   raise_smem_limit(far_backward_kernel<T, far_rb<T>()>, dst_b);
   raise_smem_limit(near_kernel<T>, leaf_smem_max_);
   near_np_max_ = 0;
   if (std::is_same<T, float>::value) {
      int rmax = 8;
      for (const auto& l : L.leaves) rmax = std::max(rmax, (l.nrows + 7) & ~7);
      if (rmax <= 256 && near_tc_smem(rmax) <= optin) {
         near_np_max_ = rmax;
         prepare_near_tc(rmax);
         tc_status_.alloc(1);
         tc_status_.zero();
      }
   }
   {
      int nb = 0;
      FFTSVD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, far_forward_n4_kernel<T>, kWarpThreads, 0));
      fwd_n4_wave_ = (int64_t)nb * sm_count_ * kWarpCubes;
      FFTSVD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, far_backward_n4_kernel<T>, kWarpThreads, 0));
      bwd_n4_wave_ = (int64_t)nb * sm_count_ * kWarpCubes;
      FFTSVD_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, near_kernel<T>, 32 * near_warps_, leaf_smem_max_));
      near_wave_ = (int64_t)nb * sm_count_ * near_warps_;
   }
   raise_smem_limit(far_forward_t_kernel<T>, std::max(src_smem_t_, 1));
   raise_smem_limit(far_backward_t_kernel<T>, std::max(dst_smem_t_, 1));
   build_chains();
   FFTSVD_CUDA(cudaDeviceSynchronize());
}

template <typename T>
Prefetch DeviceOperator<T>::prefetch(int64_t wave, int nrhs, int64_t a_bytes, int64_t b_bytes, int64_t c_bytes) const {
   Prefetch p;
   p.ahead = wave / std::max(nrhs, 1);  // the blocks of one unit for all right-hand sides are adjacent
   p.a_bytes = a_bytes;
   p.b_bytes = b_bytes;
   p.c_bytes = c_bytes;
   return p;
}

template <typename T>
void DeviceOperator<T>::enable_timing(bool on) {
   if (on && !ev_[0])
      for (auto& e : ev_) FFTSVD_CUDA(cudaEventCreate(&e));
   timing_ = on;
}

// Raise the translation kernels' dynamic shared-memory limits to what the current tiles need.
template <typename T>
void DeviceOperator<T>::raise_translate_smem(int optin) {
   int tile_smem = 0, tile_smem_b = 0;
   for (const TileGroup& g : fwd_.groups) {
      tile_smem = std::max(tile_smem, translate_smem(g, false));
      tile_smem_b = std::max(tile_smem_b, translate_smem(g, true));
   }
   for (const TileGroup& g : adj_.groups) tile_smem = std::max(tile_smem, translate_smem(g, false));
   if (tile_smem > optin || tile_smem_b > optin)
      throw Error(FFTSVD_ERR_UNSUPPORTED, "translation tile needs more shared memory than the device offers");
   if (tile_smem > 0) {
      raise_smem_limit(translate_kernel<T, false>, tile_smem);
      raise_smem_limit(translate_kernel<T, true>, tile_smem_b);
   }
}

template <typename T>
void DeviceOperator<T>::set_tiles(const TileSet& fwd, const TileSet& adj) {
   FFTSVD_REQUIRE(fwd.tile_groups.size() == fwd_.groups.size() && adj.tile_groups.size() == adj_.groups.size(),
                  "tiles of another operator");
   for (size_t i = 0; i < fwd.tile_groups.size(); i++)
      FFTSVD_REQUIRE(fwd.tile_groups[i].pg == fwd_.groups[i].pg, "tiles of another operator");
   int dev = 0, optin = 0;
   FFTSVD_CUDA(cudaGetDevice(&dev));
   FFTSVD_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
   FFTSVD_CUDA(cudaDeviceSynchronize());  // no launch may still read the old tiles
   fwd_.upload(fwd);
   adj_.upload(adj);
   raise_translate_smem(optin);
}

template <typename T>
int DeviceOperator<T>::translate_smem(const TileGroup& g, bool batch) const {
   // one chunk row per slot and per halo source, entries, groups, member offsets and
   // deltas, halo offsets; each carve aligned to 16 bytes
   // batch: two buffers of table and halo rows
   const size_t slot_row = batch ? 16 : kTileRowBytes, nbuf = batch ? 2 : 1;
   return (int)(nbuf * (343 * slot_row + (size_t)g.max_src * kTileRowBytes) + (size_t)g.max_entries * sizeof(uint32_t) +
                (size_t)g.max_groups * sizeof(int4) + (size_t)g.max_members * (sizeof(int64_t) + sizeof(int)) +
                (size_t)g.max_src * sizeof(int64_t) + 128);
}

template <typename T>
void DeviceOperator<T>::stage_ms(float* ms) const {
   for (int k = 0; k < kNumKernels; k++) ms[k] = 0.f;
   if (!ev_[0]) return;
   FFTSVD_CUDA(cudaEventSynchronize(ev_[kNumKernels]));
   for (int k = 0; k < kNumKernels; k++) FFTSVD_CUDA(cudaEventElapsedTime(&ms[k], ev_[k], ev_[k + 1]));
}

template <typename T>
bool DeviceOperator<T>::warp_path(const LaunchGroup& g) const {
   return g.n >= kWarpMinN && g.n <= kWarpMaxN && g.max_rank >= 1 && g.max_rank <= kWarpMaxRank &&
          g.count >= warp_min_cubes_ && g.units <= (int64_t)kWarpMaxMeanUnits * g.count;
}

template <typename T>
void DeviceOperator<T>::launch_forward(const LaunchGroup& g, const Bufs& b, cudaStream_t stream) {
   if (warp_path(g)) {
      const dim3 grid((g.count + kWarpCubes - 1) / kWarpCubes * b.nrhs);
      const SrcDesc* c = src_.get() + g.begin;
      if (g.n == 3)
         far_forward_warp_kernel<T, 3><<<grid, kWarpThreads, 0, stream>>>(c, g.count, src_panels_.get(), b.xsd,
                                                                         vt_.get(), pv_.get(), b.spectra, b.bs);
      else if (g.n == 4)
         far_forward_n4_kernel<T><<<grid, kWarpThreads, 0, stream>>>(c, g.count, src_panels_.get(), b.xsd, vt_.get(),
                                                                     pv_.get(), b.spectra, b.bs,
                                                                     prefetch(fwd_n4_wave_, b.nrhs, vt_.bytes(),
                                                                              pv_.bytes(), 0));
      else
         far_forward_warp_kernel<T, 5><<<grid, kWarpThreads, 0, stream>>>(c, g.count, src_panels_.get(), b.xsd,
                                                                         vt_.get(), pv_.get(), b.spectra, b.bs);
   } else {
      constexpr int RB = far_rb<T>();
      const int smem_b = far_batch_smem(g, RB, sizeof(T));
      if (b.nrhs % RB == 0 && smem_b <= smem_optin_) {  // RB right-hand sides per block
         far_forward_kernel<T, RB><<<g.count * (b.nrhs / RB), far_threads(g), smem_b, stream>>>(
             src_.get() + g.begin, src_panels_.get(), b.xsd, vt_.get(), pv_.get(), b.spectra, b.bs);
      } else {
         const int smem = (int)(g.smem_elems * sizeof(T) + 128);
         far_forward_kernel<T, 1><<<g.count * b.nrhs, far_threads(g), smem, stream>>>(
             src_.get() + g.begin, src_panels_.get(), b.xsd, vt_.get(), pv_.get(), b.spectra, b.bs);
      }
   }
   FFTSVD_CHECK_LAUNCH();
}

template <typename T>
void DeviceOperator<T>::DevTiles::upload(const TileSet& S) {
   // shared-memory bytes one single-vector translation moves: per tile and frequency
   // chunk, the staged rows (343 table slots and the halo spectra) are written once, and
   // each (group, entry) reads its source row once and one table row per member; rows are
   // kTileRowBytes wide
   smem_bytes = 0.0;
   for (const TileDesc& t : S.tiles) {
      const double chunks = (double)t.pg / (kTileRowBytes / (double)sizeof(typename Vec2<T>::type));
      double reads = 0.0;
      for (int gi = 0; gi < t.ngroups; gi++) {
         const int4 g = S.tile_grp[t.grp_off + gi];
         reads += (double)g.y * (1.0 + g.w);
      }
      smem_bytes += chunks * kTileRowBytes * ((343.0 + t.nsrc) + reads);
   }
   tiles.upload(S.tiles);
   src.upload(S.tile_src);
   dst.upload(S.tile_dst);
   delta.upload(S.tile_delta);
   grp.upload(S.tile_grp);
   entries.upload(S.tile_entries);
   groups = S.tile_groups;
}

template <typename T>
void DeviceOperator<T>::launch_translate_tiles(const DevTiles& tl, const TileGroup& g, const T2* in, T2* out,
                                               int nrhs, const BatchStrides& bs, cudaStream_t stream) {
   // split each tile's frequency chunks over blocks of cpb chunks each: the split with
   // the fewest chunk times over all waves of resident blocks (two per SM), the
   // smallest such cpb (more blocks fill the device better at the coarse levels)
   const bool batch = nrhs > 1;
   const int groups = batch ? nrhs / kBatchGroup : 1;
   const int nchunks = g.pg / (batch ? 16 / (int)sizeof(T2) : kTileRowBytes / (int)sizeof(T2));
   const int64_t slots = 2LL * sm_count_;
   // (batch: at least four chunks per block, so that the double buffer overlaps copies with
   // arithmetic and neighbouring units of a spectrum row share their L2 sectors)
   int cpb = 1;
   int64_t best = -1;
   for (int c = batch ? std::min(nchunks, 4) : 1; c <= nchunks; c++) {
      const int64_t blocks = (int64_t)g.count * ((nchunks + c - 1) / c) * groups;
      const int64_t cost = (blocks + slots - 1) / slots * c;
      if (best < 0 || cost < best) best = cost, cpb = c;
   }
   const dim3 grid(g.count, (nchunks + cpb - 1) / cpb, groups);
   const int threads = std::min(kTranslateThreads, 32 * g.max_groups);  // up to one warp per member group
   if (batch)
      translate_kernel<T, true><<<grid, threads, translate_smem(g, true), stream>>>(
          tl.tiles.get() + g.begin, tl.src.get(), tl.dst.get(), tl.delta.get(), tl.grp.get(), tl.entries.get(),
          t_.get(), in, out, cpb, bs);
   else
      translate_kernel<T, false><<<grid, threads, translate_smem(g, false), stream>>>(
          tl.tiles.get() + g.begin, tl.src.get(), tl.dst.get(), tl.delta.get(), tl.grp.get(), tl.entries.get(),
          t_.get(), in, out, cpb, bs);
   FFTSVD_CHECK_LAUNCH();
}

template <typename T>
void DeviceOperator<T>::launch_translate(const TileGroup& g, const Bufs& b, cudaStream_t stream) {
   launch_translate_tiles(fwd_, g, b.spectra, b.translated, b.nrhs, b.bs, stream);
}

template <typename T>
void DeviceOperator<T>::apply_transpose(const double* x, double* y, cudaStream_t stream) {
   const int64_t np = total_panels_ - 1;  // the zero slot is no panel
   FFTSVD_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * num_unknowns_, stream));
   FFTSVD_CUDA(cudaMemsetAsync(ut_.get(), 0, sizeof(double2) * total_panels_, stream));
   const int ew = (int)std::max<int64_t>(1, std::min<int64_t>((std::max(total_points_, np) + 255) / 256, 148 * 16));
   if (total_points_ > 0) {
      gather_points_kernel<T><<<ew, 256, 0, stream>>>(total_points_, point_out_.get(), x, zt_.get());
      FFTSVD_CHECK_LAUNCH();
   }
   // far field, backwards: destinations -> translated slots -> (transposed tiles) -> source
   // spectra, one chain per grid size on the chains' streams (as the forward operator), the
   // near-field column sums beside them; sources that no destination reaches must read zero
   FFTSVD_CUDA(cudaMemsetAsync(spectra_.get(), 0, sizeof(T2) * spectra_elems_, stream));
   FFTSVD_CUDA(cudaEventRecord(fork_, stream));
   if (n_leaf_ > 0) {
      FFTSVD_CUDA(cudaStreamWaitEvent(near_stream_, fork_, 0));
      near_t_kernel<T><<<(n_leaf_ + kWarpCubes - 1) / kWarpCubes, kWarpThreads, 0, near_stream_>>>(
          leaves_.get(), n_leaf_, leaf_rows_.get(), leaf_cols_.get(), d_.get(), zt_.get(), ut_.get(), (int32_t)np);
      FFTSVD_CHECK_LAUNCH();
      FFTSVD_CUDA(cudaEventRecord(near_done_, near_stream_));
   }
   for (const Chain& ch : chains_) {
      FFTSVD_CUDA(cudaStreamWaitEvent(ch.stream, fork_, 0));
      for (int i : ch.dst) {
         const LaunchGroup& g = dst_groups_[i];
         if (warp_path(g) && g.n == 4)
            far_backward_t_n4_kernel<T><<<(g.count + kWarpCubes - 1) / kWarpCubes, kWarpThreads, 0, ch.stream>>>(
                dst_.get() + g.begin, g.count, dst_points_.get(), zt_.get(), uti_.get(), u_.get(), translated_.get());
         else
            far_backward_t_kernel<T><<<g.count, far_threads(g.n), dst_smem_t_, ch.stream>>>(
                dst_.get() + g.begin, dst_points_.get(), zt_.get(), uti_.get(), u_.get(), translated_.get());
         FFTSVD_CHECK_LAUNCH();
      }
      const int pgp = ((2 * ch.n - 1) * (2 * ch.n - 1) * ch.n + 15) & ~15;
      for (const TileGroup& g : adj_.groups)
         if (g.pg == pgp) launch_translate_tiles(adj_, g, translated_.get(), spectra_.get(), 1, BatchStrides(), ch.stream);
      for (int i : ch.src) {
         const LaunchGroup& g = src_groups_[i];
         if (warp_path(g) && g.n == 4)
            far_forward_t_n4_kernel<T><<<(g.count + kWarpCubes - 1) / kWarpCubes, kWarpThreads, 0, ch.stream>>>(
                src_.get() + g.begin, g.count, src_panels_.get(), spectra_.get(), vt_.get(), pv_.get(), staget_.get(),
                total_panels_);
         else
            far_forward_t_kernel<T><<<g.count, far_threads(g.n), src_smem_t_, ch.stream>>>(
                src_.get() + g.begin, src_panels_.get(), spectra_.get(), vt_.get(), pv_.get(), staget_.get(),
                total_panels_);
         FFTSVD_CHECK_LAUNCH();
      }
      FFTSVD_CUDA(cudaEventRecord(ch.done, ch.stream));
   }
   for (const Chain& ch : chains_) FFTSVD_CUDA(cudaStreamWaitEvent(stream, ch.done, 0));
   if (n_leaf_ > 0) FFTSVD_CUDA(cudaStreamWaitEvent(stream, near_done_, 0));
   if (np > 0) {
      scatter_panels_kernel<T><<<ew, 256, 0, stream>>>(np, ut_.get(), staget_.get(), stage_levels_, total_panels_,
                                                       panel_jump_.get(), panel_point_.get(), zt_.get(),
                                                       join_phi_idx_.get(), join_phi_scale_.get(),
                                                       join_dphi_idx_.get(), join_dphi_scale_.get(), y);
      FFTSVD_CHECK_LAUNCH();
   }
}

template <typename T>
void DeviceOperator<T>::launch_backward(const LaunchGroup& g, const Bufs& b, cudaStream_t stream) {
   if (warp_path(g)) {
      const dim3 grid((g.count + kWarpCubes - 1) / kWarpCubes * b.nrhs);
      const DstDesc* c = dst_.get() + g.begin;
      if (g.n == 3)
         far_backward_warp_kernel<T, 3><<<grid, kWarpThreads, 0, stream>>>(
             c, g.count, dst_points_.get(), b.translated, uti_.get(), u_.get(), b.staging, total_points_, b.bs);
      else if (g.n == 4)
         far_backward_n4_kernel<T><<<grid, kWarpThreads, 0, stream>>>(
             c, g.count, dst_points_.get(), b.translated, uti_.get(), u_.get(), b.staging, total_points_, b.bs,
             prefetch(bwd_n4_wave_, b.nrhs, uti_.bytes(), u_.bytes(), 0));
      else
         far_backward_warp_kernel<T, 5><<<grid, kWarpThreads, 0, stream>>>(
             c, g.count, dst_points_.get(), b.translated, uti_.get(), u_.get(), b.staging, total_points_, b.bs);
   } else {
      constexpr int RB = far_rb<T>();
      const int smem_b = far_batch_smem(g, RB, sizeof(T));
      if (b.nrhs % RB == 0 && smem_b <= smem_optin_) {  // RB right-hand sides per block
         far_backward_kernel<T, RB><<<g.count * (b.nrhs / RB), far_threads(g), smem_b, stream>>>(
             dst_.get() + g.begin, dst_points_.get(), b.translated, uti_.get(), u_.get(), b.staging, total_points_,
             b.bs);
      } else {
         const int smem = (int)(g.smem_elems * sizeof(T) + 128);
         far_backward_kernel<T, 1><<<g.count * b.nrhs, far_threads(g), smem, stream>>>(
             dst_.get() + g.begin, dst_points_.get(), b.translated, uti_.get(), u_.get(), b.staging, total_points_,
             b.bs);
      }
   }
   FFTSVD_CHECK_LAUNCH();
}

template <typename T>
void DeviceOperator<T>::launch_chain(const Chain& ch, const Bufs& b, cudaStream_t stream) {
   for (int i : ch.src) launch_forward(src_groups_[i], b, stream);
   for (int i : ch.tile) launch_translate(fwd_.groups[i], b, stream);
   for (int i : ch.dst) launch_backward(dst_groups_[i], b, stream);
}

template <typename T>
void DeviceOperator<T>::apply(const double* x, double* y, cudaStream_t stream) {
   Bufs b;
   b.xsd = xsd_.get();
   b.spectra = spectra_.get();
   b.translated = translated_.get();
   b.staging = staging_.get();
   b.nrhs = 1;
   apply_bufs(x, y, b, stream);
}

template <typename T>
void DeviceOperator<T>::apply_batch(const double* x, double* y, int nrhs, cudaStream_t stream) {
   FFTSVD_REQUIRE(nrhs > 0 && nrhs % kBatchGroup == 0 && nrhs <= kMaxBatch, "batch size");
   if (nrhs > batch_capacity_) {
      // planar buffers, one copy of every intermediate per right-hand side; padding
      // entries, the zero slot and unwritten staging rows stay zero
      xsd_b_.alloc((int64_t)nrhs * total_panels_);
      xsd_b_.zero();
      spectra_b_.alloc((int64_t)nrhs * spectra_elems_);
      spectra_b_.zero();
      translated_b_.alloc((int64_t)nrhs * translated_elems_);
      translated_b_.zero();
      staging_b_.alloc(std::max<int64_t>((int64_t)nrhs * stage_levels_ * total_points_, 1));
      staging_b_.zero();
      FFTSVD_CUDA(cudaDeviceSynchronize());
      batch_capacity_ = nrhs;
   }
   Bufs b;
   b.xsd = xsd_b_.get();
   b.spectra = spectra_b_.get();
   b.translated = translated_b_.get();
   b.staging = staging_b_.get();
   b.nrhs = nrhs;
   b.bs.n = num_unknowns_;
   b.bs.panels = total_panels_;
   b.bs.spectra = spectra_elems_;
   b.bs.translated = translated_elems_;
   b.bs.staging = (int64_t)stage_levels_ * total_points_;
   b.bs.nrhs = nrhs;
   apply_bufs(x, y, b, stream);
}

template <typename T>
size_t DeviceOperator<T>::batch_bytes_per_rhs() const {
   return sizeof(T2) * (size_t)(total_panels_ + spectra_elems_ + translated_elems_) +
          sizeof(T) * (size_t)stage_levels_ * total_points_;
}

template <typename T>
void DeviceOperator<T>::apply_bufs(const double* x, double* y, const Bufs& b, cudaStream_t stream) {
   if (timing_) FFTSVD_CUDA(cudaEventRecord(ev_[0], stream));
   if (!full_cover_) FFTSVD_CUDA(cudaMemsetAsync(y, 0, sizeof(double) * num_unknowns_ * b.nrhs, stream));
   {
      const int64_t total = total_panels_ - 1;  // the zero slot is never written
      int blocks = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
      if (blocks < 1) blocks = 1;
      join_kernel<T><<<dim3(blocks, b.nrhs), 256, 0, stream>>>(total, join_phi_idx_.get(), join_phi_scale_.get(),
                                                              join_dphi_idx_.get(), join_dphi_scale_.get(), x, b.xsd,
                                                              b.bs);
      FFTSVD_CHECK_LAUNCH();
   }
   if (timing_) {
      // stage by stage on one stream, so that each stage can be timed
      FFTSVD_CUDA(cudaEventRecord(ev_[1], stream));
      for (const LaunchGroup& g : src_groups_) launch_forward(g, b, stream);
      FFTSVD_CUDA(cudaEventRecord(ev_[2], stream));
      for (const TileGroup& g : fwd_.groups) launch_translate(g, b, stream);
      FFTSVD_CUDA(cudaEventRecord(ev_[3], stream));
      for (const LaunchGroup& g : dst_groups_) launch_backward(g, b, stream);
      FFTSVD_CUDA(cudaEventRecord(ev_[4], stream));
      launch_near(x, y, b, stream);
   } else {
      // the near field and the far-field chains of each grid size (forward -> translate
      // -> backward) only share the joined input: all but the largest chain run on their
      // own streams, forked after the join and joined back before the far field is added
      // (the longest chain on a high-priority stream: it is the critical path)
      FFTSVD_CUDA(cudaEventRecord(fork_, stream));
      for (size_t c = 0; c < chains_.size(); c++) {
         FFTSVD_CUDA(cudaStreamWaitEvent(chains_[c].stream, fork_, 0));
         launch_chain(chains_[c], b, chains_[c].stream);
         FFTSVD_CUDA(cudaEventRecord(chains_[c].done, chains_[c].stream));
      }
      FFTSVD_CUDA(cudaStreamWaitEvent(near_stream_, fork_, 0));
      launch_near(x, y, b, near_stream_);
      FFTSVD_CUDA(cudaEventRecord(near_done_, near_stream_));
      for (size_t c = 0; c < chains_.size(); c++) FFTSVD_CUDA(cudaStreamWaitEvent(stream, chains_[c].done, 0));
      FFTSVD_CUDA(cudaStreamWaitEvent(stream, near_done_, 0));
   }
   if (n_rows_ > 0 && stage_levels_ > 0) {
      const int blocks = (int)std::min<int64_t>((n_rows_ + 255) / 256, 148 * 8);
      far_add_kernel<T><<<dim3(blocks, b.nrhs), 256, 0, stream>>>(n_rows_, leaf_rows_.get(), b.staging, stage_levels_,
                                                                 total_points_, point_out_.get(), y, b.bs);
      FFTSVD_CHECK_LAUNCH();
   }
   if (timing_) FFTSVD_CUDA(cudaEventRecord(ev_[5], stream));
}

template <typename T>
double DeviceOperator<T>::translate_smem_bytes() const {
   return fwd_.smem_bytes;
}

template <typename T>
int DeviceOperator<T>::tensor_status(bool reset) {
   if (!tc_status_.get()) return 0;
   int v = 0;
   FFTSVD_CUDA(cudaMemcpy(&v, tc_status_.get(), sizeof(int), cudaMemcpyDeviceToHost));
   if (reset && v) tc_status_.zero();
   return v;
}

template <typename T>
void DeviceOperator<T>::launch_near(const double* x, double* y, const Bufs& b, cudaStream_t stream) {
   if (n_leaf_ == 0) return;
   if constexpr (std::is_same<T, float>::value) {
      if (tensor_near_ && b.nrhs >= kBatchGroup && near_np_max_ > 0) {
         const int64_t ld = (b.nrhs + 31) / 32 * 32;
         if (xsd_t_.size() < (size_t)(total_panels_ * ld)) xsd_t_.alloc((size_t)(total_panels_ * ld));
         launch_near_tc(leaves_.get(), n_leaf_, leaf_rows_.get(), leaf_cols_.get(), d_.get(), b.xsd, b.bs.panels,
                        (int)total_panels_, xsd_t_.get(), ld, point_out_.get(), point_panel_.get(), point_jump_.get(),
                        join_phi_idx_.get(), join_phi_scale_.get(), x, y, b.nrhs, b.bs.n, near_np_max_,
                        tc_status_.get(), stream);
         return;
      }
   }
   near_kernel<T><<<(n_leaf_ + near_warps_ - 1) / near_warps_ * b.nrhs, 32 * near_warps_, leaf_smem_max_,
                    stream>>>(leaves_.get(), n_leaf_, near_stride_, leaf_rows_.get(), leaf_cols_.get(), d_.get(), b.xsd,
                              point_out_.get(), point_panel_.get(), point_jump_.get(), join_phi_idx_.get(),
                              join_phi_scale_.get(), x, y, b.bs, prefetch(near_wave_, b.nrhs, 0, 0, d_.bytes()));
   FFTSVD_CHECK_LAUNCH();
}

template <typename T>
void DeviceOperator<T>::build_chains() {
   release_chains();
   std::map<int, Chain> by_n;
   for (int i = 0; i < (int)src_groups_.size(); i++) by_n[src_groups_[i].n].src.push_back(i);
   for (int i = 0; i < (int)dst_groups_.size(); i++) by_n[dst_groups_[i].n].dst.push_back(i);
   for (auto& kv : by_n) {
      const int n = kv.first, pgp = ((2 * n - 1) * (2 * n - 1) * n + 15) & ~15;
      kv.second.n = n;
      for (int i = 0; i < (int)fwd_.groups.size(); i++)
         if (fwd_.groups[i].pg == pgp) kv.second.tile.push_back(i);
      // destinations and their interactions: a measure of the chain's length
      for (int i : kv.second.dst) kv.second.work += (double)dst_groups_[i].count * pgp;
   }
   for (auto& kv : by_n) chains_.push_back(kv.second);
   std::stable_sort(chains_.begin(), chains_.end(), [](const Chain& a, const Chain& b) { return a.work > b.work; });
   int least = 0, greatest = 0;
   FFTSVD_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
   FFTSVD_CUDA(cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming));
   FFTSVD_CUDA(cudaStreamCreateWithPriority(&near_stream_, cudaStreamNonBlocking, least));
   FFTSVD_CUDA(cudaEventCreateWithFlags(&near_done_, cudaEventDisableTiming));
   for (size_t c = 0; c < chains_.size(); c++) {
      FFTSVD_CUDA(cudaStreamCreateWithPriority(&chains_[c].stream, cudaStreamNonBlocking, c == 0 ? greatest : least));
      FFTSVD_CUDA(cudaEventCreateWithFlags(&chains_[c].done, cudaEventDisableTiming));
   }
}

template <typename T>
void DeviceOperator<T>::release_chains() {
   for (Chain& c : chains_) {
      if (c.stream) cudaStreamDestroy(c.stream);
      if (c.done) cudaEventDestroy(c.done);
   }
   chains_.clear();
   if (fork_) cudaEventDestroy(fork_);
   if (near_stream_) cudaStreamDestroy(near_stream_);
   if (near_done_) cudaEventDestroy(near_done_);
   fork_ = nullptr;
   near_stream_ = nullptr;
   near_done_ = nullptr;
}

template <typename T>
DeviceOperator<T>::~DeviceOperator() {
   release_chains();
   for (auto& e : ev_)
      if (e) cudaEventDestroy(e);
}

template <typename T>
size_t DeviceOperator<T>::device_bytes() const {
   return join_phi_idx_.bytes() + join_dphi_idx_.bytes() + join_phi_scale_.bytes() + join_dphi_scale_.bytes() +
          xsd_.bytes() + point_out_.bytes() + point_panel_.bytes() + point_jump_.bytes() + leaves_.bytes() +
          leaf_rows_.bytes() + leaf_cols_.bytes() + d_.bytes() + src_.bytes() + src_panels_.bytes() +
          vt_.bytes() + pv_.bytes() + dst_.bytes() + dst_points_.bytes() + uti_.bytes() + u_.bytes() +
          t_.bytes() + spectra_.bytes() + staging_.bytes() + fwd_.tiles.bytes() + fwd_.src.bytes() +
          fwd_.dst.bytes() + fwd_.delta.bytes() + fwd_.grp.bytes() + fwd_.entries.bytes() + translated_.bytes() + adj_.tiles.bytes() +
          adj_.src.bytes() + adj_.dst.bytes() + adj_.delta.bytes() + adj_.grp.bytes() + adj_.entries.bytes() + zt_.bytes() +
          ut_.bytes() + staget_.bytes();
}

template class DeviceOperator<float>;
template class DeviceOperator<double>;

}  // namespace fftsvd
