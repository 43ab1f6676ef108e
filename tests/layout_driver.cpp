// Test driver for the host side of surface creation: reads a problem (flat triangles and
// charges), runs the host setup with its panel integrals in batches on the host and builds
// the operator layout the device upload consumes, then prints a hash of every array of the
// flat trees and of the layout (one line each).  Run under different OMP_NUM_THREADS the
// output must not change: every parallel step writes at offsets fixed before it runs.
//
//   layout_driver problem.bin
//
// problem.bin: int64 num_panels, int64 num_charges, double eps_in, eps_out, kappa, then the
// 9 num_panels vertex coordinates, 3 num_charges charge positions and the charges.
#include <cstdint>
#include <cstdio>
#include <vector>

#include "../fftsvd_b200/csrc/operator.h"
#include "../fftsvd_b200/csrc/setup.h"

static uint64_t fnv(const void* p, size_t n) {
   const unsigned char* b = static_cast<const unsigned char*>(p);
   uint64_t h = 1469598103934665603ull;
   for (size_t i = 0; i < n; i++) {
      h ^= b[i];
      h *= 1099511628211ull;
   }
   return h;
}
template <class V>
static void H(const char* name, const V& v) {
   std::printf("%s %zu %016llx\n", name, v.size(), (unsigned long long)fnv(v.data(), v.size() * sizeof(v[0])));
}
static void HG(const char* name, const std::vector<fftsvd::LaunchGroup>& g) {  // field by field: no padding bytes
   std::vector<long long> f;
   for (const auto& x : g) {
      const long long a[8] = {x.n, x.begin, x.count, x.smem_elems, x.max_rank, (long long)x.units, x.batch_shared,
                              x.batch_per_rhs};
      f.insert(f.end(), a, a + 8);
   }
   H(name, f);
}

int main(int argc, char** argv) {
   if (argc != 2) {
      std::fprintf(stderr, "usage: %s problem.bin\n", argv[0]);
      return 2;
   }
   FILE* f = std::fopen(argv[1], "rb");
   if (!f) return 1;
   long long hdr[2];
   double par[3];
   if (std::fread(hdr, 8, 2, f) != 2 || std::fread(par, 8, 3, f) != 3) return 1;
   std::vector<double> tri(hdr[0] * 9), qp(hdr[1] * 3), q(hdr[1]);
   if (std::fread(tri.data(), 8, tri.size(), f) != tri.size() || std::fread(qp.data(), 8, qp.size(), f) != qp.size() ||
       std::fread(q.data(), 8, q.size(), f) != q.size())
      return 1;
   std::fclose(f);
   fftsvd_problem pr{};
   pr.num_panels = (int)hdr[0];
   pr.vertices = tri.data();
   pr.num_charges = (int)hdr[1];
   pr.charge_pos = qp.data();
   pr.charge = q.data();
   pr.eps_in = par[0];
   pr.eps_out = par[1];
   pr.kappa = par[2];
   pr.svd_tol = 1e-4;
   pr.max_panels_per_leaf = 32;
   pr.grid_points = 4;
   pr.num_threads = 0;  // OMP_NUM_THREADS
   fftsvd::setup::HostOperator Ho;
   const fftsvd::setup::BatchEvaluator ev = fftsvd::setup::host_evaluator();
   fftsvd::setup::host_setup(pr, Ho, &ev);
   for (int t = 0; t < 2; t++) {
      const auto& F = Ho.flat[t];
      std::printf("tree %d depth %d cubes %d\n", t, F.depth, F.num_cubes);
      H("leaf_rows", F.leaf_rows); H("leaf_cols", F.leaf_cols); H("d_single", F.d_single); H("d_double", F.d_double);
      H("cube_index", F.cube_index); H("cube_panels", F.cube_panels); H("cube_points", F.cube_points);
      H("inter_cubes", F.inter_cubes); H("vt", F.vt); H("pv_single", F.pv_single); H("pv_double", F.pv_double);
      H("uti", F.uti); H("u", F.u); H("t_ops", F.t_ops);
   }
   const fftsvd::OperatorLayout L = fftsvd::build_layout(2 * Ho.n, 2, Ho.views, Ho.maps);
   H("join_phi_idx", L.join_phi_idx); H("point_out", L.point_out); H("leaves", L.leaves); H("leaf_rows", L.leaf_rows);
   H("leaf_cols", L.leaf_cols); H("d_pairs", L.d_pairs); H("src", L.src); H("src_panels", L.src_panels);
   H("vt", L.vt); H("pv_pairs", L.pv_pairs); H("dst", L.dst); H("dst_points", L.dst_points); H("uti", L.uti);
   H("u_cm", L.u_cm); H("inter_pairs", L.inter_pairs); H("t_pairs", L.t_pairs);
   HG("src_groups", L.src_groups); HG("dst_groups", L.dst_groups);
   H("fwd.tiles", L.fwd.tiles); H("fwd.entries", L.fwd.tile_entries); H("fwd.grp", L.fwd.tile_grp);
   H("fwd.src", L.fwd.tile_src); H("fwd.dst", L.fwd.tile_dst); H("fwd.delta", L.fwd.tile_delta);
   H("adj.tiles", L.adj.tiles); H("adj.entries", L.adj.tile_entries); H("adj.grp", L.adj.tile_grp);
   H("adj.src", L.adj.tile_src); H("adj.dst", L.adj.tile_dst); H("adj.delta", L.adj.tile_delta);
   std::printf("scalars %lld %lld %lld %lld %lld\n", (long long)L.total_panels, (long long)L.spectra_elems,
               (long long)L.translated_elems, (long long)L.operator_elems, (long long)L.t_elems);
   return 0;
}
