// Host setup of the compressed FFTSVD operator (see setup.cpp).
#pragma once

#include <array>
#include <cstdint>
#include <functional>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fftsvd_b200.h"
#include "fill_later.h"
#include "integrals.h"

namespace fftsvd {
namespace setup {

struct Kernel {
   bool yukawa = false;
   double kappa = 0.0;
   void panel(const double* point, const FlatPanel& p, double* slp, double* dlp) const;
   double point(const double* dest, const double* src) const;
};

// A block of panel integrals: the single- and double-layer integrals of every panel of a
// panel list at every point of a point list, written row by row into one output array
// (point i, panel k: slp at out_s + i * ld_s + k, dlp at out_d + i * ld_d + k).
struct IntegralBlock {
   int32_t npts = 0, npan = 0;
   int64_t pt_off = 0;   // first point (xyz triple) in IntegralBatch::points
   int64_t pan_off = 0;  // first panel index in IntegralBatch::panels
   int64_t out_s = 0, out_d = 0;
   int32_t ld_s = 0, ld_d = 0;
};
struct IntegralBatch {
   std::vector<double, FillLater<double>> points;  // 3 per point (sized, then written in parallel)
   std::vector<int32_t> panels;                    // indices into the tree's panels
   std::vector<IntegralBlock> blocks;
   int64_t out_elems = 0;        // size of the output array
};

// Evaluates every block of a batch with one kernel over the tree's panels and returns the
// output array (out_elems doubles), valid until the evaluator's next call.  Trees without an
// evaluator integrate on the host, panel by panel; the device evaluator (sampling.cu) runs
// the same integrals on the GPU and returns them in a host buffer it owns.
using BatchEvaluator =
    std::function<const double*(const Kernel& k, const std::vector<FlatPanel>& panels, const IntegralBatch& b)>;

struct Cube {
   int level = 0;
   int idx[3] = {0, 0, 0};
   double b0[3] = {0, 0, 0}, b1[3] = {0, 0, 0}, center[3] = {0, 0, 0};
   int parent = -1;
   bool leaf = false;
   int child[8] = {-1, -1, -1, -1, -1, -1, -1, -1};
   std::vector<int> panels, points, local, inter, dcols;
   std::vector<double> Ds, Dd;        // near-field blocks, points x dcols
   int rowrank = 0, colrank = 0;
   std::vector<double> VT, U;         // rowrank x panels, points x colrank
   std::vector<double> PVs, PVd, UTI; // n^3 x rowrank (x2), colrank x n^3
};

// Owned flat arrays of one tree; view() exposes them as fftsvd_tree_flat.
struct FlatTree {
   int num_panels = 0, num_points = 0, depth = 0, num_cubes = 0;
   std::vector<int> grid;
   std::vector<int32_t> leaf_row_ptr, leaf_rows, leaf_col_ptr, leaf_cols;
   std::vector<int64_t> leaf_d_ptr;
   // the large arrays are sized first and filled in parallel: no zero-fill pass
   std::vector<double, FillLater<double>> d_single, d_double;
   std::vector<int32_t> cube_level, cube_index, cube_panel_ptr, cube_panels, cube_point_ptr, cube_points;
   std::vector<int32_t> cube_row_rank, cube_col_rank, inter_ptr, inter_cubes;
   std::vector<int64_t> cube_vt_ptr, cube_pv_ptr, cube_uti_ptr, cube_u_ptr, t_level_ptr;
   std::vector<double, FillLater<double>> vt, pv_single, pv_double, uti, u, t_ops;
   void view(fftsvd_tree_flat& t) const;
};

struct Tree {
   const std::vector<FlatPanel>* panels = nullptr;
   const std::vector<double>* points = nullptr;  // 3 per point
   Kernel kernel;
   double eps = 1e-5;
   int grid_points = 4;
   int depth = 0;
   std::vector<int> grid;
   double bounds0[3] = {0, 0, 0}, bounds1[3] = {0, 0, 0};
   double rootbox = 0.0;
   std::vector<Cube> cubes;                  // cubes[0] is the root
   std::vector<std::vector<double>> pinv;    // per level, n^3 x 49
   std::vector<std::vector<double>> tops;    // per level, 343 slots x padded grid complex (re, im)
   const BatchEvaluator* eval = nullptr;     // near-field blocks and first-pass samples in batches
   double eval_ms = 0.0;                     // wall time inside eval

   void build_cubes(int depth);
   using Octants = std::array<std::vector<int>, 8>;
   void octants(size_t ci, Octants& panels_in, Octants& points_in) const;  // cube ci's items by octant
   void append_children(size_t ci, Octants& panels_in, Octants& points_in);  // its children, appended
   void add_level();  // one more level below the current leaves
   void choose_depth(int max_panels);
   void make_lists();
   void make_lists_of(size_t ci);
   void fill_near();
   void fill_pinv();
   void fill_T();
   void fill_bases();
   // sampled matrices of one cube (Cube.c:1104-1281): row samples of `pass` passes
   // (2 nwp pass x m), column samples (np x 2 nwq pass), and the 49-point sphere fits
   // of its panels (49 x m each layer)
   void row_samples(const Cube& c, const std::vector<int>& withpoints, int pass, std::vector<double>& R) const;
   void col_samples(const Cube& c, const std::vector<int>& withpanels, int pass, std::vector<double>& Cm) const;
   void sphere_points(const Cube& c, double (*sphere)[3]) const;
   void flatten(FlatTree& F) const;
};

struct Timings {
   double partition_ms = 0, near_ms = 0, pinv_t_ms = 0, bases_ms = 0, flatten_ms = 0;
   double integrals_ms = 0;  // inside the evaluator (part of near_ms and bases_ms)
};

Timings build_tree(Tree& T, int max_panels);

// The complete host-side product for one molecule: both region trees in flat
// form, the region maps and the preconditioner entries.
struct HostOperator {
   int n = 0;
   double eps_in = 1, eps_out = 1, kappa = 0;
   std::vector<FlatPanel> panels;
   std::vector<double> points;
   FlatTree flat[2];
   fftsvd_tree_flat views[2];
   int depth[2] = {0, 0};
   Timings tm[2];
   std::vector<int32_t> idx_phi, idx_dphi, out_outer;
   std::vector<double> m1, ratio, jump, one, zero;
   fftsvd_region_map maps[2];
   std::vector<int32_t> col_ptr, rows;
   std::vector<double> vals;
   fftsvd_precond_csc precond;
};

// Build the two-region operator on the host.  With an evaluator the near-field blocks,
// the first-pass basis samples and the sphere fits are integrated in batches through it
// (the GPU with device_evaluator()); without one everything runs on the host.
void host_setup(const fftsvd_problem& pr, HostOperator& H, const BatchEvaluator* eval = nullptr);

// The same batches evaluated on the host, block by block (the batch layout without the
// device's rounding).
BatchEvaluator host_evaluator();

// The panel-integral evaluator on the current CUDA device (sampling.cu).  It keeps a
// device copy of the panel list between calls and throws DeviceError on a CUDA failure.
BatchEvaluator device_evaluator();
struct DeviceError : std::runtime_error {
   int code;
   DeviceError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

int column_basis(const std::vector<double>& A, int rows, int cols, double eps, std::vector<double>& Q);
int row_basis(const std::vector<double>& A, int rows, int cols, double eps, std::vector<double>& VT);
void pseudoinverse(const std::vector<double>& X, int rows, int cols, std::vector<double>& XI);

}  // namespace setup
}  // namespace fftsvd
