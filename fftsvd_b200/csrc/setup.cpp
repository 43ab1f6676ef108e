// Host setup of the two-region PBE operator: octree partitioning, local and
// interacting lists, near-field panel integrals, sampled low-rank bases,
// equivalent-density projection/interpolation and translation operators.
// OpenMP over cubes; FP64 throughout.  The result is handed to the device
// upload in the flat layout of include/fftsvd_b200.h.
//
// Reference steps restated (same algorithm and ordering, own code):
//   bounding cube, depth rule, grid per level     Tree.c:12-178
//   cube partitioning                             Cube.c:352-542
//   local / interacting lists                     Cube.c:600-713
//   near-field blocks D                           Cube.c:715-793
//   equivalent-density fitting pinv               Tree.c:295-369, EquivDensity.c:461-535, Matrix.c:467-541
//   translation operators                         Tree.c:387-445, FFT.c:10-62
//   sampled row/column bases (pivoted MGS)        Cube.c:1104-1412, Matrix.c:200-307
//   projection P, interpolation I, PV, UTI        Cube.c:795-1002, 1414-1522
//   two-region operator and its preconditioner    FFTSVDpbeAPI.c:1381-1730, SurfaceOperator.c:170-197
#include <omp.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <complex>
#include <cstring>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fftsvd_b200.h"
#include "integrals.h"
#include "fill_later.h"
#include "setup.h"

namespace fftsvd {
namespace setup {

// Points of the 49-point sphere rule used for equivalent densities with a
// 4-point grid edge (EquivDensity.c:31-81; the rule's weights are not used).
// The compressed operator depends on these exact points, so they are kept
// identical to the reference's table.
static const double kSphere49[49][3] = {
    {0.00000000000000e+00, 0.00000000000000e+00, 1.00000000000000e+00},
    {7.51710288002000e-01, 0.00000000000000e+00, 6.59493474503000e-01},
    {-9.46301615589000e-01, 1.11358268319000e-01, -3.03500557512000e-01},
    {-4.86900194038000e-01, 8.70777020028000e-01, 6.83782307220000e-02},
    {-5.27391434139000e-01, -7.04015346866000e-01, -4.75626604149000e-01},
    {-4.48505119250000e-01, -8.93582998351000e-01, -1.87771953310000e-02},
    {-9.74460149410000e-02, 9.05378953618000e-01, 4.13271369100000e-01},
    {5.50822240063000e-01, 7.94124021354000e-01, -2.56830486042000e-01},
    {-9.78434783596000e-01, -1.04177496764000e-01, 1.78360375132000e-01},
    {-8.76905216340000e-01, -4.12324764656000e-01, -2.47033459287000e-01},
    {3.98256992629000e-01, 2.61526233542000e-01, 8.79201567896000e-01},
    {-6.69306929050000e-01, -2.37181230045000e-01, -7.04111709063000e-01},
    {7.64655090996000e-01, 4.68957452919000e-01, 4.42019794993000e-01},
    {-3.47964516179000e-01, -7.92852623440000e-01, 5.00305319765000e-01},
    {8.71692511477000e-01, -4.90013429708000e-01, -6.24532957400000e-03},
    {2.93657134005000e-01, -6.40825485714000e-01, -7.09301194491000e-01},
    {-7.73116928075000e-01, -5.92554389886000e-01, 2.26206787146000e-01},
    {-4.75237224640000e-02, -9.12621548355000e-01, -4.06033748945000e-01},
    {7.31266785297000e-01, -4.73959921471000e-01, -4.90521030702000e-01},
    {-5.51465127541000e-01, 6.34615762534000e-01, 5.41432403029000e-01},
    {6.44209073277000e-01, -5.64517671640000e-02, -7.62763310530000e-01},
    {6.92722856447000e-01, 4.21884929021000e-01, -5.84934313253000e-01},
    {-2.73554241687000e-01, 8.59396086145000e-01, -4.31979680046000e-01},
    {-6.49898888274000e-01, 2.70856029608000e-01, -7.10118614208000e-01},
    {3.61976419280000e-01, -3.44213376481000e-01, 8.66308388126000e-01},
    {5.07635190992000e-01, -8.26097527172000e-01, 2.44682219352000e-01},
    {2.98735120815000e-01, 6.89801932174000e-01, 6.59492700460000e-01},
    {6.33927044960000e-02, 9.94636647537000e-01, -8.17270114050000e-02},
    {4.74133867863000e-01, 8.51450083933000e-01, 2.24120123853000e-01},
    {-6.79982125717000e-01, -3.37102260841000e-01, 6.51142361117000e-01},
    {4.53556145112000e-01, -8.56452647613000e-01, -2.46527251288000e-01},
    {-8.18011633003000e-01, 1.89869850151000e-01, 5.42960779685000e-01},
    {-4.71069574854000e-01, 9.67142748140000e-02, 8.76778081783000e-01},
    {3.08464171700000e-02, -9.90369675350000e-01, 1.34968161783000e-01},
    {8.88626055874000e-01, 4.55017273936000e-01, -5.74718473800000e-02},
    {-2.10335886608000e-01, -5.19928615979000e-01, -8.27908841051000e-01},
    {2.14118410404000e-01, 7.56561192454000e-01, -6.17874152557000e-01},
    {2.59533150783000e-01, 3.19070821555000e-01, -9.11502251493000e-01},
    {-7.08052311545000e-01, 6.13587992853000e-01, -3.49530684121000e-01},
    {9.79812177264000e-01, -1.57544226780000e-02, 1.99298508400000e-01},
    {-2.22340301508000e-01, 5.24139262435000e-01, -8.22096602535000e-01},
    {1.67477396774000e-01, -7.58248188324000e-01, 6.30088094217000e-01},
    {-8.76570276537000e-01, 4.68013139928000e-01, 1.12197375847000e-01},
    {7.24015897788000e-01, -4.70708128402000e-01, 5.04217054061000e-01},
    {-1.51937691391000e-01, 5.15313805780000e-01, 8.43425526948000e-01},
    {2.06742881789000e-01, -2.04177491376000e-01, -9.56853663234000e-01},
    {-2.11715623925000e-01, -4.49224190836000e-01, 8.67971267355000e-01},
    {-2.52573444616000e-01, 1.36078894400000e-02, -9.67482031058000e-01},
    {9.47099296608000e-01, -4.22215539400000e-03, -3.20912909943000e-01},
};
static constexpr int kNumSphere = 49;

// ------------------------------------------------------------------ kernels

void Kernel::panel(const double* point, const FlatPanel& p, double* slp, double* dlp) const {
   if (yukawa) {
      if (!yukawa_panel(point, p, kappa, slp, dlp)) throw std::runtime_error("Yukawa panel integration did not converge");
   } else {
      laplace_panel(point, p, slp, dlp);
   }
}

double Kernel::point(const double* dest, const double* src) const {
   return yukawa ? green_yukawa(dest, src, kappa) : green_laplace(dest, src);
}

// ------------------------------------------------------------------ dense linear algebra

// Orthonormal column basis of A (rows x cols, row-major) by modified
// Gram-Schmidt with column pivoting and two re-orthogonalisation passes,
// stopping when the largest remaining column norm falls below
// eps * ||A||_F (Matrix.c:214-307).  Returns rank; Q is rows x rank.
int column_basis(const std::vector<double>& Ain, int rows, int cols, double eps, std::vector<double>& Q) {
   std::vector<double> A = Ain;
   std::vector<double> Qf((size_t)rows * cols, 0.0);
   double fro = 0.0;
   for (double v : A) fro += v * v;
   fro = std::sqrt(fro);
   int rank = cols;
   std::vector<double> Rk(cols);
   for (int k = 0; k < cols; k++) {
      double maxnorm = 0.0;
      int best = 0;
      for (int l = k; l < cols; l++) {
         double s = 0.0;
         for (int i = 0; i < rows; i++) s += A[(size_t)i * cols + l] * A[(size_t)i * cols + l];
         s = std::sqrt(s);
         if (s > maxnorm) { maxnorm = s; best = l; }
      }
      if (k >= 1 && maxnorm < eps * fro) { rank = k; break; }
      if (best != k)
         for (int i = 0; i < rows; i++) std::swap(A[(size_t)i * cols + best], A[(size_t)i * cols + k]);
      for (int i = 0; i < rows; i++) Qf[(size_t)i * cols + k] = A[(size_t)i * cols + k] / maxnorm;
      if (k < cols - 1)
         for (int pass = 0; pass < 2; pass++) {
            std::fill(Rk.begin() + k + 1, Rk.end(), 0.0);
            for (int i = 0; i < rows; i++) {
               const double q = Qf[(size_t)i * cols + k];
               const double* ai = &A[(size_t)i * cols];
               for (int j = k + 1; j < cols; j++) Rk[j] += q * ai[j];
            }
            for (int i = 0; i < rows; i++) {
               const double q = Qf[(size_t)i * cols + k];
               double* ai = &A[(size_t)i * cols];
               for (int j = k + 1; j < cols; j++) ai[j] -= q * Rk[j];
            }
         }
   }
   Q.assign((size_t)rows * rank, 0.0);
   for (int i = 0; i < rows; i++)
      for (int j = 0; j < rank; j++) Q[(size_t)i * rank + j] = Qf[(size_t)i * cols + j];
   return rank;
}

// Row basis: column basis of the transpose, transposed back (Matrix.c:200-212).
int row_basis(const std::vector<double>& A, int rows, int cols, double eps, std::vector<double>& VT) {
   std::vector<double> At((size_t)cols * rows);
   for (int i = 0; i < rows; i++)
      for (int j = 0; j < cols; j++) At[(size_t)j * rows + i] = A[(size_t)i * cols + j];
   std::vector<double> Q;
   const int rank = column_basis(At, cols, rows, eps, Q);  // cols x rank
   VT.assign((size_t)rank * cols, 0.0);
   for (int i = 0; i < cols; i++)
      for (int j = 0; j < rank; j++) VT[(size_t)j * cols + i] = Q[(size_t)i * rank + j];
   return rank;
}

// Moore-Penrose pseudo-inverse of X (rows x cols, row-major) via a one-sided
// Jacobi SVD, singular values below max(rows, cols) * s_max * eps_double
// dropped (Matrix.c:467-541).  XI is cols x rows.
void pseudoinverse(const std::vector<double>& X, int rows, int cols, std::vector<double>& XI) {
   // work on B = X^T (cols x rows) when rows < cols so that B has >= as many rows as columns
   const bool tr = rows < cols;
   const int p = tr ? cols : rows, q = tr ? rows : cols;
   std::vector<double> B((size_t)p * q), V((size_t)q * q, 0.0);  // B column-major p x q
   for (int j = 0; j < q; j++)
      for (int i = 0; i < p; i++) B[(size_t)j * p + i] = tr ? X[(size_t)j * cols + i] : X[(size_t)i * cols + j];
   for (int i = 0; i < q; i++) V[(size_t)i * q + i] = 1.0;
   for (int sweep = 0; sweep < 80; sweep++) {
      double off = 0.0;
      for (int j = 0; j < q - 1; j++)
         for (int k = j + 1; k < q; k++) {
            double a = 0, b = 0, g = 0;
            double *bj = &B[(size_t)j * p], *bk = &B[(size_t)k * p];
            for (int i = 0; i < p; i++) { a += bj[i] * bj[i]; b += bk[i] * bk[i]; g += bj[i] * bk[i]; }
            if (std::fabs(g) <= 1e-300) continue;
            const double relv = std::fabs(g) / std::sqrt(a * b);
            off = std::max(off, relv);
            if (relv < 1e-17) continue;
            const double zeta = (b - a) / (2.0 * g);
            const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
            const double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
            for (int i = 0; i < p; i++) {
               const double x = bj[i], y = bk[i];
               bj[i] = c * x - s * y;
               bk[i] = s * x + c * y;
            }
            double *vj = &V[(size_t)j * q], *vk = &V[(size_t)k * q];
            for (int i = 0; i < q; i++) {
               const double x = vj[i], y = vk[i];
               vj[i] = c * x - s * y;
               vk[i] = s * x + c * y;
            }
         }
      if (off < 1e-16) break;
   }
   std::vector<double> sig(q);
   double smax = 0.0;
   for (int j = 0; j < q; j++) {
      double s = 0.0;
      for (int i = 0; i < p; i++) s += B[(size_t)j * p + i] * B[(size_t)j * p + i];
      sig[j] = std::sqrt(s);
      smax = std::max(smax, sig[j]);
   }
   const double tol = std::max(rows, cols) * smax * 2.220446049250313e-16;
   // B = W (orthogonal columns, |W_j| = sig_j), Bin = W V^T  =>  Bin^+ = V diag(1/sig^2) W^T
   // pinv(B)^T = pinv(B^T): X = B (tr == false) or X = B^T (tr == true)
   XI.assign((size_t)cols * rows, 0.0);
   for (int j = 0; j < q; j++) {
      if (!(sig[j] > tol)) continue;
      const double inv2 = 1.0 / (sig[j] * sig[j]);
      const double* w = &B[(size_t)j * p];
      const double* v = &V[(size_t)j * q];
      if (!tr) {  // X (p x q) = W V^T ; X^+ (q x p) = V diag W^T / sig^2
         for (int a = 0; a < q; a++) {
            const double va = v[a] * inv2;
            if (va == 0.0) continue;
            for (int b2 = 0; b2 < p; b2++) XI[(size_t)a * p + b2] += va * w[b2];
         }
      } else {    // X = B^T (q x p) = V W^T ; X^+ (p x q) = W V^T / sig^2
         for (int a = 0; a < p; a++) {
            const double wa = w[a] * inv2;
            if (wa == 0.0) continue;
            for (int b2 = 0; b2 < q; b2++) XI[(size_t)a * q + b2] += wa * v[b2];
         }
      }
   }
}

// Real-data forward DFT of an N x N x N array (row-major) to N x N x (N/2+1), exponent -1.
static void r2c3(int N, const std::vector<double>& in, std::vector<std::complex<double>>& out) {
   const int H = N / 2 + 1;
   std::vector<std::complex<double>> w(N), t1((size_t)N * N * H), t2((size_t)N * N * H);
   for (int k = 0; k < N; k++) w[k] = std::polar(1.0, -2.0 * M_PI * k / N);
   for (int i = 0; i < N; i++)
      for (int j = 0; j < N; j++)
         for (int b = 0; b < H; b++) {
            std::complex<double> acc = 0.0;
            for (int k = 0; k < N; k++) acc += in[((size_t)i * N + j) * N + k] * w[(b * k) % N];
            t1[((size_t)i * N + j) * H + b] = acc;
         }
   for (int i = 0; i < N; i++)
      for (int a = 0; a < N; a++)
         for (int b = 0; b < H; b++) {
            std::complex<double> acc = 0.0;
            for (int j = 0; j < N; j++) acc += t1[((size_t)i * N + j) * H + b] * w[(a * j) % N];
            t2[((size_t)i * N + a) * H + b] = acc;
         }
   out.assign((size_t)N * N * H, 0.0);
   for (int a = 0; a < N; a++)
      for (int j = 0; j < N; j++)
         for (int b = 0; b < H; b++) {
            std::complex<double> acc = 0.0;
            for (int i = 0; i < N; i++) acc += t2[((size_t)i * N + j) * H + b] * w[(a * i) % N];
            out[((size_t)a * N + j) * H + b] = acc;
         }
}

// ------------------------------------------------------------------ tree

// The octant of every panel and point of cube ci (coordinate >= the centre: upper half), in
// the cube's own order within each octant.
void Tree::octants(size_t ci, Octants& bp, Octants& bq) const {
   const Cube& par = cubes[ci];
   const double cc[3] = {par.center[0], par.center[1], par.center[2]};
   auto octant = [&](const double* p) { return (p[0] >= cc[0]) * 4 + (p[1] >= cc[1]) * 2 + (p[2] >= cc[2]); };
   for (int i : par.panels) bp[octant((*panels)[i].centroid)].push_back(i);
   for (int i : par.points) bq[octant(&(*points)[3 * (size_t)i])].push_back(i);
}

// Children of cube ci in cx, cy, cz order from its octant lists; empty octants get no cube.
void Tree::append_children(size_t ci, Octants& bp, Octants& bq) {
   const Cube& par = cubes[ci];
   const double cc[3] = {par.center[0], par.center[1], par.center[2]};
   const double pb0[3] = {par.b0[0], par.b0[1], par.b0[2]};
   const int pidx[3] = {par.idx[0], par.idx[1], par.idx[2]}, plevel = par.level;
   for (int slot = 0; slot < 8; slot++) {
      if (bp[slot].empty() && bq[slot].empty()) continue;
      const int cbit[3] = {slot >> 2, (slot >> 1) & 1, slot & 1};
      Cube ch;
      ch.panels = std::move(bp[slot]);
      ch.points = std::move(bq[slot]);
      for (int k = 0; k < 3; k++) {
         ch.b0[k] = pb0[k];
         ch.b1[k] = cc[k];
         if (cbit[k] == 1) {
            const double diff = cc[k] - ch.b0[k];
            ch.b0[k] += diff;
            ch.b1[k] += diff;
         }
         ch.idx[k] = 2 * pidx[k] + cbit[k];
      }
      ch.level = plevel + 1;
      ch.parent = (int)ci;
      cubes.push_back(std::move(ch));  // may move the parent: nothing of it is used below
      cubes[ci].child[slot] = (int)cubes.size() - 1;
   }
}

// Cubes are kept in breadth-first creation order (children of one cube in cx, cy, cz
// order), so the tree of depth d + 1 is the tree of depth d with the children of its
// leaves appended in order.  The leaves' panels and points are sorted into octants in
// parallel; the children are then appended leaf after leaf.
void Tree::add_level() {
   const size_t n0 = cubes.size();
   std::vector<size_t> split;
   for (size_t ci = 0; ci < n0; ci++)
      if (cubes[ci].level == depth - 1) split.push_back(ci);
   std::vector<Octants> bp(split.size()), bq(split.size());
#pragma omp parallel for schedule(dynamic, 16)
   for (int64_t i = 0; i < (int64_t)split.size(); i++) octants(split[i], bp[i], bq[i]);
   for (size_t i = 0; i < split.size(); i++) {
      cubes[split[i]].leaf = false;
      append_children(split[i], bp[i], bq[i]);
   }
   depth++;
   for (size_t ci = n0; ci < cubes.size(); ci++) {
      Cube& c = cubes[ci];
      for (int k = 0; k < 3; k++) c.center[k] = (c.b0[k] + c.b1[k]) * 0.5;
      for (int k = 0; k < 8; k++) c.child[k] = -1;
      c.leaf = true;
   }
}

void Tree::build_cubes(int depth_) {
   depth = 1;
   cubes.clear();
   Cube root;
   root.level = 0;
   root.idx[0] = root.idx[1] = root.idx[2] = 0;
   for (int k = 0; k < 3; k++) { root.b0[k] = bounds0[k]; root.b1[k] = bounds1[k]; }
   root.parent = -1;
   root.panels.resize(panels->size());
   for (size_t i = 0; i < panels->size(); i++) root.panels[i] = (int)i;
   root.points = root.panels;
   for (int k = 0; k < 3; k++) root.center[k] = (root.b0[k] + root.b1[k]) * 0.5;
   for (int k = 0; k < 8; k++) root.child[k] = -1;
   root.leaf = true;
   cubes.push_back(std::move(root));
   while (depth < depth_) add_level();
}

void Tree::choose_depth(int max_panels) {
   const double* c0 = (*panels)[0].centroid;
   double mn[3] = {1000000.0, 1000000.0, 1000000.0}, mx[3] = {-1000000.0, -1000000.0, -1000000.0};
   (void)c0;
   for (const auto& p : *panels)
      for (int k = 0; k < 3; k++) { mn[k] = std::min(mn[k], p.centroid[k]); mx[k] = std::max(mx[k], p.centroid[k]); }
   const size_t np = points->size() / 3;
   for (size_t i = 0; i < np; i++)
      for (int k = 0; k < 3; k++) {
         const double v = (*points)[3 * i + k];
         if (v < mn[k]) mn[k] = v;
         if (v > mx[k]) mx[k] = v;
      }
   double ext = 0.0, ctr[3];
   for (int k = 0; k < 3; k++) {
      ctr[k] = (mn[k] + mx[k]) * 0.5;
      if (mx[k] - mn[k] > ext) ext = mx[k] - mn[k];
   }
   for (int k = 0; k < 3; k++) { bounds0[k] = ctr[k] - ext * 0.5; bounds1[k] = ctr[k] + ext * 0.5; }
   for (int d = 2;; d++) {
      if (d == 2)
         build_cubes(d);
      else
         add_level();
      if (panels->empty() || np == 0) break;
      int leaves = 0, within = 0;
      for (const Cube& c : cubes)
         if (c.leaf) {
            leaves++;
            if ((int)c.panels.size() <= max_panels) within++;
         }
      if ((double)within / (double)leaves > 0.90) break;
      if (d >= FFTSVD_MAX_DEPTH) break;
   }
   grid.assign(depth, grid_points);
   for (int i = depth - 3, p = 1; i >= 0; i--, p++) grid[i] = grid_points + p;
   rootbox = bounds1[0] - bounds0[0];
}

void Tree::make_lists() {
   for (Cube& c : cubes) { c.local.clear(); c.inter.clear(); }
   // cubes are in breadth-first order, so each level is one contiguous range and a cube needs
   // only its parent's list, complete once the level above is: one level at a time, its
   // cubes in parallel
   for (size_t lo = 0; lo < cubes.size();) {
      size_t hi = lo;
      while (hi < cubes.size() && cubes[hi].level == cubes[lo].level) hi++;
#pragma omp parallel for schedule(dynamic, 256)
      for (int64_t ci = (int64_t)lo; ci < (int64_t)hi; ci++) make_lists_of((size_t)ci);
      lo = hi;
   }
}

// The local (neighbouring) and interaction lists of cube ci: the other children of its
// parent and the children of the parent's neighbours, split by whether they touch cube ci.
void Tree::make_lists_of(size_t ci) {
   Cube& c = cubes[ci];
   if (c.parent < 0) return;
   const Cube& par = cubes[c.parent];
   for (int k = 0; k < 8; k++)
      if (par.child[k] >= 0 && par.child[k] != (int)ci) c.local.push_back(par.child[k]);
   for (int pl : par.local)
      for (int k = 0; k < 8; k++) {
         const int o = cubes[pl].child[k];
         if (o < 0) continue;
         const Cube& oc = cubes[o];
         const bool near = std::abs(oc.idx[0] - c.idx[0]) <= 1 && std::abs(oc.idx[1] - c.idx[1]) <= 1 &&
                           std::abs(oc.idx[2] - c.idx[2]) <= 1;
         if (near) c.local.push_back(o);
      }
   for (int pl : par.local)
      for (int k = 0; k < 8; k++) {
         const int o = cubes[pl].child[k];
         if (o < 0) continue;
         const Cube& oc = cubes[o];
         const bool far = std::abs(oc.idx[0] - c.idx[0]) > 1 || std::abs(oc.idx[1] - c.idx[1]) > 1 ||
                          std::abs(oc.idx[2] - c.idx[2]) > 1;
         if (far) c.inter.push_back(o);
      }
}

void Tree::fill_near() {
   std::vector<int> leaves;
   for (size_t i = 0; i < cubes.size(); i++)
      if (cubes[i].leaf) leaves.push_back((int)i);
   const int64_t nl = (int64_t)leaves.size();
#pragma omp parallel for schedule(dynamic, 64)
   for (int64_t li = 0; li < nl; li++) {
      Cube& c = cubes[leaves[li]];
      c.dcols = c.panels;
      for (int o : c.local) c.dcols.insert(c.dcols.end(), cubes[o].panels.begin(), cubes[o].panels.end());
   }
   if (eval) {
      // every leaf block in one batch: Ds then Dd of each leaf, row-major.  Sizes first,
      // running offsets from them, then every leaf's part written in parallel: the batch is
      // laid out exactly as if the leaves' blocks were appended one after another.
      IntegralBatch B;
      std::vector<int64_t> off(leaves.size(), -1);
      std::vector<int64_t> pt_at(nl + 1, 0), pan_at(nl + 1, 0), out_at(nl + 1, 0), blk_at(nl + 1, 0);
      for (int64_t li = 0; li < nl; li++) {
         const Cube& c = cubes[leaves[li]];
         const int64_t nr = (int64_t)c.points.size(), nc = (int64_t)c.dcols.size();
         const bool some = nr > 0 && nc > 0;
         pt_at[li + 1] = pt_at[li] + (some ? nr : 0);
         pan_at[li + 1] = pan_at[li] + (some ? nc : 0);
         out_at[li + 1] = out_at[li] + (some ? 2 * nr * nc : 0);
         blk_at[li + 1] = blk_at[li] + (some ? 1 : 0);
      }
      B.points.resize(3 * (size_t)pt_at[nl]);
      B.panels.resize((size_t)pan_at[nl]);
      B.blocks.resize((size_t)blk_at[nl]);
      B.out_elems = out_at[nl];
#pragma omp parallel for schedule(dynamic, 64)
      for (int64_t li = 0; li < nl; li++) {
         const Cube& c = cubes[leaves[li]];
         const int nr = (int)c.points.size(), nc = (int)c.dcols.size();
         if (nr == 0 || nc == 0) continue;
         IntegralBlock b;
         b.npts = nr;
         b.npan = nc;
         b.pt_off = pt_at[li];
         double* pdst = B.points.data() + 3 * (size_t)pt_at[li];
         for (int pt : c.points)
            for (int k = 0; k < 3; k++) *pdst++ = (*points)[3 * (size_t)pt + k];
         b.pan_off = pan_at[li];
         std::copy(c.dcols.begin(), c.dcols.end(), B.panels.begin() + pan_at[li]);
         off[li] = out_at[li];
         b.out_s = out_at[li];
         b.out_d = out_at[li] + (int64_t)nr * nc;
         b.ld_s = b.ld_d = nc;
         B.blocks[blk_at[li]] = b;
      }
      const auto e0 = std::chrono::steady_clock::now();
      const double* out = (*eval)(kernel, *panels, B);
      eval_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - e0).count();
#pragma omp parallel for schedule(static)
      for (size_t li = 0; li < leaves.size(); li++) {
         if (off[li] < 0) continue;
         Cube& c = cubes[leaves[li]];
         const size_t e = c.points.size() * c.dcols.size();
         c.Ds.assign(out + off[li], out + off[li] + e);
         c.Dd.assign(out + off[li] + e, out + off[li] + 2 * e);
      }
      return;
   }
#pragma omp parallel for schedule(dynamic, 4)
   for (size_t li = 0; li < leaves.size(); li++) {
      Cube& c = cubes[leaves[li]];
      const int nr = (int)c.points.size(), nc = (int)c.dcols.size();
      if (nr == 0 || nc == 0) continue;
      c.Ds.assign((size_t)nr * nc, 0.0);
      c.Dd.assign((size_t)nr * nc, 0.0);
      for (int r = 0; r < nr; r++) {
         const double* pt = &(*points)[3 * (size_t)c.points[r]];
         for (int k = 0; k < nc; k++) kernel.panel(pt, (*panels)[c.dcols[k]], &c.Ds[(size_t)r * nc + k], &c.Dd[(size_t)r * nc + k]);
      }
   }
}

void Tree::fill_pinv() {
   pinv.assign(depth, {});
#pragma omp parallel for schedule(dynamic, 1)
   for (int d = 0; d < depth; d++) {
      const int n = grid[d], gp3 = n * n * n;
      const double box = rootbox / std::pow(2.0, d), h = box / (n - 1);
      const double ctr[3] = {0.5 * box, 0.5 * box, 0.5 * box};
      std::vector<double> Q((size_t)kNumSphere * gp3);
      for (int q = 0; q < kNumSphere; q++) {
         double sp[3];
         for (int k = 0; k < 3; k++) sp[k] = kSphere49[q][k] * (box * 1.5) + ctr[k];
         int g = 0;
         for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
               for (int k = 0; k < n; k++, g++) {
                  const double gpnt[3] = {i * h, j * h, k * h};
                  Q[(size_t)q * gp3 + g] = kernel.point(gpnt, sp);
               }
      }
      pseudoinverse(Q, kNumSphere, gp3, pinv[d]);  // gp3 x 49
   }
}

void Tree::fill_T() {
   tops.assign(depth, {});
   std::vector<std::pair<int, int>> work;
   for (int d = 0; d < depth; d++) {
      const int Np = 2 * grid[d] - 1, pg = Np * Np * grid[d];
      tops[d].assign((size_t)2 * 343 * pg, 0.0);  // (re, im) pairs
      for (int s = 0; s < 343; s++) {
         const int x = s / 49 - 3, y = (s / 7) % 7 - 3, z = s % 7 - 3;
         if (std::abs(x) <= 1 && std::abs(y) <= 1 && std::abs(z) <= 1) continue;
         work.emplace_back(d, s);
      }
   }
#pragma omp parallel for schedule(dynamic, 2)
   for (size_t wi = 0; wi < work.size(); wi++) {
      const int d = work[wi].first, s = work[wi].second;
      const int n = grid[d], N = 2 * n - 1, pg = N * N * n;
      const int x = s / 49 - 3, y = (s / 7) % 7 - 3, z = s % 7 - 3;
      const double h = rootbox / std::pow(2.0, d) / (n - 1);
      const double shift[3] = {(double)x * (n - 1), (double)y * (n - 1), (double)z * (n - 1)};
      std::vector<double> data((size_t)N * N * N);
      const double zero[3] = {0, 0, 0};
      for (int i = 0; i < N; i++) {
         const int li = (i > N / 2) ? N - i : -i;
         for (int j = 0; j < N; j++) {
            const int lj = (j > N / 2) ? N - j : -j;
            for (int k = 0; k < N; k++) {
               const int lk = (k > N / 2) ? N - k : -k;
               const double p[3] = {h * (shift[0] - li), h * (shift[1] - lj), h * (shift[2] - lk)};
               data[((size_t)i * N + j) * N + k] = kernel.point(p, zero);
            }
         }
      }
      std::vector<std::complex<double>> out;
      r2c3(N, data, out);
      double* dst = &tops[d][(size_t)2 * s * pg];
      for (int f = 0; f < pg; f++) { dst[2 * f] = out[f].real(); dst[2 * f + 1] = out[f].imag(); }
   }
}

void Tree::row_samples(const Cube& c, const std::vector<int>& withpoints, int pass, std::vector<double>& R) const {
   const int m = (int)c.panels.size(), nwp = (int)withpoints.size(), rows = 2 * nwp * pass;
   R.assign((size_t)rows * m, 0.0);
   for (int p = 0; p < pass; p++)
      for (int r = 0; r < nwp; r++) {
         const Cube& pc = cubes[withpoints[r]];
         const int pi = (int)((unsigned)p * (unsigned)pc.points.size() / (unsigned)pass);
         const double* pt = &(*points)[3 * (size_t)pc.points[pi]];
         for (int k = 0; k < m; k++)
            kernel.panel(pt, (*panels)[c.panels[k]], &R[(size_t)(p * nwp + r) * m + k],
                         &R[(size_t)(p * nwp + r + nwp * pass) * m + k]);
      }
}

void Tree::col_samples(const Cube& c, const std::vector<int>& withpanels, int pass, std::vector<double>& Cm) const {
   const int np = (int)c.points.size(), nwq = (int)withpanels.size(), cols = 2 * nwq * pass;
   Cm.assign((size_t)np * cols, 0.0);
   for (int p = 0; p < pass; p++)
      for (int q = 0; q < nwq; q++) {
         const Cube& qc = cubes[withpanels[q]];
         const int pi = (int)((unsigned)p * (unsigned)qc.panels.size() / (unsigned)pass);
         const FlatPanel& pan = (*panels)[qc.panels[pi]];
         for (int r = 0; r < np; r++) {
            const double* pt = &(*points)[3 * (size_t)c.points[r]];
            kernel.panel(pt, pan, &Cm[(size_t)r * cols + p * nwq + q], &Cm[(size_t)r * cols + p * nwq + q + nwq * pass]);
         }
      }
}

void Tree::sphere_points(const Cube& c, double (*sphere)[3]) const {
   const double box = c.b1[0] - c.b0[0];
   for (int q = 0; q < kNumSphere; q++)
      for (int k = 0; k < 3; k++) sphere[q][k] = kSphere49[q][k] * (box * 1.5) + c.center[k];
}

void Tree::fill_bases() {
   std::vector<int> work;
   for (size_t i = 0; i < cubes.size(); i++)
      if (!cubes[i].inter.empty()) work.push_back((int)i);
   // interacting cubes with panels (column samples) and with points (row samples)
   std::vector<std::vector<int>> wpan(work.size()), wpts(work.size());
   for (size_t wi = 0; wi < work.size(); wi++)
      for (int o : cubes[work[wi]].inter) {
         if (!cubes[o].panels.empty()) wpan[wi].push_back(o);
         if (!cubes[o].points.empty()) wpts[wi].push_back(o);
      }
   // With an evaluator the first sampling pass of every cube and its sphere fits are
   // integrated in one batch; a cube whose first pass does not settle its rank samples its
   // further passes on the host as before.
   const double* pre = nullptr;  // the batch's output, owned by the evaluator
   std::vector<int64_t> roff(work.size(), -1), coff(work.size(), -1), soff(work.size(), -1);
   if (eval) {
      IntegralBatch B;
      // per cube: a row block and its sphere-fit block (when it has panels and interacting
      // cubes with points), then a column block (when it has points and interacting cubes
      // with panels).  Sizes first, running offsets from them, then every cube's part
      // written in parallel at its offsets: the batch is laid out exactly as if the blocks
      // were appended one cube after another.
      const size_t nw = work.size();
      std::vector<int64_t> pan_at(nw + 1, 0), pt_at(nw + 1, 0), out_at(nw + 1, 0), blk_at(nw + 1, 0);
#pragma omp parallel for schedule(static)
      for (int64_t wi = 0; wi < (int64_t)nw; wi++) {
         const Cube& c = cubes[work[wi]];
         const int64_t m = (int64_t)c.panels.size(), np = (int64_t)c.points.size();
         const int64_t nwp = (int64_t)wpts[wi].size(), nwq = (int64_t)wpan[wi].size();
         int64_t pan = 0, pt = 0, out = 0, blk = 0;
         if (m > 0 && nwp > 0) {
            pan += m;
            pt += nwp + kNumSphere;
            out += 2 * nwp * m + 2 * (int64_t)kNumSphere * m;
            blk += 2;
         }
         if (np > 0 && nwq > 0) {
            pan += nwq;
            pt += np;
            out += np * 2 * nwq;
            blk += 1;
         }
         pan_at[wi + 1] = pan;
         pt_at[wi + 1] = pt;
         out_at[wi + 1] = out;
         blk_at[wi + 1] = blk;
      }
      for (size_t wi = 0; wi < nw; wi++) {
         pan_at[wi + 1] += pan_at[wi];
         pt_at[wi + 1] += pt_at[wi];
         out_at[wi + 1] += out_at[wi];
         blk_at[wi + 1] += blk_at[wi];
      }
      B.panels.resize((size_t)pan_at[nw]);
      B.points.resize(3 * (size_t)pt_at[nw]);
      B.blocks.resize((size_t)blk_at[nw]);
      B.out_elems = out_at[nw];
#pragma omp parallel for schedule(dynamic, 64)
      for (int64_t wi = 0; wi < (int64_t)nw; wi++) {
         const Cube& c = cubes[work[wi]];
         const int m = (int)c.panels.size(), np = (int)c.points.size();
         const int nwp = (int)wpts[wi].size(), nwq = (int)wpan[wi].size();
         int64_t pan = pan_at[wi], pt = pt_at[wi], out = out_at[wi], blk = blk_at[wi];
         auto put_point = [&](const double* p) {
            std::copy(p, p + 3, B.points.begin() + 3 * pt);
            pt++;
         };
         if (m > 0 && nwp > 0) {
            IntegralBlock b;
            b.pan_off = pan;
            std::copy(c.panels.begin(), c.panels.end(), B.panels.begin() + pan);
            pan += m;
            b.npan = m;
            b.npts = nwp;
            b.pt_off = pt;
            for (int o : wpts[wi]) put_point(&(*points)[3 * (size_t)cubes[o].points[0]]);
            roff[wi] = b.out_s = out;
            b.out_d = out + (int64_t)nwp * m;
            b.ld_s = b.ld_d = m;
            out += 2 * (int64_t)nwp * m;
            B.blocks[blk++] = b;
            // sphere fits of the same panels
            IntegralBlock sb = b;
            double sphere[kNumSphere][3];
            sphere_points(c, sphere);
            sb.npts = kNumSphere;
            sb.pt_off = pt;
            for (int q = 0; q < kNumSphere; q++) put_point(sphere[q]);
            soff[wi] = sb.out_s = out;
            sb.out_d = out + (int64_t)kNumSphere * m;
            out += 2 * (int64_t)kNumSphere * m;
            B.blocks[blk++] = sb;
         }
         if (np > 0 && nwq > 0) {
            IntegralBlock b;
            b.pan_off = pan;
            for (int o : wpan[wi]) B.panels[pan++] = cubes[o].panels[0];
            b.npan = nwq;
            b.npts = np;
            b.pt_off = pt;
            for (int p : c.points) put_point(&(*points)[3 * (size_t)p]);
            coff[wi] = b.out_s = out;
            b.out_d = out + nwq;
            b.ld_s = b.ld_d = 2 * nwq;
            out += (int64_t)np * 2 * nwq;
            B.blocks[blk++] = b;
         }
      }
      const auto e0 = std::chrono::steady_clock::now();
      pre = (*eval)(kernel, *panels, B);
      eval_ms += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - e0).count();
   }
#pragma omp parallel for schedule(dynamic, 1)
   for (size_t wi = 0; wi < work.size(); wi++) {
      Cube& c = cubes[work[wi]];
      const std::vector<int>& withpanels = wpan[wi];
      const std::vector<int>& withpoints = wpts[wi];
      const int m = (int)c.panels.size(), np = (int)c.points.size();
      const int nwp = (int)withpoints.size(), nwq = (int)withpanels.size();
      c.rowrank = 0;
      c.colrank = 0;
      if (m > 0 && nwp > 0) {
         for (int pass = 1;; pass++) {
            const int rows = 2 * nwp * pass;
            std::vector<double> R;
            if (pass == 1 && roff[wi] >= 0)
               R.assign(pre + roff[wi], pre + roff[wi] + (int64_t)rows * m);
            else
               row_samples(c, withpoints, pass, R);
            std::vector<double> VT;
            const int rank = row_basis(R, rows, m, eps, VT);
            if (rank < rows / 2) {
               c.rowrank = rank;
               c.VT = std::move(VT);
               break;
            }
         }
      }
      if (np > 0 && nwq > 0) {
         for (int pass = 1;; pass++) {
            const int cols = 2 * nwq * pass;
            std::vector<double> Cm;
            if (pass == 1 && coff[wi] >= 0)
               Cm.assign(pre + coff[wi], pre + coff[wi] + (int64_t)np * cols);
            else
               col_samples(c, withpanels, pass, Cm);
            std::vector<double> U;
            const int rank = column_basis(Cm, np, cols, eps, U);
            if (rank < cols / 2) {
               c.colrank = rank;
               c.U = std::move(U);
               break;
            }
         }
      }
      // projection (P) and interpolation (I) on the equivalent-density grid, then PV and UTI
      const int n = grid[c.level], gp3 = n * n * n;
      const std::vector<double>& Pi = pinv[c.level];  // gp3 x 49
      double sphere[kNumSphere][3];
      sphere_points(c, sphere);
      if (m > 0 && c.rowrank > 0) {
         std::vector<double> Qs((size_t)kNumSphere * m), Qd((size_t)kNumSphere * m);
         if (soff[wi] >= 0) {
            const int64_t e = (int64_t)kNumSphere * m;
            std::copy(pre + soff[wi], pre + soff[wi] + e, Qs.begin());
            std::copy(pre + soff[wi] + e, pre + soff[wi] + 2 * e, Qd.begin());
         } else {
            for (int q = 0; q < kNumSphere; q++)
               for (int k = 0; k < m; k++)
                  kernel.panel(sphere[q], (*panels)[c.panels[k]], &Qs[(size_t)q * m + k], &Qd[(size_t)q * m + k]);
         }
         // P = pinv Q2S (gp3 x m); PV = P VT^T (gp3 x r)
         const int r = c.rowrank;
         std::vector<double> Ps((size_t)gp3 * m, 0.0), Pd((size_t)gp3 * m, 0.0);
         for (int g = 0; g < gp3; g++)
            for (int q = 0; q < kNumSphere; q++) {
               const double a = Pi[(size_t)g * kNumSphere + q];
               for (int k = 0; k < m; k++) {
                  Ps[(size_t)g * m + k] += a * Qs[(size_t)q * m + k];
                  Pd[(size_t)g * m + k] += a * Qd[(size_t)q * m + k];
               }
            }
         // VT transposed, so that the innermost loop runs over contiguous j; every PV entry
         // still accumulates over k in ascending order
         std::vector<double> VTt((size_t)m * r);
         for (int j = 0; j < r; j++)
            for (int k = 0; k < m; k++) VTt[(size_t)k * r + j] = c.VT[(size_t)j * m + k];
         c.PVs.assign((size_t)gp3 * r, 0.0);
         c.PVd.assign((size_t)gp3 * r, 0.0);
         for (int g = 0; g < gp3; g++) {
            double* pvs = &c.PVs[(size_t)g * r];
            double* pvd = &c.PVd[(size_t)g * r];
            for (int k = 0; k < m; k++) {
               const double ps = Ps[(size_t)g * m + k], pd = Pd[(size_t)g * m + k];
               const double* vt = &VTt[(size_t)k * r];
               for (int j = 0; j < r; j++) {
                  pvs[j] += ps * vt[j];
                  pvd[j] += pd * vt[j];
               }
            }
         }
      }
      if (np > 0 && c.colrank > 0) {
         // I^T = (pinv Q2S_points)^T (np x gp3); UTI = U^T I^T (r x gp3)
         const int r = c.colrank;
         std::vector<double> Qp((size_t)kNumSphere * np);
         for (int q = 0; q < kNumSphere; q++)
            for (int k = 0; k < np; k++) Qp[(size_t)q * np + k] = kernel.point(&(*points)[3 * (size_t)c.points[k]], sphere[q]);
         // accumulated transposed (contiguous in k; each entry still sums over q in ascending
         // order), then turned back into np x gp3
         std::vector<double> ItT((size_t)gp3 * np, 0.0), It((size_t)np * gp3);
         for (int g = 0; g < gp3; g++) {
            double* it = &ItT[(size_t)g * np];
            for (int q = 0; q < kNumSphere; q++) {
               const double a = Pi[(size_t)g * kNumSphere + q];
               const double* qp = &Qp[(size_t)q * np];
               for (int k = 0; k < np; k++) it[k] += a * qp[k];
            }
         }
         for (int g = 0; g < gp3; g++)
            for (int k = 0; k < np; k++) It[(size_t)k * gp3 + g] = ItT[(size_t)g * np + k];
         c.UTI.assign((size_t)r * gp3, 0.0);
         for (int k = 0; k < np; k++)
            for (int j = 0; j < r; j++) {
               const double u = c.U[(size_t)k * r + j];
               for (int g = 0; g < gp3; g++) c.UTI[(size_t)j * gp3 + g] += u * It[(size_t)k * gp3 + g];
            }
      }
   }
}

void Tree::flatten(FlatTree& F) const {
   F = FlatTree();
   F.num_panels = (int)panels->size();
   F.num_points = (int)(points->size() / 3);
   F.depth = depth;
   F.grid = grid;
   // offsets first (serial, cheap), then every leaf's and cube's blocks copied in parallel
   std::vector<int> leaves, fcubes, flat_of(cubes.size(), -1);
   for (size_t i = 0; i < cubes.size(); i++) {
      const Cube& c = cubes[i];
      if (c.leaf && !c.points.empty() && !c.dcols.empty()) leaves.push_back((int)i);
      if (!c.inter.empty()) {
         flat_of[i] = (int)fcubes.size();
         fcubes.push_back((int)i);
      }
   }
   const int nl = (int)leaves.size(), nc = (int)fcubes.size();
   F.leaf_row_ptr.assign(nl + 1, 0);
   F.leaf_col_ptr.assign(nl + 1, 0);
   F.leaf_d_ptr.assign(nl + 1, 0);
   for (int l = 0; l < nl; l++) {
      const Cube& c = cubes[leaves[l]];
      F.leaf_row_ptr[l + 1] = F.leaf_row_ptr[l] + (int32_t)c.points.size();
      F.leaf_col_ptr[l + 1] = F.leaf_col_ptr[l] + (int32_t)c.dcols.size();
      F.leaf_d_ptr[l + 1] = F.leaf_d_ptr[l] + (int64_t)c.Ds.size();
   }
   F.leaf_rows.resize(F.leaf_row_ptr[nl]);
   F.leaf_cols.resize(F.leaf_col_ptr[nl]);
   F.d_single.resize(F.leaf_d_ptr[nl]);
   F.d_double.resize(F.leaf_d_ptr[nl]);
   F.cube_level.resize(nc);
   F.cube_index.resize(3 * (size_t)nc);
   F.cube_row_rank.resize(nc);
   F.cube_col_rank.resize(nc);
   for (auto* v : {&F.cube_panel_ptr, &F.cube_point_ptr, &F.inter_ptr}) v->assign(nc + 1, 0);
   for (auto* v : {&F.cube_vt_ptr, &F.cube_pv_ptr, &F.cube_uti_ptr, &F.cube_u_ptr}) v->assign(nc + 1, 0);
   for (int k = 0; k < nc; k++) {
      const Cube& c = cubes[fcubes[k]];
      F.cube_panel_ptr[k + 1] = F.cube_panel_ptr[k] + (int32_t)c.panels.size();
      F.cube_point_ptr[k + 1] = F.cube_point_ptr[k] + (int32_t)c.points.size();
      F.inter_ptr[k + 1] = F.inter_ptr[k] + (int32_t)c.inter.size();
      F.cube_vt_ptr[k + 1] = F.cube_vt_ptr[k] + (c.rowrank > 0 ? (int64_t)c.VT.size() : 0);
      F.cube_pv_ptr[k + 1] = F.cube_pv_ptr[k] + (c.rowrank > 0 ? (int64_t)c.PVs.size() : 0);
      F.cube_uti_ptr[k + 1] = F.cube_uti_ptr[k] + (c.colrank > 0 ? (int64_t)c.UTI.size() : 0);
      F.cube_u_ptr[k + 1] = F.cube_u_ptr[k] + (c.colrank > 0 ? (int64_t)c.U.size() : 0);
   }
   F.cube_panels.resize(F.cube_panel_ptr[nc]);
   F.cube_points.resize(F.cube_point_ptr[nc]);
   F.inter_cubes.resize(F.inter_ptr[nc]);
   F.vt.resize(F.cube_vt_ptr[nc]);
   F.pv_single.resize(F.cube_pv_ptr[nc]);
   F.pv_double.resize(F.cube_pv_ptr[nc]);
   F.uti.resize(F.cube_uti_ptr[nc]);
   F.u.resize(F.cube_u_ptr[nc]);
#pragma omp parallel
   {
#pragma omp for schedule(dynamic, 16) nowait
      for (int l = 0; l < nl; l++) {
         const Cube& c = cubes[leaves[l]];
         std::copy(c.points.begin(), c.points.end(), F.leaf_rows.begin() + F.leaf_row_ptr[l]);
         std::copy(c.dcols.begin(), c.dcols.end(), F.leaf_cols.begin() + F.leaf_col_ptr[l]);
         std::copy(c.Ds.begin(), c.Ds.end(), F.d_single.begin() + F.leaf_d_ptr[l]);
         std::copy(c.Dd.begin(), c.Dd.end(), F.d_double.begin() + F.leaf_d_ptr[l]);
      }
#pragma omp for schedule(dynamic, 16)
      for (int k = 0; k < nc; k++) {
         const Cube& c = cubes[fcubes[k]];
         F.cube_level[k] = c.level;
         for (int q = 0; q < 3; q++) F.cube_index[3 * (size_t)k + q] = c.idx[q];
         F.cube_row_rank[k] = c.rowrank;
         F.cube_col_rank[k] = c.colrank;
         std::copy(c.panels.begin(), c.panels.end(), F.cube_panels.begin() + F.cube_panel_ptr[k]);
         std::copy(c.points.begin(), c.points.end(), F.cube_points.begin() + F.cube_point_ptr[k]);
         for (size_t q = 0; q < c.inter.size(); q++) F.inter_cubes[F.inter_ptr[k] + q] = flat_of[c.inter[q]];
         if (c.rowrank > 0) {
            std::copy(c.VT.begin(), c.VT.end(), F.vt.begin() + F.cube_vt_ptr[k]);
            std::copy(c.PVs.begin(), c.PVs.end(), F.pv_single.begin() + F.cube_pv_ptr[k]);
            std::copy(c.PVd.begin(), c.PVd.end(), F.pv_double.begin() + F.cube_pv_ptr[k]);
         }
         if (c.colrank > 0) {
            std::copy(c.UTI.begin(), c.UTI.end(), F.uti.begin() + F.cube_uti_ptr[k]);
            std::copy(c.U.begin(), c.U.end(), F.u.begin() + F.cube_u_ptr[k]);
         }
      }
   }
   F.num_cubes = nc;
   int64_t off = 0;
   size_t t_total = 0;
   for (int d = 0; d < depth; d++) t_total += tops[d].size();
   F.t_ops.reserve(t_total);
   for (int d = 0; d < depth; d++) {
      F.t_level_ptr.push_back(off);
      off += (int64_t)tops[d].size() / 2;
      F.t_ops.insert(F.t_ops.end(), tops[d].begin(), tops[d].end());
   }
   F.t_level_ptr.push_back(off);
}

void FlatTree::view(fftsvd_tree_flat& t) const {
   std::memset(&t, 0, sizeof(t));
   t.num_panels = num_panels;
   t.num_points = num_points;
   t.depth = depth;
   for (int d = 0; d < depth && d < FFTSVD_MAX_DEPTH; d++) t.grid[d] = grid[d];
   t.num_leaves = (int32_t)leaf_row_ptr.size() - 1;
   t.leaf_row_ptr = leaf_row_ptr.data(); t.leaf_rows = leaf_rows.data();
   t.leaf_col_ptr = leaf_col_ptr.data(); t.leaf_cols = leaf_cols.data();
   t.leaf_d_ptr = leaf_d_ptr.data(); t.d_single = d_single.data(); t.d_double = d_double.data();
   t.num_cubes = num_cubes;
   t.cube_level = cube_level.data(); t.cube_index = cube_index.data();
   t.cube_panel_ptr = cube_panel_ptr.data(); t.cube_panels = cube_panels.data();
   t.cube_point_ptr = cube_point_ptr.data(); t.cube_points = cube_points.data();
   t.cube_row_rank = cube_row_rank.data(); t.cube_col_rank = cube_col_rank.data();
   t.cube_vt_ptr = cube_vt_ptr.data(); t.vt = vt.data();
   t.cube_pv_ptr = cube_pv_ptr.data(); t.pv_single = pv_single.data(); t.pv_double = pv_double.data();
   t.cube_uti_ptr = cube_uti_ptr.data(); t.uti = uti.data();
   t.cube_u_ptr = cube_u_ptr.data(); t.u = u.data();
   t.inter_ptr = inter_ptr.data(); t.inter_cubes = inter_cubes.data();
   t.t_level_ptr = t_level_ptr.data(); t.t_ops = t_ops.data();
}

BatchEvaluator host_evaluator() {
   auto store = std::make_shared<std::vector<double, FillLater<double>>>();
   return [store](const Kernel& k, const std::vector<FlatPanel>& pl, const IntegralBatch& B) -> const double* {
      store->resize((size_t)B.out_elems);  // every entry is written below
      double* out = store->data();
      const int64_t nb = (int64_t)B.blocks.size();
#pragma omp parallel for schedule(dynamic, 4)
      for (int64_t bi = 0; bi < nb; bi++) {
         const IntegralBlock& b = B.blocks[bi];
         for (int i = 0; i < b.npts; i++) {
            const double* p = &B.points[3 * (size_t)(b.pt_off + i)];
            for (int j = 0; j < b.npan; j++)
               k.panel(p, pl[B.panels[b.pan_off + j]], &out[b.out_s + (int64_t)i * b.ld_s + j],
                       &out[b.out_d + (int64_t)i * b.ld_d + j]);
         }
      }
      return out;
   };
}

Timings build_tree(Tree& T, int max_panels) {
   Timings tm;
   auto now = [] { return std::chrono::steady_clock::now(); };
   auto ms = [](auto a, auto b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
   auto t0 = now();
   T.choose_depth(max_panels);
   T.make_lists();
   auto t1 = now();
   T.fill_near();
   auto t2 = now();
   T.fill_pinv();
   T.fill_T();
   auto t3 = now();
   T.fill_bases();
   auto t4 = now();
   tm.partition_ms = ms(t0, t1);
   tm.near_ms = ms(t1, t2);
   tm.pinv_t_ms = ms(t2, t3);
   tm.bases_ms = ms(t3, t4);
   tm.integrals_ms = T.eval_ms;
   return tm;
}

void host_setup(const fftsvd_problem& pr, HostOperator& H, const BatchEvaluator* eval) {
   if (pr.num_panels <= 0 || !pr.vertices) throw std::invalid_argument("no panels");
   if (!(pr.eps_in > 0 && pr.eps_out > 0)) throw std::invalid_argument("dielectric constants must be positive");
   if (!(pr.kappa >= 0 && std::isfinite(pr.kappa))) throw std::invalid_argument("kappa must be non-negative");
   if (!(pr.svd_tol > 0 && pr.svd_tol < 1)) throw std::invalid_argument("svd_tol out of range");
   if (pr.max_panels_per_leaf <= 0) throw std::invalid_argument("max_panels_per_leaf must be positive");
   if (pr.grid_points != 4) throw std::invalid_argument("only the 4-point equivalent-density grid is supported");
   const int n = pr.num_panels;
   for (int64_t i = 0; i < 9LL * n; i++)
      if (!std::isfinite(pr.vertices[i])) throw std::invalid_argument("non-finite vertex");
   H.n = n;
   H.eps_in = pr.eps_in;
   H.eps_out = pr.eps_out;
   H.kappa = pr.kappa;
   const int saved_threads = omp_get_max_threads();
   if (pr.num_threads > 0) omp_set_num_threads(pr.num_threads);
   H.panels.resize(n);
   H.points.resize(3 * (size_t)n);
#pragma omp parallel for schedule(static)
   for (int i = 0; i < n; i++) {
      const double* v = pr.vertices + 9 * (size_t)i;
      make_flat_panel(H.panels[i], v, v + 3, v + 6);
   }
   for (int i = 0; i < n; i++) {
      if (!(H.panels[i].area > 0.0)) throw std::invalid_argument("degenerate panel " + std::to_string(i));
      for (int k = 0; k < 3; k++) H.points[3 * (size_t)i + k] = H.panels[i].centroid[k];
   }
   std::vector<double> ds(n, 0.0), dd(n, 0.0);
   for (int t = 0; t < 2; t++) {
      Tree T;
      T.panels = &H.panels;
      T.points = &H.points;
      T.eps = pr.svd_tol;
      T.grid_points = pr.grid_points;
      T.kernel.yukawa = (t == 0) && pr.kappa > 0.0;
      T.kernel.kappa = (t == 0) ? pr.kappa : 0.0;
      T.eval = eval;
      H.tm[t] = build_tree(T, pr.max_panels_per_leaf);
      H.depth[t] = T.depth;
      const auto f0 = std::chrono::steady_clock::now();
      T.flatten(H.flat[t]);
      H.tm[t].flatten_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - f0).count();
      if (t == 1)  // interior self terms for the preconditioner (Cube.c:2349-2390)
         for (const auto& c : T.cubes) {
            if (!c.leaf || c.points.empty() || c.dcols.empty()) continue;
            const size_t nc = c.dcols.size();
            for (size_t r = 0; r < c.points.size(); r++) {
               ds[c.points[r]] = c.Ds[r * nc + r];
               dd[c.points[r]] = c.Dd[r * nc + r];
            }
         }
   }
   if (pr.num_threads > 0) omp_set_num_threads(saved_threads);
   for (int t = 0; t < 2; t++) H.flat[t].view(H.views[t]);

   // region maps of the single-molecule operator (SurfaceOperator.c:51-158)
   H.idx_phi.resize(n);
   H.idx_dphi.resize(n);
   H.out_outer.resize(n);
   for (int k = 0; k < n; k++) {
      H.idx_phi[k] = k;
      H.idx_dphi[k] = n + k;
      H.out_outer[k] = n + k;
   }
   H.m1.assign(n, -1.0);
   H.ratio.assign(n, pr.eps_in / pr.eps_out);
   H.jump.assign(n, -4.0 * M_PI);
   H.one.assign(n, 1.0);
   H.zero.assign(n, 0.0);
   H.maps[0] = {H.idx_phi.data(), H.m1.data(), H.idx_dphi.data(), H.ratio.data(), H.out_outer.data(), H.jump.data()};
   H.maps[1] = {H.idx_phi.data(), H.one.data(), H.idx_dphi.data(), H.m1.data(), H.idx_phi.data(), H.zero.data()};

   // per-panel 2x2 preconditioner blocks (SurfaceOperator.c:170-197)
   const double rel = pr.eps_in / pr.eps_out;
   H.col_ptr.resize(2 * (size_t)n + 1);
   H.rows.resize(4 * (size_t)n);
   H.vals.resize(4 * (size_t)n);
   for (int c = 0; c <= 2 * n; c++) H.col_ptr[c] = 2 * c;
   for (int i = 0; i < n; i++) {
      H.rows[2 * i] = i;
      H.vals[2 * i] = dd[i];
      H.rows[2 * i + 1] = n + i;
      H.vals[2 * i + 1] = dd[i];
      H.rows[2 * (n + i)] = i;
      H.vals[2 * (n + i)] = -ds[i];
      H.rows[2 * (n + i) + 1] = n + i;
      H.vals[2 * (n + i) + 1] = rel * ds[i];
   }
   H.precond = {2 * n, H.col_ptr.data(), H.rows.data(), H.vals.data()};
}

}  // namespace setup
}  // namespace fftsvd

// ---- host-only C entry points (no GPU needed)

namespace fftsvd {
void set_last_error(const std::string& msg);
}

struct fftsvd_host_operator {
   fftsvd::setup::HostOperator h;
};

extern "C" int fftsvd_b200_host_setup(const fftsvd_problem* problem, fftsvd_host_operator** out) {
   if (!problem || !out) return FFTSVD_ERR_ARGUMENT;
   *out = nullptr;
   auto* op = new (std::nothrow) fftsvd_host_operator();
   if (!op) return FFTSVD_ERR_ARGUMENT;
   try {
      fftsvd::setup::host_setup(*problem, op->h);
   } catch (const std::exception& e) {
      fftsvd::set_last_error(e.what());
      delete op;
      return FFTSVD_ERR_ARGUMENT;
   }
   *out = op;
   return FFTSVD_OK;
}

extern "C" int fftsvd_b200_host_setup_batched(const fftsvd_problem* problem, fftsvd_host_operator** out) {
   if (!problem || !out) return FFTSVD_ERR_ARGUMENT;
   *out = nullptr;
   auto* op = new (std::nothrow) fftsvd_host_operator();
   if (!op) return FFTSVD_ERR_ARGUMENT;
   try {
      const fftsvd::setup::BatchEvaluator eval = fftsvd::setup::host_evaluator();
      fftsvd::setup::host_setup(*problem, op->h, &eval);
   } catch (const std::exception& e) {
      fftsvd::set_last_error(e.what());
      delete op;
      return FFTSVD_ERR_ARGUMENT;
   }
   *out = op;
   return FFTSVD_OK;
}

extern "C" int fftsvd_b200_device_setup(const fftsvd_problem* problem, fftsvd_host_operator** out) {
   if (!problem || !out) return FFTSVD_ERR_ARGUMENT;
   *out = nullptr;
   auto* op = new (std::nothrow) fftsvd_host_operator();
   if (!op) return FFTSVD_ERR_ARGUMENT;
   try {
      const fftsvd::setup::BatchEvaluator eval = fftsvd::setup::device_evaluator();
      fftsvd::setup::host_setup(*problem, op->h, &eval);
   } catch (const fftsvd::setup::DeviceError& e) {
      fftsvd::set_last_error(e.what());
      delete op;
      return e.code;
   } catch (const std::exception& e) {
      fftsvd::set_last_error(e.what());
      delete op;
      return FFTSVD_ERR_ARGUMENT;
   }
   *out = op;
   return FFTSVD_OK;
}

extern "C" int fftsvd_b200_host_operator_tree(const fftsvd_host_operator* op, int32_t tree, fftsvd_tree_flat* view) {
   if (!op || !view || tree < 0 || tree > 1) return FFTSVD_ERR_ARGUMENT;
   *view = op->h.views[tree];
   return FFTSVD_OK;
}

extern "C" int fftsvd_b200_host_operator_precond(const fftsvd_host_operator* op, fftsvd_precond_csc* out) {
   if (!op || !out) return FFTSVD_ERR_ARGUMENT;
   *out = op->h.precond;
   return FFTSVD_OK;
}

extern "C" int fftsvd_b200_host_operator_timings(const fftsvd_host_operator* op, double* ms6) {
   if (!op || !ms6) return FFTSVD_ERR_ARGUMENT;
   const fftsvd::setup::Timings* t = op->h.tm;
   ms6[0] = t[0].partition_ms + t[1].partition_ms;
   ms6[1] = t[0].near_ms + t[1].near_ms;
   ms6[2] = t[0].pinv_t_ms + t[1].pinv_t_ms;
   ms6[3] = t[0].bases_ms + t[1].bases_ms;
   ms6[4] = t[0].flatten_ms + t[1].flatten_ms;
   ms6[5] = t[0].integrals_ms + t[1].integrals_ms;
   return FFTSVD_OK;
}

extern "C" void fftsvd_b200_host_operator_free(fftsvd_host_operator* op) { delete op; }

namespace fftsvd {
namespace setup {

}  // namespace setup
}  // namespace fftsvd
