// Device-resident FFTSVD operator for all region trees of one surface, in a
// layout chosen for the four matvec kernels (see operator.cu):
//
//   join          x (FP64, global unknowns) -> per tree panel {xs, xd} in T
//   far_forward   per source cube: VT x, PV (.), zero-padded r2c DFT -> spectrum
//   far_backward  per destination cube: sum_T T[offset] * spectrum, c2r DFT,
//                 UTI (.), U (.) -> per-level staging rows
//   near          per leaf: D_single xs + D_double xd + staged far field + jump
//                 -> y (FP64), one exclusive writer per row
//
// T is float (the reference's as-shipped FP32 operator storage) or double.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "common.h"

namespace fftsvd {

struct SrcDesc {        // one far-field source cube (panels > 0, row rank > 0)
   int32_t n;           // grid edge of its level
   int32_t m;           // panels
   int32_t r;           // row rank
   int32_t panel_off;   // into src_panels (global tree-panel indices)
   int64_t vt_off;      // into vt, r x m row-major
   int64_t pv_off;      // into pv, r x n^3 of {PV_single, PV_double}
   int64_t spec_off;    // into spectra, (2n-1)^2 n complex
};

struct DstDesc {        // one far-field destination cube (points > 0, column rank > 0)
   int32_t n;
   int32_t p;           // points
   int32_t r;           // column rank
   int32_t point_off;   // into dst_points (global tree-point indices)
   int64_t uti_off;     // into uti, r x n^3 row-major
   int64_t u_off;       // into u, r x p (column-major copy of Udest)
   int32_t inter_off;   // into inter pairs
   int32_t inter_cnt;
   int32_t stage;       // staging slot (level)
   int32_t pad;
};

struct LeafDesc {       // one leaf with points
   int32_t row_off;     // into leaf_rows
   int32_t nrows;
   int32_t col_off;     // into leaf_cols
   int32_t ncols;       // padded to a multiple of 2
   int64_t d_off;       // into d (element pairs), nrows x ncols
};

// A contiguous range of source or destination cubes of one grid size, launched
// together with shared memory sized for that range.
struct LaunchGroup {
   int n = 0;
   int begin = 0;
   int count = 0;
   int smem_elems = 0;  // in units of the operator element type
};

// Algorithmic bytes of each matvec kernel [join, far_forward, far_backward, near]:
// elems * (operator element size) + fixed (FP64 vectors and int32 indices).
struct KernelBytes {
   double elems[4] = {0, 0, 0, 0};
   double fixed[4] = {0, 0, 0, 0};
};

// Host-side relayout product, independent of the element type.
struct OperatorLayout {
   int num_unknowns = 0;
   int num_trees = 0;
   int64_t total_panels = 0;   // sum over trees (+1 zero slot used by padding columns)
   int64_t total_points = 0;
   int stage_levels = 0;
   bool full_cover = true;     // every unknown row is written by some leaf row
   std::vector<int64_t> tree_panel_off, tree_point_off;
   // join
   std::vector<int32_t> join_phi_idx, join_dphi_idx;
   std::vector<double> join_phi_scale, join_dphi_scale;
   // per tree point
   std::vector<int32_t> point_out, point_panel;
   std::vector<double> point_jump;
   // near field
   std::vector<LeafDesc> leaves;
   std::vector<int32_t> leaf_rows, leaf_cols;
   std::vector<double> d_pairs;        // interleaved {Ds, Dd}
   // far field
   std::vector<SrcDesc> src;
   std::vector<int32_t> src_panels;
   std::vector<double> vt;
   std::vector<double> pv_pairs;       // interleaved {PVs, PVd}, r x n^3
   std::vector<DstDesc> dst;
   std::vector<int32_t> dst_points;
   std::vector<double> uti, u_cm;
   std::vector<int64_t> inter_pairs;   // {spectrum offset, T offset} packed as 2 x int64
   std::vector<double> t_pairs;        // translation operators {re, im}
   int64_t spectra_elems = 0;
   int max_src_smem_elems = 0, max_dst_smem_elems = 0;
   std::vector<LaunchGroup> src_groups, dst_groups;
   // algorithmic bytes per matvec at 4-byte or 8-byte element size (excluding vectors)
   int64_t operator_elems = 0;          // D pairs*2 + VT + PV*2 + UTI + U
   int64_t t_elems = 0;                 // unique translation operator reals
   KernelBytes kernel_bytes;
};

OperatorLayout build_layout(int num_unknowns, int num_trees, const fftsvd_tree_flat* trees,
                            const fftsvd_region_map* maps);

template <typename T>
class DeviceOperator {
 public:
   using T2 = typename Vec2<T>::type;
   void upload(const OperatorLayout& L);
   // y = A x on `stream`; x, y device pointers of num_unknowns doubles.
   void apply(const double* x, double* y, cudaStream_t stream);
   // per-stage events for timing (recorded when enabled)
   void enable_timing(bool on);
   void stage_ms(float* join_ms, float* fwd_ms, float* bwd_ms, float* near_ms) const;
   size_t device_bytes() const;

 private:
   int num_unknowns_ = 0;
   int64_t total_panels_ = 0, total_points_ = 0;
   int stage_levels_ = 0;
   bool full_cover_ = true;
   int n_src_ = 0, n_dst_ = 0, n_leaf_ = 0;
   int src_smem_ = 0, dst_smem_ = 0, leaf_smem_max_ = 0;
   std::vector<LaunchGroup> src_groups_, dst_groups_;
   DevBuf<int32_t> join_phi_idx_, join_dphi_idx_;
   DevBuf<double> join_phi_scale_, join_dphi_scale_;
   DevBuf<T2> xsd_;
   DevBuf<int32_t> point_out_, point_panel_;
   DevBuf<double> point_jump_;
   DevBuf<LeafDesc> leaves_;
   DevBuf<int32_t> leaf_rows_, leaf_cols_;
   DevBuf<T2> d_;
   DevBuf<SrcDesc> src_;
   DevBuf<int32_t> src_panels_;
   DevBuf<T> vt_;
   DevBuf<T2> pv_;
   DevBuf<DstDesc> dst_;
   DevBuf<int32_t> dst_points_;
   DevBuf<T> uti_, u_;
   DevBuf<longlong2> inter_;
   DevBuf<T2> t_;
   DevBuf<T2> spectra_;
   DevBuf<T> staging_;
   bool timing_ = false;
   cudaEvent_t ev_[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
};

}  // namespace fftsvd
