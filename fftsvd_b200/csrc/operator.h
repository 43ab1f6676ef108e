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
#include <memory>
#include <utility>
#include <vector>

#include "common.h"
#include "fill_later.h"

namespace fftsvd {

struct SrcDesc {        // one far-field source cube (panels > 0, row rank > 0)
   int32_t n;           // grid edge of its level
   int32_t m;           // panels
   int32_t r;           // row rank
   int32_t panel_off;   // into src_panels (global tree-panel indices)
   int64_t vt_off;      // into vt, r x m row-major
   int64_t pv_off;      // into pv, r x n^3 of {PV_single, PV_double}
   int64_t spec_off;    // into spectra, (2n-1)^2 n complex
   int32_t level;       // staging slot of the transposed operator
   int32_t pad;
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
   int64_t s_off;       // into the translated spectra, (2n-1)^2 n complex
};

// Translation tile: sibling destination cubes (outputs) of one tree and level, in
// member groups of up to kGroupMax siblings, that share a halo of source spectra.
// The halo and the level's 343 translation slots are staged through shared memory
// one frequency chunk at a time.  A group's sources are listed once (the union of
// its members' interaction lists); one entry carries the halo row, the mask of the
// members that interact with that source and a base slot.  The slot of member j is
// base + delta_j, because a slot is a linear function of the offset between the two
// cubes (slot = ((dx+3)*7 + (dy+3))*7 + dz+3 for output minus input).
struct TileDesc {
   int32_t ngroups;     // member groups (one thread row each)
   int32_t nsrc;        // halo sources
   int32_t nentries;    // (group, source) entries, each group's list padded to a multiple of four
   int32_t nmembers;    // outputs in the tile
   int32_t pg;          // frequencies per cube, (2n-1)^2 n padded to 16
   int32_t pad;
   int64_t grp_off;     // into tile_grp
   int64_t mem_off;     // into tile_dst and tile_delta
   int64_t src_off;     // into tile_src (spectrum offsets)
   int64_t ent_off;     // into tile_entries
   int64_t t_off;       // translation table of slot 0 of this tree and level (complex elements)
};

struct TileGroup {      // tiles with the same frequency count, one launch
   int pg = 0;
   int begin = 0, count = 0;
   int max_src = 0, max_entries = 0, max_groups = 0, max_members = 0;
};

// Entry word: bits 0-8 base slot + kEntryBaseBias, bits 9-16 member mask, bits 17-31 halo row.
constexpr int kEntryBaseBias = 64;
constexpr int kGroupMax = 8;

// Tiles of one translation direction, as uploaded.
struct TileSet {
   std::vector<TileDesc> tiles;
   std::vector<int64_t> tile_src, tile_dst;
   std::vector<int32_t> tile_delta;    // per member: slot of the member = entry base + delta
   std::vector<int4> tile_grp;         // per group: {entry begin, entry count, member begin, member count},
                                       // relative to the tile's ent_off and mem_off
   std::vector<uint32_t> tile_entries;
   std::vector<TileGroup> tile_groups;
};

// One translation problem before tiling: each output (destination spectrum) with its tree
// and level key, Morton code, slot-0 table offset, padded frequency count, and its
// interactions (input spectrum offset, table slot) in in_off/slot[ptr[o] .. ptr[o+1]).
struct TileProblem {
   std::vector<int> key;
   std::vector<uint64_t> morton;
   std::vector<int64_t> t_base;
   std::vector<int> pg;
   std::vector<int64_t> out_off;
   std::vector<int64_t> ptr{0};
   std::vector<int64_t> in_off;
   std::vector<int> slot;
   void add_output(int key, uint64_t morton, int64_t t_base, int pg, int64_t out);
   void add_pair(int64_t in, int slot);
};

constexpr int kTileMaxGroups = 32;   // thread rows per block
constexpr int kTileMaxSrc = 320;
constexpr int kTileMaxEntries = 3072;

// Limits of one translation tile (at most the kernel's bounds above).  Smaller tiles
// give more blocks and less shared memory per block, larger ones stage each table
// chunk for more destinations.
struct TileLimits {
   int max_groups = kTileMaxGroups;
   int max_src = kTileMaxSrc;
   int max_entries = kTileMaxEntries;
};

// Both translation problems of an operator with the buffer sizes their indices are
// checked against, kept so that the tiles can be rebuilt with other limits.
struct TileProblems {
   TileProblem fwd, adj;
   int64_t nt = 0, spectra_elems = 0, translated_elems = 0;
};

// Tiles of both directions under the given limits, range-checked.
void make_tiles(const TileProblems& P, const TileLimits& lim, TileSet& fwd, TileSet& adj);

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
   int max_rank = 0;    // largest row (sources) or column (destinations) rank
   int64_t units = 0;   // panels (sources) or points (destinations) of all the group's cubes
   // shared memory of a block that serves several right-hand sides: batch_shared +
   // right-hand sides x batch_per_rhs elements
   int batch_shared = 0, batch_per_rhs = 0;
};

// Per-right-hand-side strides of the planar batch buffers: right-hand side r of a
// batched launch reads and writes base + r * stride.  Per-cube and per-leaf
// kernels take r = blockIdx.x % nrhs and their unit blockIdx.x / nrhs, so the
// blocks of one cube for all right-hand sides run together and its operator
// data is fetched from DRAM once; the join and far-field add take r = blockIdx.y
// and the translation group blockIdx.z of kBatchGroup.  Strides zero and nrhs 1
// for a single vector.
struct BatchStrides {
   int nrhs = 1;
   int64_t n = 0;           // x, y (FP64 unknowns)
   int64_t panels = 0;      // joined panel values
   int64_t spectra = 0;     // source spectra (complex)
   int64_t translated = 0;  // translated spectra (complex)
   int64_t staging = 0;     // far-field staging rows
};
constexpr int kBatchGroup = 8;   // right-hand sides per batched translation row
constexpr int kMaxBatch = 65535; // grid y limit

// Small grids (n <= kWarpMaxN) whose cubes all have rank <= 32 run one cube per
// warp instead of one cube per block.
constexpr int kWarpMinN = 3;
constexpr int kWarpMaxN = 5;
constexpr int kWarpMaxRank = 32;
constexpr int kWarpMinCubes = 2000;  // fewer cubes leave too few warps per SM to hide latency
// A warp per cube walks the cube's panels 32 at a time; with many panels per cube a block per
// cube spreads them over more threads (B200: the 5^3 grid with 75 panels per cube ran the
// single solve 1.2 % and the 256-column block solve 4 % faster on warps; with 284 panels
// per cube the single solve ran 1.3 % slower).
constexpr int kWarpMaxMeanUnits = 160;

// Algorithmic bytes of each matvec kernel [join, far_forward, translate, far_backward, near]:
// elems * (operator element size) + fixed (FP64 vectors and int32 indices).
constexpr int kNumKernels = 5;
struct KernelBytes {
   double elems[kNumKernels] = {0, 0, 0, 0, 0};
   double fixed[kNumKernels] = {0, 0, 0, 0, 0};
};

using LayoutDoubles = std::vector<double, FillLater<double>>;

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
   LayoutDoubles d_pairs;              // interleaved {Ds, Dd}
   // far field
   std::vector<SrcDesc> src;
   std::vector<int32_t> src_panels;
   LayoutDoubles vt;
   LayoutDoubles pv_pairs;             // interleaved {PVs, PVd}, r x n^3
   std::vector<DstDesc> dst;
   std::vector<int32_t> dst_points;
   LayoutDoubles uti, u_cm;
   std::vector<int64_t> inter_pairs;   // {spectrum offset, T offset} packed as 2 x int64
   LayoutDoubles t_pairs;              // translation operators {re, im}
   int64_t spectra_elems = 0;
   int64_t translated_elems = 0;       // S buffer, complex elements
   int max_src_smem_elems = 0, max_dst_smem_elems = 0;
   std::vector<LaunchGroup> src_groups, dst_groups;
   // translation tiles, grouped by frequency count (one launch per group): the operator's
   // (spectra -> translated) and the transposed operator's (translated -> spectra)
   TileSet fwd, adj;
   std::shared_ptr<TileProblems> problems;
   // algorithmic bytes per matvec at 4-byte or 8-byte element size (excluding vectors)
   int64_t operator_elems = 0;          // D pairs*2 + VT + PV*2 + UTI + U
   int64_t t_elems = 0;                 // unique translation operator reals
   KernelBytes kernel_bytes;
};

OperatorLayout build_layout(int num_unknowns, int num_trees, const fftsvd_tree_flat* trees,
                            const fftsvd_region_map* maps);

// Near field of a multi-vector FP32 matvec on the tensor cores (near_tc.cu): the joined
// panel values are transposed to [panel][rhs] (xsd_t, ld >= nrhs) and each leaf's block
// product runs as kind::tf32 MMAs with three-product splitting, 128 right-hand sides per
// CTA.  np_max: the largest leaf row count padded to 8 (at most 256).  A bounded wait that
// gives up sets *status.
int near_tc_smem(int np_max);
// Runs one wait on an mbarrier that nothing arrives at, bounded by `polls` polls, as the
// tensor-core kernels bound theirs: 1 when the wait gave up (the expected result), 2 when
// it completed.  Synchronous.
int bounded_wait_selftest(int polls);
void prepare_near_tc(int np_max);
void launch_near_tc(const LeafDesc* leaves, int n_leaf, const int32_t* rows, const int32_t* cols, const float2* d,
                    const float2* xsd, int64_t panels, int np_panels, float2* xsd_t, int64_t ld,
                    const int32_t* point_out, const int32_t* point_panel, const double* point_jump,
                    const int32_t* phi_idx, const double* phi_scale, const double* x, double* y, int nrhs, int64_t ldn,
                    int np_max, int* status, cudaStream_t stream);

template <typename T>
class DeviceOperator {
 public:
   using T2 = typename Vec2<T>::type;
   DeviceOperator() = default;
   DeviceOperator(const DeviceOperator&) = delete;
   DeviceOperator& operator=(const DeviceOperator&) = delete;
   ~DeviceOperator();
   void upload(const OperatorLayout& L);
   // y = A x on `stream`; x, y device pointers of num_unknowns doubles.
   void apply(const double* x, double* y, cudaStream_t stream);
   // Y = A X for nrhs right-hand sides (a multiple of kBatchGroup, at most kMaxBatch),
   // X and Y column-major (right-hand side r at x + r * num_unknowns).  Every column
   // goes through the same arithmetic as apply(); the batch buffers grow on demand.
   void apply_batch(const double* x, double* y, int nrhs, cudaStream_t stream);
   // device bytes of the batch buffers per right-hand side
   size_t batch_bytes_per_rhs() const;
   // Replace the translation tiles (the same problems under other limits, make_tiles):
   // results are unchanged bit for bit, only the launch shapes differ.  Synchronises.
   void set_tiles(const TileSet& fwd, const TileSet& adj);
   // y = A^T x (the transposed operator), x and y device vectors of num_unknowns doubles.
   // Column sums are accumulated with FP64 atomics: not bitwise reproducible run to run.
   void apply_transpose(const double* x, double* y, cudaStream_t stream);
   // Multi-vector FP32 matvecs take the tensor-core near field (near_tc.cu) while this is
   // set; the columns then differ from single matvecs at FP32 rounding level (the block
   // solve sets it; the lockstep batch keeps the single-matvec arithmetic).
   void set_tensor_near(bool on) { tensor_near_ = on; }
   bool tensor_near_available() const { return near_np_max_ > 0; }
   // Shared-memory bytes one single-vector translation moves (staged rows written, source
   // and table rows read): the translation's bound is the SMs' shared-memory bandwidth.
   double translate_smem_bytes() const;
   // nonzero when a tensor-core near-field wait gave up since the last reset
   int tensor_status(bool reset);
   // per-stage events for timing (recorded when enabled)
   void enable_timing(bool on);
   // milliseconds of [join, far_forward, translate, far_backward, near] of the last timed apply
   void stage_ms(float* ms) const;
   size_t device_bytes() const;

 private:
   // launch groups of one grid size: forward, translate and backward depend only on
   // each other, so the chains of different grid sizes run concurrently
   struct Chain {
      int n = 0;
      double work = 0;
      std::vector<int> src, tile, dst;  // indices into the launch groups
      cudaStream_t stream = nullptr;    // own stream (the first, longest chain at high priority)
      cudaEvent_t done = nullptr;
   };
   // intermediate buffers of one apply: the single-vector members or the planar batch
   struct Bufs {
      T2* xsd = nullptr;
      T2* spectra = nullptr;
      T2* translated = nullptr;
      T* staging = nullptr;
      int nrhs = 1;
      BatchStrides bs;
   };
   int translate_smem(const TileGroup& g, bool batch) const;
   void raise_translate_smem(int optin);
   void apply_bufs(const double* x, double* y, const Bufs& b, cudaStream_t stream);
   void launch_forward(const LaunchGroup& g, const Bufs& b, cudaStream_t stream);
   void launch_translate(const TileGroup& g, const Bufs& b, cudaStream_t stream);
   void launch_backward(const LaunchGroup& g, const Bufs& b, cudaStream_t stream);
   void launch_chain(const Chain& ch, const Bufs& b, cudaStream_t stream);
   void launch_near(const double* x, double* y, const Bufs& b, cudaStream_t stream);
   bool warp_path(const LaunchGroup& g) const;
   int warp_min_cubes_ = kWarpMinCubes;
   // resident warps of one wave of the 4^3 forward/backward and the near-field launches:
   // how far ahead their warps prefetch operator blocks into L2
   int64_t fwd_n4_wave_ = 0, bwd_n4_wave_ = 0, near_wave_ = 0;
   bool tensor_near_ = false;
   int near_np_max_ = 0;               // 0: some leaf has more than 256 rows (no tensor path)
   DevBuf<float2> xsd_t_;              // joined values [panel][rhs] of the tensor-core near field
   int64_t xsd_t_ld_ = 0;
   DevBuf<int> tc_status_;
   struct Prefetch prefetch(int64_t wave, int nrhs, int64_t a_bytes, int64_t b_bytes, int64_t c_bytes) const;
   int sm_count_ = 148;
   int smem_optin_ = 0;  // largest dynamic shared memory a block may opt into
   int64_t spectra_elems_ = 1, translated_elems_ = 1;
   int batch_capacity_ = 0;
   DevBuf<T2> xsd_b_, spectra_b_, translated_b_;
   DevBuf<T> staging_b_;
   void build_chains();
   void release_chains();
   std::vector<Chain> chains_;
   cudaEvent_t fork_ = nullptr;
   cudaStream_t near_stream_ = nullptr;
   cudaEvent_t near_done_ = nullptr;
   int64_t n_rows_ = 0;  // leaf rows (one per written output row)
   int num_unknowns_ = 0;
   int64_t total_panels_ = 0, total_points_ = 0;
   int stage_levels_ = 0;
   bool full_cover_ = true;
   int n_src_ = 0, n_dst_ = 0, n_leaf_ = 0;
   int src_smem_ = 0, dst_smem_ = 0, leaf_smem_max_ = 0;
   int near_warps_ = 1, near_stride_ = 2;
   std::vector<LaunchGroup> src_groups_, dst_groups_;
   // device copy of one direction's tiles
   struct DevTiles {
      DevBuf<TileDesc> tiles;
      DevBuf<int64_t> src, dst;
      DevBuf<int32_t> delta;
      DevBuf<int4> grp;
      DevBuf<uint32_t> entries;
      std::vector<TileGroup> groups;
      double smem_bytes = 0.0;  // shared-memory traffic of one single-vector translation
      void upload(const TileSet& S);
   };
   DevTiles fwd_, adj_;
   void launch_translate_tiles(const DevTiles& tl, const TileGroup& g, const T2* in, T2* out, int nrhs,
                               const BatchStrides& bs, cudaStream_t stream);
   // transposed operator: gathered input, per-panel near-field sums, per-level far-field rows
   DevBuf<T> zt_;
   DevBuf<double2> ut_;
   DevBuf<typename Vec2<T>::type> staget_;
   DevBuf<double> panel_jump_;
   DevBuf<int32_t> panel_point_;
   int src_smem_t_ = 0, dst_smem_t_ = 0;
   DevBuf<typename Vec2<T>::type> translated_;
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
   DevBuf<T2> t_;
   DevBuf<T2> spectra_;
   DevBuf<T> staging_;
   bool timing_ = false;
   cudaEvent_t ev_[kNumKernels + 1] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
};

}  // namespace fftsvd
