// Tile-shape autotuner: the translation tiles of a surface's operators are rebuilt
// under a few candidate limits, the concurrent matvec of each precision is timed with
// each, and the fastest stays.  Tile limits change launch shapes only (the member
// groups and the order of every sum are fixed before tiling), so the tuned operator
// gives bit-for-bit the results of the untuned one.
#include <algorithm>
#include <vector>

#include "surface.h"

namespace fftsvd {

namespace {

// candidate limits {member groups, halo sources, entries}; the first is the default
const TileLimits kCandidates[] = {
    {32, 320, 3072}, {32, 256, 2048}, {24, 256, 2304}, {16, 192, 1536}, {8, 128, 768},
};
constexpr int kNumCandidates = (int)(sizeof(kCandidates) / sizeof(kCandidates[0]));
static_assert(kNumCandidates <= FFTSVD_TUNE_MAX_CANDIDATES, "too many tile candidates");

constexpr int kWarmReps = 3, kTimedReps = 10;

template <typename T>
double time_matvec(DeviceOperator<T>& op, const double* x, double* y, cudaStream_t s) {
   for (int r = 0; r < kWarmReps; r++) op.apply(x, y, s);
   cudaEvent_t e[2];
   for (auto& ev : e) FFTSVD_CUDA(cudaEventCreate(&ev));
   float ms = 0.f;
   try {
      FFTSVD_CUDA(cudaEventRecord(e[0], s));
      for (int r = 0; r < kTimedReps; r++) op.apply(x, y, s);
      FFTSVD_CUDA(cudaEventRecord(e[1], s));
      FFTSVD_CUDA(cudaEventSynchronize(e[1]));
      FFTSVD_CUDA(cudaEventElapsedTime(&ms, e[0], e[1]));
   } catch (...) {
      for (auto& ev : e) cudaEventDestroy(ev);
      throw;
   }
   for (auto& ev : e) cudaEventDestroy(ev);
   return (double)ms / kTimedReps;
}

template <typename T>
int tune_one(DeviceOperator<T>& op, const std::vector<TileSet>& fwd, const std::vector<TileSet>& adj,
             const double* x, double* y, cudaStream_t s, double* ms) {
   int best = 0;
   for (int c = 0; c < kNumCandidates; c++) {
      op.set_tiles(fwd[c], adj[c]);
      ms[c] = time_matvec(op, x, y, s);
      if (ms[c] < ms[best]) best = c;
   }
   op.set_tiles(fwd[best], adj[best]);
   return best;
}

}  // namespace

void Surface::set_tile_limits(int max_groups, int max_src, int max_entries) {
   FFTSVD_REQUIRE(tile_problems != nullptr, "surface without translation problems");
   TileLimits lim;
   lim.max_groups = max_groups;
   lim.max_src = max_src;
   lim.max_entries = max_entries;
   TileSet fwd, adj;
   make_tiles(*tile_problems, lim, fwd, adj);
   release_step_graphs();  // they hold the old tiles' buffers
   op32.set_tiles(fwd, adj);
   op64.set_tiles(fwd, adj);
}

void Surface::autotune(fftsvd_tune_info* info) {
   FFTSVD_REQUIRE(tile_problems != nullptr, "surface without translation problems");
   release_step_graphs();  // they hold the current tiles' buffers
   std::vector<TileSet> fwd(kNumCandidates), adj(kNumCandidates);
   for (int c = 0; c < kNumCandidates; c++) make_tiles(*tile_problems, kCandidates[c], fwd[c], adj[c]);
   // timing input: zeros (the kernels' speed does not depend on the values)
   FFTSVD_CUDA(cudaMemsetAsync(t0.get(), 0, sizeof(double) * n, stream));
   double ms[2][FFTSVD_TUNE_MAX_CANDIDATES] = {};
   const int best32 = tune_one(op32, fwd, adj, t0.get(), t1.get(), stream, ms[0]);
   const int best64 = tune_one(op64, fwd, adj, t0.get(), t1.get(), stream, ms[1]);
   if (info) {
      *info = fftsvd_tune_info{};
      info->candidates = kNumCandidates;
      info->chosen[0] = best32;
      info->chosen[1] = best64;
      for (int c = 0; c < kNumCandidates; c++) {
         info->max_groups[c] = kCandidates[c].max_groups;
         info->max_src[c] = kCandidates[c].max_src;
         info->max_entries[c] = kCandidates[c].max_entries;
         info->matvec_ms[0][c] = ms[0][c];
         info->matvec_ms[1][c] = ms[1][c];
      }
   }
}

}  // namespace fftsvd

using namespace fftsvd;

namespace {
// Runs f with the surface's device current, restoring the caller's device afterwards.
template <typename F>
int on_device(fftsvd_surface* s, F&& f) {
   return guarded([&] {
      int previous = -1;
      FFTSVD_CUDA(cudaGetDevice(&previous));
      if (previous != s->s.device) FFTSVD_CUDA(cudaSetDevice(s->s.device));
      try {
         f();
      } catch (...) {
         if (previous != s->s.device) cudaSetDevice(previous);
         throw;
      }
      if (previous != s->s.device) FFTSVD_CUDA(cudaSetDevice(previous));
   });
}
}  // namespace

extern "C" int fftsvd_b200_surface_autotune(fftsvd_surface* s, fftsvd_tune_info* info) {
   if (!s) return FFTSVD_ERR_ARGUMENT;
   return on_device(s, [&] { s->s.autotune(info); });
}

extern "C" int fftsvd_b200_surface_set_tile_limits(fftsvd_surface* s, int32_t max_groups, int32_t max_src,
                                                   int32_t max_entries) {
   if (!s) return FFTSVD_ERR_ARGUMENT;
   return on_device(s, [&] { s->s.set_tile_limits(max_groups, max_src, max_entries); });
}
