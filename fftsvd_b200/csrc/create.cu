// fftsvd_b200_surface_create: the library's own replacement for the reference
// operator construction of the single-molecule PBE problem
// (generateSurfaceOperator + Tree_fill + generateSurfaceOperatorPreconditioner,
// FFTSVDpbeAPI.c:1053-1739, 1853-1861): setup (setup.cpp) with its panel integrals
// on the device (sampling.cu), then upload.
#include <chrono>
#include <cmath>
#include <vector>

#include "nbody.h"
#include "setup.h"
#include "surface.h"

using namespace fftsvd;

extern "C" int fftsvd_b200_surface_create(const fftsvd_problem* pr, fftsvd_surface** out) {
   if (!out || !pr) return FFTSVD_ERR_ARGUMENT;
   *out = nullptr;
   fftsvd_surface* s = new (std::nothrow) fftsvd_surface();
   if (!s) return FFTSVD_ERR_ARGUMENT;
   const auto c0 = std::chrono::steady_clock::now();
   auto ms_since = [](std::chrono::steady_clock::time_point t) {
      return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
   };
   try {
      int ndev = 0;
      if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw Error(FFTSVD_ERR_NO_DEVICE, "no CUDA device visible");
      setup::HostOperator H;
      try {
         const setup::BatchEvaluator eval = setup::device_evaluator();
         setup::host_setup(*pr, H, &eval);
      } catch (const std::invalid_argument& e) {
         throw Error(FFTSVD_ERR_ARGUMENT, e.what());
      } catch (const setup::DeviceError& e) {
         throw Error(e.code, e.what());
      }
      Surface& S = s->s;
      const auto u0 = std::chrono::steady_clock::now();
      init_surface(S, 2 * H.n, 2, H.views, H.maps, &H.precond);
      S.stats.setup_ms[6] = ms_since(u0);
      S.eps_in = pr->eps_in;
      std::vector<int32_t> dphi_rows(H.n);
      for (int i = 0; i < H.n; i++) dphi_rows[i] = H.n + i;
      set_geometry(S, H.n, pr->vertices, H.idx_phi.data(), dphi_rows.data());
      set_charges(S, pr->num_charges, pr->charge_pos, pr->charge);
      for (int t = 0; t < 2; t++) {
         S.stats.depth[t] = H.depth[t];
         S.stats.num_leaves[t] = H.views[t].num_leaves;
         S.stats.num_cubes[t] = H.views[t].num_cubes;
      }
      S.stats.setup_ms[0] = H.tm[0].partition_ms + H.tm[1].partition_ms;
      S.stats.setup_ms[1] = H.tm[0].near_ms + H.tm[1].near_ms;
      S.stats.setup_ms[2] = H.tm[0].pinv_t_ms + H.tm[1].pinv_t_ms;
      S.stats.setup_ms[3] = H.tm[0].bases_ms + H.tm[1].bases_ms;
      S.stats.setup_ms[4] = H.tm[0].flatten_ms + H.tm[1].flatten_ms;
      S.stats.setup_ms[5] = H.tm[0].integrals_ms + H.tm[1].integrals_ms;
      S.stats.setup_ms[7] = ms_since(c0);
   } catch (const Error& e) {
      set_last_error(e.what());
      delete s;
      return e.code;
   } catch (const std::exception& e) {
      set_last_error(e.what());
      delete s;
      return FFTSVD_ERR_ARGUMENT;
   }
   *out = s;
   return FFTSVD_OK;
}

extern "C" int fftsvd_b200_surface_stats(const fftsvd_surface* s, fftsvd_surface_stats* out) {
   if (!s || !out) return FFTSVD_ERR_ARGUMENT;
   *out = s->s.stats;
   out->device_bytes = (double)(s->s.op32.device_bytes() + s->s.op64.device_bytes());
   out->matvec_bytes_fp32 = (double)s->s.operator_elems * 4.0 + (double)s->s.t_elems * 4.0 + 2.0 * s->s.n * 8.0;
   out->matvec_bytes_fp64 = (double)s->s.operator_elems * 8.0 + (double)s->s.t_elems * 8.0 + 2.0 * s->s.n * 8.0;
   return FFTSVD_OK;
}
