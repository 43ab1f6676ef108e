// Host-side operator setup (placeholder until the octree setup lands).
#include "../../include/fftsvd_b200.h"

extern "C" int fftsvd_b200_surface_create(const fftsvd_problem* problem, fftsvd_surface** out) {
   (void)problem;
   if (out) *out = nullptr;
   return FFTSVD_ERR_UNSUPPORTED;
}

extern "C" void solveSurfaceOperator(double** solution, struct _SurfaceOperator* so, struct _Preconditioner* p,
                                     double* rhs, unsigned int n) {
   (void)so; (void)p; (void)rhs; (void)n;
   if (solution) *solution = nullptr;
}

extern "C" void generateRHS(double** rhs, struct _SurfaceOperator* so, unsigned int n) {
   (void)so; (void)n;
   if (rhs) *rhs = nullptr;
}
