// Point-charge right-hand side and reaction-potential collection: dense
// charge x panel interactions evaluated on the GPU in FP64.
#pragma once

#include <vector>

#include "common.h"
#include "integrals.h"

namespace fftsvd {

struct Surface;

struct PanelGeometry {
   int num_panels = 0;
   DevBuf<FlatPanel> panels;          // panel geometry (device)
   DevBuf<int32_t> phi_row, dphi_row; // unknown rows of phi and dphi/dn of each panel
   std::vector<FlatPanel> host;
};

// Panel geometry of the charge-bearing (interior) region and the rows that
// hold phi / dphi/dn of each of its panels (SurfaceOperator.c:291-321, 364-396).
void set_geometry(Surface& S, int num_panels, const double* vertices, const int32_t* phi_row, const int32_t* dphi_row);
void set_charges(Surface& S, int num_charges, const double* pos, const double* q);

// rhs[phi_row[i]] = sum_j q_j / |x_j - c_i|, other rows zero.  Device pointer.
void rhs_device(Surface& S, double* rhs);
// rhs[rows[i]] += sum_j q_j / |x_j - c_i| for nt target centroids c (xyz triples), charges in
// order (SurfaceOperator.c:298-312).  Device pointers; asynchronous on `stream`.
void rhs_points_device(int nt, const double* centroids, const int32_t* rows, int nq, const double* qpos,
                       const double* q, double* rhs, cudaStream_t stream);
// phi_j = sum_i (dphi_i SLP(x_j, i) - phi_i DLP(x_j, i)) - 4 pi phi_i [x_j == c_i].  Device pointers.
void reaction_device(Surface& S, const double* sol, double* phi);
// The same sum for nq points against an explicit panel set, all device arrays:
// phi_j = sum_k (dens[dphi_row[k]] SLP(x_j, k) - dens[phi_row[k]] DLP(x_j, k))
//         - 4 pi dens[phi_row[k]] [x_j == centroid_k].
// np may be 0 (phi is zeroed).  Synchronises the stream.
void reaction_points_device(int np, const FlatPanel* panels, const int32_t* phi_row, const int32_t* dphi_row,
                            const double* dens, int nq, const double* qpos, double* phi, cudaStream_t stream);
// 0.5 * sum q phi * 332.112 / eps_in
double energy_device(Surface& S, const double* phi);

}  // namespace fftsvd
