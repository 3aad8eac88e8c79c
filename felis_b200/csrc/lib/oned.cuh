// The 1D model (dimension = 1) of the FP64 path: one field value per slice,
// harmonic and polarisation (nx = ny = 1), no transverse push.
//   solve_Sc_1D        solveField.cpp:422-549
//   solve_Field_U_1D   solveField.cpp:409-416
//   push_theta_gamma_1D particlePush.cpp:388-524
#pragma once

#include "common.cuh"

namespace felis {

struct OneDLaunch {
  DevGeom G;
  int ns, ring_base;
  const int64_t* soff;   // [ns][S+1]
  const double* weight;  // [ns][S]
  double* th;
  double* ga;
  double2* U;            // field planes (field_plane, N = 1)
  double2* Sc;           // [H][2][S] source of the last solve, logical slices
  double2* Ez;           // [L][S+2]
  int* err;
  // per-call scalars, formed on the host in FP64 in the reference's order
  double Phi, K0, ue, ku, dz, K2, dPhi, e_mc2, sq;  // sq = sqrt(ue*ue + 1)
  cd etaX, etaY;
  double coefU[FELIS_MAX_SPECIES];                    // source coefficient per species
  double coefE[FELIS_MAX_SPECIES];                    // space-charge coefficient per species
  cd fsrc[FELIS_MAX_HARMONY][2];                      // source fx, fy (zero for even harmonics)
  cd fpush[FELIS_MAX_HARMONY][2];                     // push fx, fy (zero for even harmonics)
};

// solveField for dimension 1: the source of every slice when `current`
// (else zero), then U += source; one thread per slice, particles in order.
cudaError_t launch_1d_field(const OneDLaunch& a, int current, cudaStream_t st);
// push_theta_gamma for dimension 1: one CTA per slice, thread per particle.
cudaError_t launch_1d_push(const OneDLaunch& a, cudaStream_t st);

}  // namespace felis
