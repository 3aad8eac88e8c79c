// Particle kernels of the FELIS slice loop: declarations shared by the
// launch code and the kernels.
#pragma once

#include "common.cuh"

namespace felis {

// Operation bits of one particle-kernel launch.  A launch applies, in this
// order: transverse push with t0, transverse push with t1, push_theta_gamma
// or drift, the phase shifter's theta delay, theta wrap, deposit records for
// the next solveField, and the twiss / bFactor partial sums of the resulting
// state.
enum ParticleOps : unsigned {
  OP_T0 = 1u << 0,
  OP_T1 = 1u << 1,
  OP_PUSH = 1u << 2,
  OP_DRIFT = 1u << 3,
  OP_WRAP = 1u << 4,
  OP_PREP = 1u << 5,
  OP_DIAG = 1u << 6,
  OP_PHASE = 1u << 7
};

// particlePush.cpp:42-68 scalars of one transversePush call.
struct TransCoef {
  double dz, ku, K0, ue, aa, bb, cc, xCoef, yCoef;
  int K0_alpha;
  int valid;
};

// particlePush.cpp:213-244 / 124-139 scalars of one push or drift call.
struct PushCoef {
  double dz, ku, ks, K0, ue, K0_alpha, dPhi, e_mc2, gamR, Phi;
  cd etaX, etaY;
};

// solveField.cpp:200-243 scalars of one solve_Sc_3D call.
struct PrepCoef {
  double K0, ue, K0_alpha, Phi, coef_U, xi, coef_Ez;
};

struct ParticleLaunch {
  unsigned ops;
  DevGeom G;
  DevParticles P;
  const double2* U;   // field planes, see field_plane()
  int ring_base;
  const double2* Ez;  // [L][(S+2)*F*nr]
  TransCoef t0, t1;
  PushCoef pc;
  PrepCoef prep;
  DevDeposit dep;
  double* diag;       // [ntiles][diag_stride]
  int diag_stride;
  double theta_shift;  // OP_PHASE: added to theta before the wrap
  int* err;
};

void launch_particles(const ParticleLaunch& a, cudaStream_t st);
// Deterministic two-level reduction of the per-tile partial sums; l1 holds
// l1_blocks * (7*nspecies + 2H + 1) doubles.
void launch_diag_finalize(const double* partials, int ntiles, int stride, int nspecies, int H,
                          const int4* tiles, double* l1, int l1_blocks, double* out_twiss, double* out_bf,
                          cudaStream_t st);

}  // namespace felis
