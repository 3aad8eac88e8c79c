// Field kernels of the FELIS slice loop: declarations.
#pragma once

#include "common.cuh"

namespace felis {

// Coefficient tables of the ADI sweeps for one harmonic (solveField.cpp:
// 110-181), built on the host with the same complex formulas as the CPU
// restatement so the recurrences below reproduce it bit for bit.
struct AdiTab {
  // x-sweep right-hand side (index j): -betaP, (H + betaP + beta), beta
  const cd *rx_m, *rx_0, *rx_p;
  // x-sweep recurrence (index i): alphaP and 1/|alphaP|^2, alpha,
  // Q = alphaP*CC[i-1] and 1/|Q|^2, CC and 1/|CC|^2
  const cd *ax_p, *ax_a, *ax_q, *ax_cc;
  const double *ax_pinv, *ax_qinv, *ax_ccinv;
  // y-sweep right-hand side (index i): -alphaP, (H + alphaP + alpha), alpha
  const cd *ry_m, *ry_0, *ry_p;
  // y-sweep recurrence (index j)
  const cd *ay_p, *ay_a, *ay_q, *ay_cc;
  const double *ay_pinv, *ay_qinv, *ay_ccinv;
};

struct AdiLaunch {
  DevGeom G;
  double2* U;          // ring of S planes per (h, pol)
  int ring_base;
  const double2* Sc;   // [H][2][S][N]
  const int4* box;     // per slice: {i0, i1, j0, j1} of written source cells
  int use_source;      // currentFlag of solveField
  const AdiTab* tab;   // [H] (device array of structs)
  double* energy;      // [H][2][S] plane sums of |U|^2 after the solve (may be null)
  int nxp;             // padded row length of the shared-memory plane
  double2* scratch;    // k_adi_big: one plane per CTA
  int* err;            // [ERR_SLOTS] (ERR_TIMEOUT: a bounded staging wait ran out)
};

struct DepositLaunch {
  DevGeom G;
  DevDeposit dep;
  const int64_t* soff;  // [nspecies][S+1]
  int64_t total;
  double2* Sc;          // [H][2][S][N]
  int4* box;            // [S]
  double2* Ez;          // [L][(S+2)*F*nr]
  double2 fconst[FELIS_MAX_HARMONY][2];  // odd-harmonic fx, fy (per call constants)
  cd etaX, etaY;
  double A;             // Ez Thomas coefficient (solveField.cpp:320)
  int cap;              // particles per chunk (<= 4096, the radix sort's u16 counters)
  int neven;            // number of even harmonics
  int* err;
};

void launch_deposit(const DepositLaunch& a, cudaStream_t st);
size_t deposit_smem_bytes(int chunk, int H, int neven, int L, int F, int nr);
void deposit_set_smem(size_t bytes);
void adi_set_smem(size_t bytes);
void launch_adi(const AdiLaunch& a, cudaStream_t st);
size_t adi_smem_bytes(int nx, int ny, int nxp);
// Planes larger than shared memory: `grid` CTAs, each with one scratch plane.
void launch_adi_big(const AdiLaunch& a, int grid, cudaStream_t st);
size_t adi_big_smem_bytes(int nx, int ny);
void launch_energy(const DevGeom& G, const double2* U, int ring_base, double* out_planes, cudaStream_t st);
void launch_sum_planes(const double* planes, int H, int S, int skip_last, double* out, cudaStream_t st);

}  // namespace felis
