// Device-side definitions shared by the FELIS slice-loop kernels.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../detmath.h"
#include "../../../include/felis_b200.h"

namespace felis {

// constants.h:1-10 of the reference.
#define K_MU0 1.2566370614e-6
#define K_VELOCITYC 299792458.0
#define K_EMASS 9.10938291e-31
#define K_ECHARGE 1.60217662e-19
#define K_MC2 0.510998918
#define K_Z0 376.730313668

// [Phase_shifter] (README.md:57-70): the theta delay of iteration it, minus
// pi times the phases of the shifters at z in [it dz, (it+1) dz), summed in
// list order; 0 when none sits in that step.
inline double phase_shift_of(int n, const double* z, const double* phase, int it, double dz) {
  double d = 0.0;
  const double z0 = it * dz, z1 = (it + 1) * dz;
  for (int k = 0; k < n; ++k)
    if (z[k] >= z0 && z[k] < z1) d -= M_PI * phase[k];
  return d;
}

// ---- complex arithmetic ----------------------------------------------------
// Same operand order as std::complex<double> in the reference; division is
// the limited-range, reciprocal expansion its -ffast-math build selects.
struct cd {
  double re, im;
};
__host__ __device__ __forceinline__ cd C(double r, double i) { return cd{r, i}; }
__host__ __device__ __forceinline__ cd cadd(cd a, cd b) { return C(a.re + b.re, a.im + b.im); }
__host__ __device__ __forceinline__ cd csub(cd a, cd b) { return C(a.re - b.re, a.im - b.im); }
__host__ __device__ __forceinline__ cd cneg(cd a) { return C(-a.re, -a.im); }
__host__ __device__ __forceinline__ cd cmul(cd a, cd b) {
  return C(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
__host__ __device__ __forceinline__ cd cscale(cd a, double s) { return C(a.re * s, a.im * s); }
__host__ __device__ __forceinline__ cd cdivr(cd a, double s) { return C(a.re / s, a.im / s); }
__host__ __device__ __forceinline__ double cnorm(cd a) { return a.re * a.re + a.im * a.im; }
__host__ __device__ __forceinline__ cd cconj(cd a) { return C(a.re, -a.im); }
__host__ __device__ __forceinline__ cd cradd(double d, cd c) { return C(d + c.re, c.im); }
__host__ __device__ __forceinline__ cd crsub(double d, cd c) { return C(d - c.re, -c.im); }
__host__ __device__ __forceinline__ double cinvnorm(cd b) { return 1.0 / (b.re * b.re + b.im * b.im); }
// a / b with inv = cinvnorm(b) precomputed (identical bits to the full formula).
__host__ __device__ __forceinline__ cd cdiv_inv(cd a, cd b, double inv) {
  return C((a.re * b.re + a.im * b.im) * inv, (a.im * b.re - a.re * b.im) * inv);
}
__host__ __device__ __forceinline__ cd cdiv(cd a, cd b) { return cdiv_inv(a, b, cinvnorm(b)); }
// std::exp(z) for z = (+-0, phase).
__device__ __forceinline__ cd cexpi(double phase) {
  double s, c;
  fm::sincos(phase, &s, &c);
  return C(c, s);
}

// ---- error flags (device word array, read back by the host) ---------------
enum ErrSlot {
  ERR_THETA_OVERFLOW = 0,  // particlePush.cpp:371-374
  ERR_OUT_OF_RANGE = 1,    // rearrangeParticles.cpp:105-108
  ERR_NAN = 2,
  ERR_RADIAL = 3,          // in-grid particle outside the radial Ez grid (Em carry-over case)
  ERR_EDGE_DEPOSIT = 4,    // q6 edge cells (count)
  ERR_DEPOSIT_CAPACITY = 5,
  ERR_TIMEOUT = 6,         // a bounded device wait ran out
  ERR_SLOTS = 8
};

// ---- handle-wide constants --------------------------------------------------
struct DevGeom {
  int S, nx, ny, N, H, L, F, nr, bn, bcols, nspecies, numSlice, minI, wakeOn, mode;
  int harmony[FELIS_MAX_HARMONY];
  double ks, lambda0, dz, dx, dy, dr, minX, minY, gamR, dBessel;
  const double* bessel;   // [bn][bcols]
  const double* wakeE;    // global slices
  const double* logtab;   // log((j+0.5)/(j-0.5)), j < nr (index 0 unused)
};

// Lattice-dependent scalars for one kernel call (updateK_quadG output plus
// the per-call constants of particlePush.cpp / solveField.cpp).
struct DevLattice {
  double K0, ue, ku, g;
  int K0_alpha, und_type, current, drift;
  double Phi;
  cd etaX, etaY;
};

// Particles of all species, concatenated species-major; each species is
// slice-major.  Tiles of <= 256 particles never straddle a slice.
struct DevParticles {
  double *x, *y, *px, *py, *th, *ga;
  const int64_t* soff;   // [nspecies][S + 1] absolute offsets into the arrays
  const double* weight;  // [nspecies][S]
  const int4* tiles;     // {species, slice, begin, end}
  int ntiles;
  int64_t total;
};

// Per-particle deposit records (written before the ordered deposit).
struct DevDeposit {
  int* key;        // idxJ*nx + idxI, or -1
  int* rkey;       // idxR (0 <= idxR < nr), or -1
  double* wx1;     // wx[1]
  double* wy1;     // wy[1]
  double* wr1;     // wr[1]
  double2* coef;   // [H][total]: macro_expTheta_coef
  double2* fx;     // [H][total] (even harmonics only)
  double2* fy;
  double2* ez;     // [L*F][total]: coefComp before the radial weight
};

__device__ __forceinline__ void set_flag(int* err, int slot) { atomicOr(err + slot, 1); }

// Index of field plane (h, pol, logical slice s in [0, S)) in the ring of S
// planes per (h, pol): the slippage shift only moves ring_base.
__host__ __device__ __forceinline__ size_t field_plane(int S, int h, int pol, int s, int ring_base) {
  int phys = s + ring_base;
  phys %= S;
  if (phys < 0) phys += S;
  return ((size_t)(h * 2 + pol) * S + phys);
}


}  // namespace felis
