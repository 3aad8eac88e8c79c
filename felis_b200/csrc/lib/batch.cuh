// Mixed-precision ensemble engine: declarations shared by the host code and
// the kernels.
#pragma once

#include "common.cuh"

namespace felis {

// Fixed-point source accumulators (32-bit integers; see k_batch.cu).
typedef int acc_t;

// One instance (one FELIS Domain) of the ensemble.  FP32 particle state and
// field; theta in FP64.  Gamma is kept as dg = gamma - gamR in FP32: an
// absolute FP32 gamma near 1.6e4 has an ulp of 1e-3, which rounds away the
// per-step energy exchange, while dg (of the size of the energy spread)
// resolves it to 1e-7.
struct BInst {
  int S, nx, ny, N, H, L, F, nr, bn, bcols, numSlice, minI, wakeOn;
  // ADI: row pitch of the shared-memory plane of interior cells (odd, >= nx - 2)
  // and the four chunks each interior row / column is split into (starts,
  // then the interior count): cx over the nx - 2 columns, cy over the rows
  int pitch, cx[5], cy[5];
  // per harmonic, from its tables (batch.cu adi_ranges): the interior index
  // ranges [kx0, kx1) over columns and [ky0, ky1) over rows where every
  // coefficient table of that direction holds one value, and the lengths
  // over which the chunk products matter (a component >= 2^-40): G from a
  // chunk's start, Q from its end.  {kx0, kx1, ky0, ky1, gx, qx, gy, qy}
  int adi_k[FELIS_MAX_HARMONY][8];
  int nsrc;                             // source planes per slice
  int harmony[FELIS_MAX_HARMONY];
  int src_plane[FELIS_MAX_HARMONY];     // first source plane of each harmonic
  double ks, dz, dx, dy, dr, minX, minY, gamR, dBessel;
  float *x, *y, *px, *py, *dg;
  double* th;
  const int64_t* soff;   // [S+1]
  const float* weight;   // [S]
  float2* U;             // [H][2][S][N] ring per (H, pol)
  float2* Ez;            // [L][S][F][nr]
  float2* src;           // [S][nsrc][N] source of the next ADI, box-compact
  int4* sbox;            // [S] cell box of that source (bi0, bi1, bj0, bj1)
  const float* bessel;   // [bn][bcols]
  const double* wakeE;   // global slices
  const float2* adi_c;   // per harmonic: 16 complex tables of max(nx, ny), interior index (batch.cu)
  double* part_e;        // [S][H*2] plane energies of the last ADI
  double* part_b;        // [S][7 + 2H + 1] beam partial sums of the last push
  int* err;              // [ERR_SLOTS]
};

// Deposit constants of one lattice state (solveField.cpp:209-243).
struct BDep {
  float K0, ue, K0a, Phi_half, coef_U, xi, coef_Ez;
  double A;
  float2 etaX, etaY;
  float fconst[FELIS_MAX_HARMONY][2];
};

// Per-iteration scalars of one instance (updateK_quadG on the host, FP64,
// rounded to the precision each kernel computes in).
struct BStep {
  int ring_base;  // ring offset during this step
  int shift;      // this step ends with the slippage shift
  int drift;      // drift instead of push_theta_gamma
  int current;    // the ADI of this step adds the source (solveField's flag)
  int deposit;    // the push launch deposits the source of the next step
  // both transverse half-pushes as one linear map of (x, y, px, py), to
  // second order in da = 1/gamma - 1/gamR: s += D0 s + da (M1 s + da M2 s)
  float tD0[16], tM1[16], tM2[16];
  // push_theta_gamma (lattice after updateK(it, 0.5)).  The theta slope
  //   ku - ks / (2 gamma^2) (K2 + X)
  // is a small difference of two terms near ku; with gamma = gamR (1 + d),
  // K2 = Q0 + k2 and A0 = ks / (2 gamR^2) it is evaluated in FP32 as
  //   R0 + AQ0 (1 - (1 + d)^-2) - A0 (1 + d)^-2 (k2 + X),
  // R0 = ku - A0 Q0 and AQ0 = A0 Q0 formed in FP64 on the host.
  float R0, A0, AQ0, c1, c2, K0, ue, K0a, Phi_half, cxi, sq, ksK0, e_mc2, dPhi;
  double ku, A0d;  // drift: theta += (ku - A0d (1 + px^2 + py^2 + sumU2)) dz, FP64
  double theta_shift;  // [Phase_shifter] delay added to theta before the wrap
  float2 etaX, etaY;
  BDep dep;       // deposit done by this launch
  float2 sfac[FELIS_MAX_HARMONY][2];  // ADI source factor per harmonic and polarisation
  // the radial Ez elimination of this launch's deposit (data-independent:
  // it depends on dep.A, l, f and nr only), made on the host: per (l, f) mode
  // nr pairs (w_j, b_j) at BatchLaunch::rad + rad_off, b_0 in the first pair
  int64_t rad_off;
};

constexpr int kPushThreads = 128;  // threads per CTA of the push launch

struct BatchLaunch {
  const BInst* inst;
  const BStep* step;  // [ninst] for this iteration
  const int4* work;   // ADI: {instance, slice, plane}; push: {instance, slice}
  int nwork;
  int smem_bytes;     // dynamic shared memory of the launch
  int mode;           // push launch: BATCH_PUSH or BATCH_DEPOSIT_ONLY
  const double* rad;  // push launch: the radial elimination tables of the run (BStep::rad_off)
};

enum { BATCH_PUSH = 0, BATCH_DEPOSIT_ONLY = 1 };

void launch_batch_adi(const BatchLaunch& a, int threads, cudaStream_t st);
// dst[i] = (float)(src[i] - off) on the device (particle uploads).
cudaError_t launch_f64_to_f32(const double* src, float* dst, int64_t n, double off, cudaStream_t st);
// dst[i] = off + (double)src[i] on the device (particle downloads).
cudaError_t launch_f32_to_f64(const float* src, double* dst, int64_t n, double off, cudaStream_t st);
// Slices [s0, s0 + ns) of one field plane set, complex FP64 in the reference
// layout (slice s at src + 2 (s - s0) N doubles), rounded into the ring U
// (slice s at ring plane (s + ring_base) % S).
cudaError_t launch_field_to_f32(const double* src, float2* U, int s0, int ns, int S, int N, int ring_base,
                                cudaStream_t st);
// H: the largest harmonic count of the ensemble (selects the kernel instance).
// The push launch: 128 threads per CTA (kPushThreads), the instance of the
// ensemble's largest harmonic count H and Ez mode count L.
void launch_batch_push(const BatchLaunch& a, int H, int L, cudaStream_t st);
void launch_batch_measure(const BInst* inst, const BStep* step, const int4* work, int nwork, cudaStream_t st);
// Per instance {sum |U|^2, Re, Im sum conj(U_s) U_{s+1}} of harmonic index
// hidx over slices (bunch order from ring[i]), cells and polarisations.
void launch_batch_spectrum(const BInst* inst, int ninst, const int* ring, int hidx, double* out, cudaStream_t st);
void launch_batch_reduce(const BInst* inst, int ninst, const BStep* step, double* hist_e, double* hist_t,
                         double* hist_b, int hist_stride_e, int hist_stride_t, int hist_stride_b, cudaStream_t st);
// Threads of the ADI launch of one grid size: four chunk groups of the
// interior line count rounded up to whole warps.
int batch_adi_threads(int nx, int ny);
// Shared memory of the ADI launch of one grid size with `src_cells` source
// cells staged.
size_t batch_adi_smem(int nx, int ny, int src_cells);
// Shared memory of the push launch with room for the accumulators of
// `box_cells` source cells of every source plane.
size_t batch_push_smem(int nsrc_max, int LF_max, int nr_max, int box_cells);
cudaError_t batch_set_smem(int H, int L, int adi_bytes, int push_bytes);
// CTAs of each kernel that fit on one SM with this shape.
int batch_resident_adi(int threads, int smem_bytes);

}  // namespace felis
