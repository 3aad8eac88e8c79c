/* felis_b200.h — C ABI of the B200-native FELIS slice loop.
 *
 * The reference (scienter/felis) has no plugin API: its per-step loop
 * (main.cpp:92-156) calls plain C++ functions that mutate one shared Domain
 * (mesh.h:150-178), and its errors end the process (exit / MPI_Abort).
 * This header replaces those functions one for one with entry points that
 * take an opaque handle, keep every array resident in HBM, and return a
 * status instead of exiting.  Each declaration cites the reference function
 * it stands in for.
 *
 * Conventions
 *   - Every function returns felis_status; felis_last_error() gives text.
 *     The library never calls exit().
 *   - The library owns device memory.  Callers own host buffers; copies are
 *     synchronous (the call returns when the host buffer may be reused).
 *   - One handle per host thread; one CUDA stream per handle.
 *   - Complex numbers are interleaved (re, im) FP64, the memory layout of
 *     std::complex<double>.
 *   - Field arrays use the reference layout: per harmonic and polarisation
 *     (slice_n + 2) planes of ny rows by nx points, ghost planes 0 and
 *     slice_n + 1 included (boundary.cpp:49-53).
 *   - Particles are structure-of-arrays, concatenated slice by slice in
 *     slice order, with slice_offsets[slice_n + 1] giving each slice's range
 *     (the per-slice ptclList of particle.h:24-35, flattened).
 */
#ifndef FELIS_B200_H
#define FELIS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FELIS_ABI_VERSION 3
#define FELIS_MAX_HARMONY 8
#define FELIS_MAX_SPECIES 8

typedef enum felis_status {
  FELIS_OK = 0,
  FELIS_BAD_ARG = 1,        /* invalid argument or size */
  FELIS_CUDA_ERROR = 2,     /* a CUDA runtime call failed */
  FELIS_THETA_OVERFLOW = 3, /* |dtheta| > 2 pi numSlice in the push (particlePush.cpp:371-374) */
  FELIS_OUT_OF_RANGE = 4,   /* theta outside [0, dTh] after the wrap (rearrangeParticles.cpp:105-108) */
  FELIS_NAN = 5,            /* non-finite value found in the particle state */
  FELIS_TIMEOUT = 6,        /* a bounded device wait gave up */
  FELIS_UNSUPPORTED = 7,    /* configuration the library does not implement */
  FELIS_NO_DEVICE = 8,      /* no CUDA device */
  FELIS_IO = 9,             /* input file could not be read or parsed */
  FELIS_NOT_FOUND = 10      /* a key or block is missing from the input file */
} felis_status;

typedef enum felis_mode { FELIS_STATIC = 1, FELIS_TIME_DEPENDENT = 2 } felis_mode;
typedef enum felis_und_type { FELIS_BIPOLAR = 1, FELIS_QUADPOLAR = 2 } felis_und_type;
typedef enum felis_precision {
  FELIS_FP64 = 0,  /* plain path: FP64 everywhere, bit-exact with the CPU restatement */
  FELIS_MIXED = 1  /* FP32 push and ADI; FP64 theta, reductions and lattice */
} felis_precision;

/* One [Undulator] block after parameterSetting.cpp:345-429 (UndList, mesh.h:44-56). */
typedef struct felis_undulator {
  int32_t type;     /* felis_und_type */
  int32_t K0_alpha; /* +1: By major, -1: Bx major */
  int32_t numbers;  /* units in this block */
  int32_t air;      /* in_air */
  double lambdaU;   /* [m] */
  double slopeK;    /* slope_K / sqrt(2) [1/m] */
  double ue;        /* polarity */
  const double* unit_start; /* [numbers] each, [m] */
  const double* unit_end;
  const double* und_start;
  const double* und_end;
  const double* K0;
} felis_undulator;

/* One [Quad] block after parameterSetting.cpp:287-338 (QuadList, mesh.h:58-63). */
typedef struct felis_quad {
  int32_t numbers;
  int32_t pad_;
  const double* unit_start;
  const double* unit_end;
  const double* qd_start;
  const double* qd_end;
  const double* g; /* [T/m] */
} felis_quad;

/* Domain scalars and tables after parameterSetting() + boundary()
 * (parameterSetting.cpp:42-285, boundary.cpp:20-124).  Arrays are read
 * during felis_create() only. */
typedef struct felis_params {
  int32_t abi_version; /* FELIS_ABI_VERSION */
  int32_t precision;   /* felis_precision */
  int32_t dimension;   /* 3, or 1 for the 1D model (FP64 handle) */
  int32_t mode;        /* felis_mode */
  int32_t num_harmony;
  int32_t harmony[FELIS_MAX_HARMONY];
  int32_t slice_n;        /* slices held by this handle (subSliceN) */
  int32_t min_i;          /* global index of the first slice (D->minI) */
  int32_t global_slice_n; /* D->sliceN; length of wake_e */
  int32_t nx, ny;         /* grid points (input key + 1, parameterSetting.cpp:108-111) */
  int32_t num_slice;      /* slices_in_bucket */
  int32_t num_lambda_u;   /* lambdaUs_in_iteration */
  int32_t num_species;
  int32_t scl_mode, scf_mode, nr; /* L, F, radial grid of the Ez solve */
  int32_t bessel_rows, bessel_cols; /* bn, BesselMaxOrder */
  int32_t abc_n;
  int32_t wake_on;
  int32_t max_step;
  int32_t num_undulators, num_quads;
  double ks, lambda0, dz, dx, dy, dr;
  double min_x, max_x, min_y, max_y, min_z, max_z;
  double gamma0, gam_r, d_bessel, abc_sig, spot_sig_r;
  /* lattice state after parameterSetting (D->K0, ue, K0_alpha, lambdaU, undType) */
  double K0_init, ue_init, lambdaU_init;
  int32_t K0_alpha_init, und_type_init;
  /* tables from boundary(): ABC coefficients (complex, nx or ny entries),
   * Bessel table (bessel_rows x bessel_cols, row-major), wake energy loss per
   * global slice (wakeField.cpp:9-50; may be NULL when wake_on == 0). */
  const double* abc_alpha;
  const double* abc_alpha_p;
  const double* abc_beta;
  const double* abc_beta_p;
  const double* bessel;
  const double* wake_e;
  const felis_undulator* undulators;
  const felis_quad* quads;
  /* 1D model: the area 2 pi sigX sigY of each species' matched beam, which
   * normalises its source and space-charge field (solveField.cpp:455-470) */
  double beam_area[FELIS_MAX_SPECIES];
  /* [Phase_shifter] blocks (README.md:57-70; the reference documents them but
   * its parser does not read them): shifter k sits at z = phase_shift_z[k]
   * [m] and delays the electrons against the field by phase_shift_phase[k]
   * * pi of the ponderomotive phase: theta -= phase * pi for every particle,
   * after the push or drift of the iteration whose step [it dz, (it+1) dz)
   * contains z, before the wrap (felis_phase_shift in the per-function
   * sequence).  Arrays of num_phase_shifts entries; may be NULL when 0. */
  int32_t num_phase_shifts;
  int32_t pad_ps_;
  const double* phase_shift_z;
  const double* phase_shift_phase;
} felis_params;

/* Lattice state that updateK_quadG() leaves in Domain (updateK_quadG.cpp:8-94). */
typedef struct felis_lattice {
  double K0, ue, lambdaU, ku, g;
  int32_t K0_alpha, und_type, current_flag, drift_flag;
} felis_lattice;

typedef struct felis_handle felis_handle;

/* ---- lifecycle (boundary.cpp:20-71 allocation) ------------------------- */
felis_status felis_create(const felis_params* params, felis_handle** out);
void felis_destroy(felis_handle* h);
const char* felis_last_error(const felis_handle* h);
felis_status felis_device_info(char* name, size_t name_len, int32_t* sm_count);

/* ---- data in / out ------------------------------------------------------
 * Particles of one species (loadBeam.cpp:158-246 / restoreParticleHDF.cpp:166-214
 * fill the same per-slice arrays).  slice_offsets has slice_n + 1 entries,
 * weights has slice_n entries (ptclList::weight). */
felis_status felis_upload_particles(felis_handle* h, int32_t species,
                                    const double* x, const double* y,
                                    const double* px, const double* py,
                                    const double* theta, const double* gamma,
                                    const int64_t* slice_offsets,
                                    const double* weights);
felis_status felis_download_particles(felis_handle* h, int32_t species,
                                      double* x, double* y, double* px,
                                      double* py, double* theta, double* gamma);
/* Field of one harmonic index and polarisation (0: Ux, 1: Uy), reference
 * layout with ghost planes (loadSeed.cpp:74-75 writes it). */
felis_status felis_upload_field(felis_handle* h, int32_t harmonic_index,
                                int32_t pol, const double* data);
felis_status felis_download_field(felis_handle* h, int32_t harmonic_index,
                                  int32_t pol, double* data);
/* Source term ScUx/ScUy of the last solve (solveField.cpp:233-312), same
 * layout; cells the ADI never reads (grid edges) are returned as zero. */
felis_status felis_download_source(felis_handle* h, int32_t harmonic_index,
                                   int32_t pol, double* data);
/* Ez[l][(slice_n+2) * F * nr] of the last space-charge solve. */
felis_status felis_download_ez(felis_handle* h, double* data);

/* ---- lattice (updateK_quadG.cpp:8-94, evaluated on the host in FP64) ---- */
felis_status felis_update_lattice(felis_handle* h, int32_t iteration, double half);
felis_status felis_get_lattice(felis_handle* h, felis_lattice* out);
felis_status felis_set_lattice(felis_handle* h, const felis_lattice* in);

/* ---- per-step functions (main.cpp:117-149) ------------------------------ */
/* updateTotalEnergy.cpp:7-45: out[2*h] = sum |Ux_h|^2, out[2*h+1] = sum |Uy_h|^2
 * over slices 1..slice_n (unscaled, as stored in totalEnergyX/Y). */
felis_status felis_update_total_energy(felis_handle* h, int32_t iteration, double* out);
/* twiss.cpp:7-99: per species {emitX, betaX, alphaX, emitY, betaY, alphaY}
 * (emittance unnormalised, as computed before the file write). */
felis_status felis_twiss(felis_handle* h, int32_t iteration, double* out);
/* saveFile.cpp:109-172: per harmonic {Re b, Im b} of sum w e^{iH theta} / sum w. */
felis_status felis_bfactor(felis_handle* h, int32_t iteration, double* out);
/* solveField.cpp:49-78: source deposit + Ez (if the lattice's current flag is
 * set) and the ADI solve of Ux then Uy, every slice and harmonic. */
felis_status felis_solve_field(felis_handle* h, int32_t iteration);
/* particlePush.cpp:32-117 (one dz/2 RK4 call with the current lattice). */
felis_status felis_transverse_push(felis_handle* h, int32_t iteration);
/* particlePush.cpp:198-386 (push_theta_gamma_3D). */
felis_status felis_push_theta_gamma(felis_handle* h, int32_t iteration);
/* particlePush.cpp:119-195 (drift_theta_gamma). */
felis_status felis_drift_theta_gamma(felis_handle* h, int32_t iteration);
/* rearrangeParticles.cpp:77-114 (periodicParticles). */
/* [Phase_shifter] (README.md:57-70): theta -= phase * pi for every particle
 * when a shifter sits in this iteration's step (see felis_params); a no-op
 * otherwise.  No reference counterpart in the loop: call it between the push
 * or drift and felis_periodic_particles. */
felis_status felis_phase_shift(felis_handle* h, int32_t iteration);
felis_status felis_periodic_particles(felis_handle* h, int32_t iteration);
/* solveField.cpp:19-47 + fieldShareZ.cpp:39-78 at one rank (shiftField). */
felis_status felis_shift_field(felis_handle* h, int32_t iteration);

/* ---- fused helpers ----------------------------------------------------- */
/* One whole iteration of main.cpp:117-155 (diagnostics recorded on the
 * device, lattice updated on the host), using the fused kernels. */
felis_status felis_step(felis_handle* h, int32_t iteration);
/* Iterations [it0, it1) replayed from one captured CUDA graph. */
felis_status felis_run(felis_handle* h, int32_t it0, int32_t it1);
/* Diagnostics recorded by felis_step / felis_run for iterations [it0, it1):
 * energy[(it-it0)*2H + ...] as felis_update_total_energy, twiss
 * [(it-it0)*6*num_species + ...] as felis_twiss, bfactor [(it-it0)*2H + ...]
 * as felis_bfactor.  Any pointer may be NULL. */
felis_status felis_get_diagnostics(felis_handle* h, int32_t it0, int32_t it1,
                                   double* energy, double* twiss, double* bfactor);
/* Count of deposit particles that hit the q6 edge case (cell index nx-1 or
 * ny-1 accepted by solveField.cpp:273), accumulated since creation. */
felis_status felis_edge_deposit_count(felis_handle* h, int64_t* count);

/* ---- measurement ------------------------------------------------------ */
/* Waits for the handle's stream and reports a device error raised since the
 * last check (felis_step and felis_run return device errors the same way). */
felis_status felis_sync(felis_handle* h);
/* Kernel kinds counted / timed by felis_kernel_stats. */
enum {
  FELIS_KERNEL_PARTICLES = 0, /* push / drift / wrap / deposit records / beam partial sums */
  FELIS_KERNEL_DEPOSIT = 1,   /* ordered source deposit + Ez solve */
  FELIS_KERNEL_ADI = 2,       /* ADI sweeps of every plane */
  FELIS_KERNEL_REDUCE = 3,    /* power, twiss and bFactor reductions */
  FELIS_KERNEL_SHIFT = 4,     /* slippage shift (clears one plane per harmonic and pol) */
  FELIS_KERNEL_KINDS = 8
};
/* Resets the launch counters; with enable != 0, brackets each of the next
 * max_launches kernel launches with CUDA events on the handle's stream
 * (recorded into the graph by felis_run). */
felis_status felis_profile(felis_handle* h, int32_t enable, int32_t max_launches);
/* Launches of one kind (kind -1: all kinds) since felis_profile, and the sum
 * of their event-timed durations in milliseconds. */
felis_status felis_kernel_stats(felis_handle* h, int32_t kind, int64_t* launches, double* total_ms);
/* Device time of the last felis_run graph launch (CUDA events around it). */
felis_status felis_last_run_ms(felis_handle* h, double* ms);

/* ---- slices sharded across processes (boundary.cpp:33-46, fieldShareZ.cpp:39-78)
 * A process holds slices [min_i, min_i + slice_n) of global_slice_n.  In
 * exchange mode the slippage shift leaves the plane that becomes this
 * block's first slice holding the block's old last slice; the caller sends
 * those planes to the next process (felis_get_first_planes) and writes the
 * planes received from the previous one in their place
 * (felis_set_first_planes; zeros on the first process), as MPI_Transfer1F_Zplus
 * does.  Call it between iterations (felis_step, or the per-function loop). */
felis_status felis_set_slice_exchange(felis_handle* h, int32_t enable);
/* [H][2][ny*nx] interleaved complex, host buffers. */
felis_status felis_get_first_planes(felis_handle* h, double* out);
felis_status felis_set_first_planes(felis_handle* h, const double* in);
/* The same planes as felis_get_first_planes, as device addresses: planes
 * receives 2 H pointers ([h][pol] order) to ny*nx interleaved complex
 * values in this handle's device memory, valid until the next shift.  A
 * caller that exchanges them in device memory (NCCL send/recv over NVLink,
 * peer copies) orders its work after the step on the handle's stream
 * (felis_get_stream) and before the next step, and writes zeros on the
 * first process (MPI_Transfer1F_Zplus of fieldShareZ.cpp:39-78). */
felis_status felis_first_planes_device(felis_handle* h, double** planes);
/* The CUDA stream (cudaStream_t) on which the handle queues all its work. */
felis_status felis_get_stream(felis_handle* h, void** stream);
/* Unfinished sums of the current state for reductions across processes
 * (twiss.cpp:46-64 per species: sum x^2, y^2, x'^2, y'^2, x x', y y', count;
 * then saveFile.cpp:126-137 per harmonic: sum w cos(H theta), sum w
 * sin(H theta); then sum w): 7 * num_species + 2 * num_harmony + 1 values. */
felis_status felis_diagnostic_sums(felis_handle* h, int32_t it, double* out);

/* ---- slice sort (the slice binning of restoreParticleHDF.cpp:166-214 and
 * the slice-major write order of saveParticleHDF.cpp:95-109) -------------
 * Stable sort of n particles by integer slice key on the GPU: perm[k] is the
 * input row that lands at position k; equal keys keep input order.  Keys
 * must lie in [0, 2^30). */
felis_status felis_sort_by_slice(const int32_t* keys, int64_t n, int64_t* perm);

/* Allocation-free slice sort.  No counterpart in the reference: FELIS itself
 * never runs on a GPU.  It serves callers that must not allocate device
 * memory themselves or through this library, for example a host code whose
 * HBM is owned by another allocator (a framework's caching pool, a
 * pre-partitioned MPI job) or a loop that cannot afford cudaMalloc's implicit
 * device synchronisation.  Same result as felis_sort_by_slice for keys in
 * [0, 2^30) (keys are ordered as unsigned 32-bit values), but keys_dev and
 * perm_dev are device buffers the caller owns, the work is queued on
 * `stream` (a cudaStream_t, NULL for the default stream) and the call returns
 * without waiting for it.  Scratch is a fixed array inside the library
 * (about 4 MB on every GPU that loads it, kept until exit), so n is limited
 * to FELIS_SORT_NOALLOC_MAX_KEYS; larger n returns FELIS_BAD_ARG.  keys_dev
 * and perm_dev must be device (or managed) memory of the current device;
 * other pointers return FELIS_BAD_ARG (checked outside stream capture).  The
 * array's device address belongs to the current CUDA context: every call made
 * outside stream capture resolves it in that context, and a call made during
 * capture uses the address resolved by an earlier call in the same context,
 * so make one call in a context (after any cudaDeviceReset, and in every
 * context you make current) before capturing.  Calls that overlap on the GPU
 * share the array and race: serialise them (one stream, or events). */
#define FELIS_SORT_NOALLOC_MAX_KEYS 262144
felis_status felis_sort_by_slice_noalloc(const int32_t* keys_dev, int64_t n, int64_t* perm_dev, void* stream);

/* ---- mixed-precision ensemble ------------------------------------------
 * Many independent FELIS runs (one felis_params each: own slices, grid,
 * harmonics, lattice and beam) advanced together on one GPU.  No counterpart
 * in the reference, which runs one Domain per MPI job; each instance follows
 * the loop of main.cpp:92-156 with the FP64 plain path's operator order, but
 * computes in mixed precision: particles x, y, px, py, gamma - gamR, the
 * field, the ADI sweeps and the theta slope (taken relative to the
 * resonance) in FP32; theta itself, the lattice (updateK_quadG.cpp on the
 * host), the radial Ez solve and all diagnostic sums in FP64.  The source deposit accumulates fixed-point integers, so a
 * run is reproducible bit for bit, and an instance's results depend neither
 * on the launch shape nor on the other instances, as long as the ensemble's
 * largest harmonic count stays in the same class (1, 2, 3-4 or 5-8: it
 * selects the compiled kernel).  One species, 3D,
 * SCLmode <= 4, grids up to 256 points wide.  Every iteration is two kernel
 * launches over all instances (the ADI of every field plane; the push of
 * every slice with the deposit of the next iteration's source) plus one
 * reduction launch; felis_batch_run captures a range of iterations as one
 * CUDA graph. */
typedef struct felis_batch felis_batch;
felis_status felis_batch_create(const felis_params* const* instances, int32_t n, felis_batch** out);
void felis_batch_destroy(felis_batch* b);
const char* felis_batch_last_error(const felis_batch* b);
/* Same arrays and layouts as felis_upload_particles / felis_upload_field
 * (species 0), converted to the ensemble's storage precision. */
felis_status felis_batch_upload_particles(felis_batch* b, int32_t inst, const double* x, const double* y,
                                          const double* px, const double* py, const double* theta,
                                          const double* gamma, const int64_t* slice_offsets,
                                          const double* weights);
felis_status felis_batch_download_particles(felis_batch* b, int32_t inst, double* x, double* y, double* px,
                                            double* py, double* theta, double* gamma);
felis_status felis_batch_upload_field(felis_batch* b, int32_t inst, int32_t harmonic_index, int32_t pol,
                                      const double* data);
felis_status felis_batch_download_field(felis_batch* b, int32_t inst, int32_t harmonic_index, int32_t pol,
                                        double* data);
/* Iterations [it0, it1) of every instance. */
felis_status felis_batch_run(felis_batch* b, int32_t it0, int32_t it1);
/* Per-iteration energy (2H), twiss (6) and bFactor (2H) of one instance,
 * same meaning as felis_get_diagnostics. */
felis_status felis_batch_get_diagnostics(felis_batch* b, int32_t inst, int32_t it0, int32_t it1,
                                         double* energy, double* twiss, double* bfactor);
/* First-lag spectral moments of every instance's field, harmonic index hidx:
 * out[3 i + 0] = sum |U_s|^2, out[3 i + 1] + i out[3 i + 2] = sum conj(U_s)
 * U_{s+1}, over the slices s in bunch order, every cell and both
 * polarisations (FP64 sums).  With the slice spectrum P(nu) of the field,
 * R1 / R0 = <e^{2 pi i nu}>: arg(R1) / (2 pi) is the spectral centroid and
 * sqrt(-2 ln(|R1| / R0)) / (2 pi) the rms bandwidth of a Gaussian line, in
 * units of the slice frequency.  Instances without harmonic index hidx give
 * zeros.  (No reference counterpart: the reference writes fields to disk.) */
felis_status felis_batch_spectral_moments(felis_batch* b, int32_t hidx, double* out);
/* Launch shape: the source cells the push launch stages in shared memory
 * (512 .. 6144, default 3072: seven one-harmonic push CTAs of 128 threads share
 * an SM; larger areas take fewer cells of wide beams through global memory)
 * and the CTAs per SM the ADI launch sizes its shared memory for (1 or 2; the
 * rest stages the slice's source box).  Results do not depend on it. */
felis_status felis_batch_set_launch(felis_batch* b, int32_t push_box, int32_t adi_ctas);
felis_status felis_batch_get_launch(felis_batch* b, int32_t* push_box, int32_t* adi_ctas);
/* Tries each launch shape for `steps` real iterations starting at it0 (the
 * ensemble advances; results do not depend on the shape), keeps the fastest
 * and returns the next iteration to run in *next_it.  Shapes are cached per
 * ensemble geometry and GPU kind, in memory and in the text file named by
 * FELIS_TUNE_CACHE ($HOME/.cache/felis_b200_batch_tune_v2.txt by default): a
 * later call on a matching ensemble, in this process or another, runs
 * nothing. */
felis_status felis_batch_tune(felis_batch* b, int32_t it0, int32_t steps, int32_t* next_it);
/* Device time of the last felis_batch_run graph launch. */
felis_status felis_batch_last_run_ms(felis_batch* b, double* ms);
/* Kernel kinds of the ensemble, event-timed like felis_profile /
 * felis_kernel_stats (the measure + reduce pair of a run's first iteration
 * counts as one REDUCE launch). */
enum {
  FELIS_BATCH_KERNEL_ADI = 0,    /* field planes of one grid size */
  FELIS_BATCH_KERNEL_PUSH = 1,   /* push + next deposit (or the first deposit) */
  FELIS_BATCH_KERNEL_REDUCE = 2, /* per-instance diagnostics */
  FELIS_BATCH_KERNEL_KINDS = 4
};
felis_status felis_batch_profile(felis_batch* b, int32_t enable, int32_t max_launches);
felis_status felis_batch_kernel_stats(felis_batch* b, int32_t kind, int64_t* launches, double* total_ms);

/* ---- taper surrogate network ---------------------------------------------
 * No counterpart in the reference.  A multilayer perceptron of four linear
 * layers (n_in -> width -> width -> width -> n_out, GELU after the first
 * three) that learns per-segment power and bandwidth from taper and beam
 * parameters, trained on runs of the ensemble engine.  Forward and backward
 * passes run on the tensor cores (BF16 weights and activations, FP32
 * accumulation); FP32 master parameters with AdamW.  width is 128 or 256;
 * n_in <= 256, n_out <= width.  Inputs and outputs are row-major FP32 host
 * arrays, [n][n_in] and [n][n_out]; the loss is the mean squared error over
 * all outputs (normalise the targets beforehand). */
/* Self-test of the bounded device wait that guards the tensor-core pipeline
 * (no reference counterpart: the reference has no device waits).  Runs the
 * library's mbarrier wait, `limit` tries, on a barrier phase that nothing
 * completes, on the current device: returns FELIS_TIMEOUT with *timed_out = 1
 * when the wait gave up as designed (the context stays usable), FELIS_OK with
 * *timed_out = 0 if it did not. */
felis_status felis_wait_selftest(int32_t limit, int32_t* timed_out);

typedef struct felis_mlp felis_mlp;
felis_status felis_mlp_create(int32_t n_in, int32_t width, int32_t n_out, uint64_t seed, felis_mlp** out);
void felis_mlp_destroy(felis_mlp* m);
const char* felis_mlp_last_error(const felis_mlp* m);
/* Parameters flattened as W1 [width][n_in], b1, W2, b2, W3, b3, W4 [n_out][width], b4. */
felis_status felis_mlp_param_count(const felis_mlp* m, int64_t* count);
felis_status felis_mlp_get_params(felis_mlp* m, float* out);
/* Sets the parameters and resets the optimiser state. */
felis_status felis_mlp_set_params(felis_mlp* m, const float* in);
/* Inference: y [n][n_out] of x [n][n_in].  With hidden width 256, n_in <= 64
 * and n_out <= 256 the four layers run as one fused tensor-core kernel
 * (activations kept on chip); otherwise, or after felis_mlp_set_fused(m, 0),
 * as the layer-by-layer GEMM chain.  Both round at the same places. */
felis_status felis_mlp_forward(felis_mlp* m, const float* x, int64_t n, float* y);
/* Chooses the fused inference kernel (enable != 0, the default where the
 * shape allows it) or the layer-by-layer chain; FELIS_UNSUPPORTED when the
 * fused kernel is asked for a shape it does not cover. */
felis_status felis_mlp_set_fused(felis_mlp* m, int32_t enable);
/* Device time (CUDA events on the network's stream) and floating-point
 * operations (2 M N K summed over the four layers, M the padded rows) of the
 * inference kernels of the last chunk of the last felis_mlp_forward (chunks are up
 * to 1,048,576 rows). */
felis_status felis_mlp_last_forward(const felis_mlp* m, double* ms, double* flops);
/* Gradient of the loss over n <= 65536 samples, in the parameter layout, and
 * the loss itself. */
felis_status felis_mlp_gradients(felis_mlp* m, const float* x, const float* t, int64_t n, float* grads,
                                 double* loss);
/* Training set kept on the device for felis_mlp_train. */
felis_status felis_mlp_set_data(felis_mlp* m, const float* x, const float* t, int64_t n);
/* Shuffled minibatches (batch a multiple of 128, at most 65536) with AdamW
 * (beta 0.9 / 0.999, weight decay on the weights only); writes the mean loss
 * of every epoch. */
felis_status felis_mlp_train(felis_mlp* m, int32_t epochs, int32_t batch, float lr, float weight_decay,
                             uint64_t seed, double* loss_per_epoch);

/* ---- host-side setup of the reference's input format -------------------- */
/* Parses a FELIS input file ([Domain], [Save], [Seed], [Undulator], [Quad],
 * [EBeam], [Wake_field], [Bessel_table], [Phase_shifter] blocks;
 * findparam.cpp:30-116, parameterSetting.cpp:42-627) and builds the tables
 * of boundary.cpp:73-124.  The returned object owns every array that
 * felis_params points to. */
typedef struct felis_config felis_config;
felis_status felis_config_load(const char* path, int32_t num_ranks, int32_t rank,
                               felis_config** out);
void felis_config_free(felis_config* c);
const felis_params* felis_config_params(const felis_config* c);
const char* felis_config_error(void);
/* Initial particles of one species (loadBeam.cpp:28-269): writes counts per
 * slice (slice_n entries) when the arrays are NULL; fills them otherwise.
 * `seed` plays the role of GSL_RNG_SEED. */
felis_status felis_config_load_beam(felis_config* c, int32_t species, uint64_t seed,
                                    int64_t* counts, double* x, double* y,
                                    double* px, double* py, double* theta,
                                    double* gamma, double* weights);
/* The same particles computed on the device (loadBeam.cpp:28-269): x .. gamma
 * are device pointers (beamlet-major, the order of felis_config_load_beam),
 * counts and weights host arrays; counts first when x is NULL.  The host
 * keeps the per-slice setup and the sequential noise stream; one kernel
 * computes the Halton points, the transverse and energy transforms and the
 * mirrored phases.  Equal to felis_config_load_beam up to the last bits of
 * log / sin / cos (the device's against the host C library's). */
felis_status felis_config_load_beam_device(felis_config* c, int32_t species, uint64_t seed,
                                           int64_t* counts, double* x, double* y,
                                           double* px, double* py, double* theta,
                                           double* gamma, double* weights);
/* Initial seed field (loadSeed.cpp:25-80), reference layout, both pols. */
felis_status felis_config_load_seed(felis_config* c, int32_t harmonic_index,
                                    double* ux, double* uy);
/* Wake energy loss per slice (wakeField.cpp:9-50,53-159,161-223) from the
 * per-slice charge (den[s] = weight * count, summed over species). */
felis_status felis_config_wake(felis_config* c, const double* den, double* wake_e);
/* The same computed on the GPU (wakeField.cpp:9-50, 53-159; host buffers,
 * the device arrays are allocated per call): the wake function when none is
 * cached yet (agrees with the host's to about 1e-13), then the convolution
 * with the density in the reference's order (bit-identical to
 * felis_config_wake for the same wake function).  The wake function is
 * cached in the config for later calls of either entry point. */
felis_status felis_config_wake_device(felis_config* c, const double* den, double* wake_e);
/* The cached wake function W(i dZ) per global slice distance
 * (wakeField.cpp:128-140), computed on the host when none is cached. */
felis_status felis_config_wake_function(felis_config* c, double* wake_f);

/* ---- deterministic elementary functions (host versions, for tests) ------ */
void felis_detmath_sincos(double x, double* s, double* c);
double felis_detmath_atan(double x);
double felis_detmath_atan2(double y, double x);

#ifdef __cplusplus
}
#endif
#endif /* FELIS_B200_H */
