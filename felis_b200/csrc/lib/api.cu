// C ABI of the FELIS slice loop on one B200: the handle, device memory, the
// host-side lattice (updateK_quadG in FP64) and the per-step call sequence.
//
// Device memory layout (FP64 plain path, all resident in HBM):
//   particles   6 SoA arrays of double, species-major then slice-major,
//               slice_offsets -> absolute offsets; 256-particle tiles that
//               never straddle a slice drive the particle kernels
//   U           [H][pol][S] planes of ny*nx double2, used as a ring per
//               (H, pol): the slippage shift (solveField.cpp:19-47) only
//               moves ring_base and clears one plane
//   Sc          [H][pol][S][ny*nx] source of the last deposit, with a
//               per-slice box of written cells (the ADI treats the rest as 0)
//   Ez          [L][(S+2)*F*nr] in the reference layout (ghost slices kept)
//   deposit     per-particle records written by the particle kernel
//   tables      ABC/ADI recurrence coefficients per harmonic, Bessel table,
//               wake loss, log table of the Ez solve
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "field.cuh"
#include "oned.cuh"
#include "particles.cuh"

using namespace felis;

namespace {

struct HostUnd {
  int type, K0_alpha, numbers, air;
  double lambdaU, slopeK, ue;
  std::vector<double> unitStart, unitEnd, undStart, undEnd, K0;
};
struct HostQuad {
  int numbers;
  std::vector<double> qdStart, qdEnd, g;
};

struct AdiHost {
  std::vector<cd> v;       // all complex arrays back to back
  std::vector<double> d;   // all real arrays back to back
};

}  // namespace

struct felis_handle {
  felis_params p{};
  int device = 0;
  cudaStream_t st = nullptr;
  DevGeom G{};
  std::string err;
  // lattice (Domain fields written by updateK_quadG)
  felis_lattice lat{};
  std::vector<HostUnd> und;
  std::vector<HostQuad> quad;
  std::vector<double> ps_z, ps_phase;  // [Phase_shifter] positions [m] and phases [pi]
  // particles
  std::vector<int64_t> counts;   // [nspecies]
  std::vector<int64_t> soff;     // [nspecies][S+1] absolute
  std::vector<double> weight;    // [nspecies][S]
  std::vector<char> uploaded;
  int64_t total = 0;
  double *x = nullptr, *y = nullptr, *px = nullptr, *py = nullptr, *th = nullptr, *ga = nullptr;
  int64_t* d_soff = nullptr;
  double* d_weight = nullptr;
  int4* d_tiles = nullptr;
  std::vector<int4> tiles;
  // deposit records
  DevDeposit dep{};
  int64_t dep_cap = 0;
  bool has_even = false;
  int dep_pcap = 0;
  // field
  double2* U = nullptr;
  double2* Sc = nullptr;
  int4* box = nullptr;
  double2* Ez = nullptr;
  int ring_base = 0;
  // tables
  double* d_bessel = nullptr;
  std::vector<double> bessel_host;
  double* d_wake = nullptr;
  double* d_log = nullptr;
  std::vector<AdiHost> adi_host;
  std::vector<void*> adi_dev;
  AdiTab* d_adi = nullptr;
  int nxp = 0;
  double2* adi_scratch = nullptr;  // planes larger than shared memory: one per CTA
  int adi_big_grid = 0;
  int sms = 148;
  // diagnostics
  double* d_part = nullptr;
  int diag_stride = 0;
  double* d_planes = nullptr;     // [H][2][S] ADI plane energies
  double* d_planes2 = nullptr;    // scratch for direct energy
  double* d_hist_e = nullptr;     // [max_step+1][2H]
  double* d_hist_t = nullptr;     // [max_step+1][6*nspecies]
  double* d_hist_b = nullptr;     // [max_step+1][2H]
  int hist_n = 0;
  double* d_tmp = nullptr;        // small scratch for per-call outputs
  double* d_l1 = nullptr;         // level-1 rows of the diagnostic reduction
  int l1_blocks = 148;
  int* d_err = nullptr;
  int* h_err = nullptr;           // pinned
  int64_t edge_total = 0;
  // measurement: per-kernel CUDA events on the handle's stream and launch counts
  bool prof = false;
  std::vector<cudaEvent_t> ev;
  size_t ev_used = 0;
  std::vector<std::pair<int, size_t>> marks;
  int64_t launches[FELIS_KERNEL_KINDS] = {0};
  double last_run_ms = 0.0;
  // fused-step state
  bool prep_valid = false;        // deposit records match particles + lattice
  bool diag_valid = false;        // hist row for the next iteration already written
  int diag_iter = -1;
  bool capturing = false;
  // slice sharding across processes: the shift leaves the plane that becomes
  // the first slice holding the old last slice, for the caller to exchange
  bool exchange = false;
};

namespace {

// Brackets one kernel launch: counts it and, when profiling, records CUDA
// events around it on the handle's stream (event nodes when captured).
struct KernelScope {
  felis_handle* h;
  int kind;
  size_t slot = (size_t)-1;
  KernelScope(felis_handle* hh, int k) : h(hh), kind(k) {
    h->launches[k] += 1;
    if (h->prof && h->ev_used + 2 <= h->ev.size()) {
      slot = h->ev_used;
      h->ev_used += 2;
      cudaEventRecordWithFlags(h->ev[slot], h->st, h->capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
    }
  }
  ~KernelScope() {
    if (slot != (size_t)-1) {
      cudaEventRecordWithFlags(h->ev[slot + 1], h->st, h->capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
      h->marks.emplace_back(kind, slot);
    }
  }
};

#define CK(call)                                                                     \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      h->err = std::string(#call) + ": " + cudaGetErrorString(e_);                   \
      return FELIS_CUDA_ERROR;                                                       \
    }                                                                                \
  } while (0)

felis_status fail(felis_handle* h, felis_status s, const std::string& m) {
  if (h) h->err = m;
  return s;
}

// updateK_quadG.cpp:8-94 on the host.
void update_lattice(felis_handle* h, int iteration, double half) {
  felis_lattice& D = h->lat;
  const double dz = h->p.dz;
  const double z = (iteration + half) * dz;
  double K0 = D.K0, ue = D.ue, lambdaU = D.lambdaU;
  int K0_alpha = D.K0_alpha, undType = D.und_type;
  bool inUnd = false, inInter = false, airPosition = false;
  D.current_flag = 0;
  D.drift_flag = 0;
  for (const HostUnd& UL : h->und)
    for (size_t n = 0; n < UL.unitStart.size(); ++n) {
      if (z >= UL.unitStart[n] && z < UL.unitEnd[n]) {
        if (z >= UL.undStart[n] && z < UL.undEnd[n]) {
          inUnd = true;
          K0 = UL.K0[n] * (1 + UL.slopeK * (z - UL.undStart[n]));
          K0_alpha = UL.K0_alpha;
          ue = UL.ue;
          undType = UL.type;
          lambdaU = UL.lambdaU;
        } else {
          inInter = true;
          if (UL.air) airPosition = true;
        }
      }
    }
  D.K0 = K0;
  D.ue = ue;
  D.K0_alpha = K0_alpha;
  D.lambdaU = lambdaU;
  D.ku = 2 * M_PI / lambdaU;
  D.und_type = undType;
  if (K0 == 0.0) airPosition = true;
  if (!inUnd && !inInter) airPosition = true;
  if (inUnd) D.current_flag = 1;
  if (airPosition) {
    D.ku = 0.0;
    D.drift_flag = 1;
    D.current_flag = 0;
  }
  double g = 0;
  const double x0 = z, x1 = z + dz * 0.5;
  for (const HostQuad& QD : h->quad)
    for (int n = 0; n < QD.numbers; ++n) {
      const double q0 = QD.qdStart[n], q1 = QD.qdEnd[n];
      if (q1 <= x0 || q0 >= x1) continue;
      if (x0 < q0 && q1 < x1) g = (q1 - q0) / dz * 2.0 * QD.g[n];
      else if (x0 < q0 && q0 < x1) g = (x1 - q0) / dz * 2.0 * QD.g[n];
      else if (x0 < q1 && q1 < x1) g = (q1 - x0) / dz * 2.0 * QD.g[n];
      else g = 1.0 * QD.g[n];
      break;
    }
  D.g = g;
}

// Phi, eta of particlePush.cpp:222-238 (C library, as the CPU restatement).
bool polarisation(const felis_lattice& L, double* Phi, cd* etaX, cd* etaY) {
  const double ue = L.ue;
  const double re = (1.0 - ue * ue + 0.0 * ue) / (1.0 + ue * ue);
  const double im = (2.0 * ue) / (1.0 + ue * ue);
  *Phi = atan2(im, re);
  if (L.K0_alpha == 1) {
    *etaX = C(cos(*Phi * 0.5), 0.0);
    *etaY = C(0.0, sin(*Phi * 0.5));
  } else if (L.K0_alpha == -1) {
    *etaX = C(0.0, sin(*Phi * 0.5));
    *etaY = C(cos(*Phi * 0.5), 0.0);
  } else {
    return false;
  }
  return true;
}

// particlePush.cpp:42-68
bool trans_coef(const felis_handle* h, const felis_lattice& L, TransCoef* t) {
  t->dz = h->p.dz * 0.5;
  t->ku = L.ku;
  t->K0 = L.K0;
  t->ue = L.ue;
  t->aa = L.K0 * L.K0 * 0.25 * L.ue * L.ku;
  t->bb = L.K0 * L.K0 * 0.25 * (1.0 + L.ue * L.ue) * L.ku * L.ku;
  t->cc = K_ECHARGE * L.g / K_EMASS / K_VELOCITYC;
  t->xCoef = 0.0;
  t->yCoef = 0.0;
  t->K0_alpha = L.K0_alpha;
  t->valid = 1;
  if (L.und_type == FELIS_BIPOLAR) {
    if (L.K0_alpha == 1) { t->xCoef = 1; t->yCoef = 0; }
    else if (L.K0_alpha == -1) { t->xCoef = 0; t->yCoef = 1; }
  } else if (L.und_type == FELIS_QUADPOLAR) {
    t->xCoef = 1; t->yCoef = 1;
  } else {
    return false;
  }
  return true;
}

bool push_coef(const felis_handle* h, const felis_lattice& L, PushCoef* c) {
  c->dz = h->p.dz;
  c->ku = L.ku;
  c->ks = h->p.ks;
  c->K0 = L.K0;
  c->ue = L.ue;
  c->K0_alpha = L.K0_alpha;
  c->dPhi = 2 * M_PI * h->p.num_slice;
  c->e_mc2 = K_ECHARGE / K_EMASS / K_VELOCITYC / K_VELOCITYC;
  c->gamR = h->p.gam_r;
  return polarisation(L, &c->Phi, &c->etaX, &c->etaY);
}

// solveField.cpp:209-243
bool prep_coef(const felis_handle* h, const felis_lattice& L, PrepCoef* c) {
  const double K0 = L.K0, ue = L.ue, ks = h->p.ks;
  c->K0 = K0;
  c->ue = ue;
  c->K0_alpha = L.K0_alpha;
  cd ex, ey;
  if (!polarisation(L, &c->Phi, &ex, &ey)) return false;
  c->coef_U = h->p.dz * K_ECHARGE * K_ECHARGE * K_MU0 * K0 * sqrt(1.0 + ue * ue) /
              (4.0 * ks * K_EMASS * (h->p.lambda0 * h->p.num_slice) * h->p.dx * h->p.dy);
  c->xi = 0.25 * K0 * K0 * (1.0 - ue * ue) / (1.0 + (1.0 + ue * ue) * K0 * K0 * 0.5);
  c->coef_Ez = K_ECHARGE * K_VELOCITYC * K_VELOCITYC * K_MU0 * ks * (1.0 + 0.5 * (1.0 + ue * ue) * K0 * K0) /
               (2.0 * M_PI * h->p.lambda0 * h->p.num_slice * h->p.gam_r * h->p.gam_r);
  return true;
}

// ADI coefficient tables of one harmonic (solveField.cpp:112-181).
void build_adi(felis_handle* h, int hidx, const std::vector<cd>& al, const std::vector<cd>& alP,
               const std::vector<cd>& be, const std::vector<cd>& beP, std::vector<cd>& cv, std::vector<double>& dv,
               size_t offs_c[14], size_t offs_d[6]) {
  const int nx = h->p.nx, ny = h->p.ny;
  const double H = (double)h->p.harmony[hidx];
  // layout: complex arrays rx_m, rx_0, rx_p (ny), ax_p, ax_a, ax_q, ax_cc (nx),
  //         ry_m, ry_0, ry_p (nx), ay_p, ay_a, ay_q, ay_cc (ny)
  const int sizes_c[14] = {ny, ny, ny, nx, nx, nx, nx, nx, nx, nx, ny, ny, ny, ny};
  size_t o = 0;
  for (int k = 0; k < 14; ++k) { offs_c[k] = o; o += sizes_c[k]; }
  cv.assign(o, C(0, 0));
  const int sizes_d[6] = {nx, nx, nx, ny, ny, ny};  // ax_pinv, ax_qinv, ax_ccinv, ay_*
  o = 0;
  for (int k = 0; k < 6; ++k) { offs_d[k] = o; o += sizes_d[k]; }
  dv.assign(o, 0.0);
  cd* rx_m = &cv[offs_c[0]]; cd* rx_0 = &cv[offs_c[1]]; cd* rx_p = &cv[offs_c[2]];
  cd* ax_p = &cv[offs_c[3]]; cd* ax_a = &cv[offs_c[4]]; cd* ax_q = &cv[offs_c[5]]; cd* ax_cc = &cv[offs_c[6]];
  cd* ry_m = &cv[offs_c[7]]; cd* ry_0 = &cv[offs_c[8]]; cd* ry_p = &cv[offs_c[9]];
  cd* ay_p = &cv[offs_c[10]]; cd* ay_a = &cv[offs_c[11]]; cd* ay_q = &cv[offs_c[12]]; cd* ay_cc = &cv[offs_c[13]];
  double* ax_pinv = &dv[offs_d[0]]; double* ax_qinv = &dv[offs_d[1]]; double* ax_ccinv = &dv[offs_d[2]];
  double* ay_pinv = &dv[offs_d[3]]; double* ay_qinv = &dv[offs_d[4]]; double* ay_ccinv = &dv[offs_d[5]];
  for (int j = 1; j < ny - 1; ++j) {
    rx_m[j] = cneg(beP[j]);
    rx_0[j] = cadd(cradd(H, beP[j]), be[j]);
    rx_p[j] = be[j];
  }
  for (int i = 1; i < nx - 1; ++i) {
    ry_m[i] = cneg(alP[i]);
    ry_0[i] = cadd(cradd(H, alP[i]), al[i]);
    ry_p[i] = al[i];
  }
  // x recurrence
  std::vector<cd> CC(nx, C(0, 0));
  CC[1] = cdiv(csub(crsub(H, alP[1]), al[1]), alP[1]);
  for (int i = 2; i < nx - 2; ++i) {
    const cd Hx = csub(crsub(H, alP[i]), al[i]);
    const cd Q = cmul(alP[i], CC[i - 1]);
    CC[i] = csub(cdiv(Hx, alP[i]), cdiv(al[i], Q));
    ax_q[i] = Q;
    ax_qinv[i] = cinvnorm(Q);
  }
  CC[nx - 2] = csub(csub(crsub(H, alP[nx - 2]), al[nx - 2]), cdiv(C(1.0, 0.0), CC[nx - 3]));
  for (int i = 1; i < nx - 1; ++i) {
    ax_p[i] = alP[i];
    ax_pinv[i] = cinvnorm(alP[i]);
    ax_a[i] = al[i];
    ax_cc[i] = CC[i];
    ax_ccinv[i] = cinvnorm(CC[i]);
  }
  // y recurrence (the reference's loop runs to ny-2, then overwrites ny-2)
  std::vector<cd> CY(ny, C(0, 0));
  CY[1] = cdiv(csub(crsub(H, beP[1]), be[1]), beP[1]);
  for (int j = 2; j < ny - 1; ++j) {
    const cd Hy = csub(crsub(H, beP[j]), be[j]);
    const cd Q = cmul(beP[j], CY[j - 1]);
    CY[j] = csub(cdiv(Hy, beP[j]), cdiv(be[j], Q));
    ay_q[j] = Q;
    ay_qinv[j] = cinvnorm(Q);
  }
  CY[ny - 2] = csub(csub(crsub(H, beP[ny - 2]), be[ny - 2]), cdiv(C(1.0, 0.0), CY[ny - 3]));
  for (int j = 1; j < ny - 1; ++j) {
    ay_p[j] = beP[j];
    ay_pinv[j] = cinvnorm(beP[j]);
    ay_a[j] = be[j];
    ay_cc[j] = CY[j];
    ay_ccinv[j] = cinvnorm(CY[j]);
  }
}

felis_status check_err(felis_handle* h) {
  if (h->capturing) return FELIS_OK;
  CK(cudaMemcpyAsync(h->h_err, h->d_err, ERR_SLOTS * sizeof(int), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  const int* e = h->h_err;
  felis_status s = FELIS_OK;
  if (e[ERR_EDGE_DEPOSIT]) {
    h->edge_total += e[ERR_EDGE_DEPOSIT];
  }
  if (e[ERR_THETA_OVERFLOW]) s = fail(h, FELIS_THETA_OVERFLOW, "push_theta_gamma: |dtheta| > 2 pi numSlice");
  else if (e[ERR_OUT_OF_RANGE]) s = fail(h, FELIS_OUT_OF_RANGE, "periodicParticles: theta outside [0, dTh]");
  else if (e[ERR_NAN]) s = fail(h, FELIS_NAN, "non-finite particle state");
  else if (e[ERR_RADIAL]) s = fail(h, FELIS_UNSUPPORTED, "particle outside the radial Ez grid or the Bessel table");
  else if (e[ERR_DEPOSIT_CAPACITY]) s = fail(h, FELIS_UNSUPPORTED, "slice holds more particles than the deposit sort");
  else if (e[ERR_TIMEOUT]) s = fail(h, FELIS_TIMEOUT, "a bounded device wait ran out");
  if (e[ERR_EDGE_DEPOSIT] || s != FELIS_OK) CK(cudaMemsetAsync(h->d_err, 0, ERR_SLOTS * sizeof(int), h->st));
  return s;
}

ParticleLaunch base_launch(felis_handle* h) {
  ParticleLaunch a{};
  a.G = h->G;
  a.P.x = h->x; a.P.y = h->y; a.P.px = h->px; a.P.py = h->py; a.P.th = h->th; a.P.ga = h->ga;
  a.P.soff = h->d_soff;
  a.P.weight = h->d_weight;
  a.P.tiles = h->d_tiles;
  a.P.ntiles = (int)h->tiles.size();
  a.P.total = h->total;
  a.U = h->U;
  a.ring_base = h->ring_base;
  a.Ez = h->Ez;
  a.dep = h->dep;
  a.diag = h->d_part;
  a.diag_stride = h->diag_stride;
  a.err = h->d_err;
  return a;
}

felis_status ensure_ready(felis_handle* h) {
  for (int s = 0; s < h->p.num_species; ++s)
    if (!h->uploaded[s]) return fail(h, FELIS_BAD_ARG, "particles of every species must be uploaded first");
  return FELIS_OK;
}

double theta_shift(const felis_handle* h, int it) {
  return phase_shift_of((int)h->ps_z.size(), h->ps_z.data(), h->ps_phase.data(), it, h->p.dz);
}

felis_status run_particles(felis_handle* h, unsigned ops, const felis_lattice* l0, const felis_lattice* l1,
                           double shift = 0.0) {
  ParticleLaunch a = base_launch(h);
  a.ops = ops;
  a.theta_shift = shift;
  if (ops & OP_T0)
    if (!trans_coef(h, *l0, &a.t0)) return fail(h, FELIS_BAD_ARG, "transversePush: no undulator_mode");
  if (ops & OP_T1)
    if (!trans_coef(h, *l1, &a.t1)) return fail(h, FELIS_BAD_ARG, "transversePush: no undulator_mode");
  if (ops & (OP_PUSH | OP_DRIFT))
    if (!push_coef(h, *l1, &a.pc)) return fail(h, FELIS_BAD_ARG, "invalid K0_alpha");
  if (ops & OP_PREP)
    if (!prep_coef(h, *l1, &a.prep)) return fail(h, FELIS_BAD_ARG, "invalid K0_alpha");
  {
    KernelScope ks(h, FELIS_KERNEL_PARTICLES);
    launch_particles(a, h->st);
  }
  CK(cudaGetLastError());
  return FELIS_OK;
}

felis_status run_deposit(felis_handle* h, const felis_lattice& L) {
  DepositLaunch d{};
  d.G = h->G;
  d.dep = h->dep;
  d.soff = h->d_soff;
  d.total = h->total;
  d.Sc = h->Sc;
  d.box = h->box;
  d.Ez = h->Ez;
  PrepCoef pc;
  if (!prep_coef(h, L, &pc)) return fail(h, FELIS_BAD_ARG, "invalid K0_alpha");
  double Phi;
  if (!polarisation(L, &Phi, &d.etaX, &d.etaY)) return fail(h, FELIS_BAD_ARG, "invalid K0_alpha");
  // odd-harmonic fx, fy (solveField.cpp:277-287) with the constant xi
  for (int hh = 0; hh < h->p.num_harmony; ++hh) {
    const int H = h->p.harmony[hh];
    d.fconst[hh][0] = make_double2(0, 0);
    d.fconst[hh][1] = make_double2(0, 0);
    if (H % 2 == 1) {
      const double dbH = (double)H;
      const double sign = ((H - 1) / 2 % 2 == 0) ? 1.0 : -1.0;
      const int ib0 = (dbH * pc.xi) / h->p.d_bessel;
      double w[2];
      w[1] = (dbH * pc.xi / h->p.d_bessel) - ib0;
      w[0] = 1.0 - w[1];
      const int ib = std::max(0, std::min(ib0, h->p.bessel_rows - 1));
      const int ib1 = std::max(0, std::min(ib0 + 1, h->p.bessel_rows - 1));
      const double* B = h->p.bessel;
      const int bc = h->p.bessel_cols;
      int order = (H - 1) / 2;
      const double J1 = B[(size_t)ib * bc + order] * w[0] + B[(size_t)ib1 * bc + order] * w[1];
      order = (H + 1) / 2;
      const double J2 = B[(size_t)ib * bc + order] * w[0] + B[(size_t)ib1 * bc + order] * w[1];
      const double K0a = L.K0_alpha;
      d.fconst[hh][0] = make_double2(sign * (J1 - K0a * J2), 0.0);
      d.fconst[hh][1] = make_double2(sign * (J1 + K0a * J2), 0.0);
    }
  }
  const double ks = h->p.ks, ue = L.ue, K0 = L.K0, gamR = h->p.gam_r, dr = h->p.dr;
  d.A = ks * ks * (1.0 + 0.5 * (1.0 + ue * ue) * K0 * K0) / (gamR * gamR) * dr * dr;
  d.cap = h->dep_pcap;
  d.neven = 0;
  for (int k = 0; k < h->p.num_harmony; ++k) d.neven += (h->p.harmony[k] % 2 == 0);
  d.err = h->d_err;
  {
    KernelScope ks(h, FELIS_KERNEL_DEPOSIT);
    launch_deposit(d, h->st);
  }
  CK(cudaGetLastError());
  return FELIS_OK;
}

felis_status run_adi(felis_handle* h, int use_source) {
  AdiLaunch a{};
  a.G = h->G;
  a.U = h->U;
  a.ring_base = h->ring_base;
  a.Sc = h->Sc;
  a.box = h->box;
  a.use_source = use_source;
  a.tab = h->d_adi;
  a.energy = h->d_planes;
  a.nxp = h->nxp;
  a.scratch = h->adi_scratch;
  a.err = h->d_err;
  {
    KernelScope ks(h, FELIS_KERNEL_ADI);
    if (h->adi_scratch) launch_adi_big(a, h->adi_big_grid, h->st);
    else launch_adi(a, h->st);
  }
  CK(cudaGetLastError());
  return FELIS_OK;
}

felis_status do_shift(felis_handle* h) {
  const int S = h->p.slice_n;
  h->ring_base = ((h->ring_base - 1) % S + S) % S;
  const size_t N = (size_t)h->p.nx * h->p.ny;
  if (h->exchange) return FELIS_OK;  // fieldShareZ.cpp:39-78 fills it
  KernelScope ks(h, FELIS_KERNEL_SHIFT);
  for (int hh = 0; hh < h->p.num_harmony; ++hh)
    for (int pol = 0; pol < 2; ++pol)
      CK(cudaMemsetAsync(h->U + field_plane(S, hh, pol, 0, h->ring_base) * N, 0, N * sizeof(double2), h->st));
  return FELIS_OK;
}

void invalidate_particles(felis_handle* h) {
  h->prep_valid = false;
  h->diag_valid = false;
}

// Builds tiles, offsets and the deposit capacity after the particle layout changed.
felis_status relayout(felis_handle* h, const std::vector<int64_t>& new_counts_per_slice /*[ns][S]*/) {
  const int S = h->p.slice_n, ns = h->p.num_species;
  std::vector<int64_t> soff((size_t)ns * (S + 1));
  int64_t base = 0;
  for (int sp = 0; sp < ns; ++sp) {
    soff[(size_t)sp * (S + 1)] = base;
    for (int s = 0; s < S; ++s) {
      base += new_counts_per_slice[(size_t)sp * S + s];
      soff[(size_t)sp * (S + 1) + s + 1] = base;
    }
  }
  const int64_t total = base;
  if (total != h->total || h->x == nullptr) {
    double** arrs[6] = {&h->x, &h->y, &h->px, &h->py, &h->th, &h->ga};
    for (auto a : arrs) {
      if (*a) cudaFree(*a);
      *a = nullptr;
      CK(cudaMalloc(a, std::max<int64_t>(total, 1) * sizeof(double)));
    }
    for (int sp = 0; sp < ns; ++sp) h->uploaded[sp] = 0;
    h->total = total;
  }
  h->soff = soff;
  // tiles
  h->tiles.clear();
  int64_t maxslice = 0;
  for (int s = 0; s < S; ++s) {
    int64_t c = 0;
    for (int sp = 0; sp < ns; ++sp) c += soff[(size_t)sp * (S + 1) + s + 1] - soff[(size_t)sp * (S + 1) + s];
    maxslice = std::max(maxslice, c);
  }
  for (int sp = 0; sp < ns; ++sp)
    for (int s = 0; s < S; ++s) {
      const int64_t b = soff[(size_t)sp * (S + 1) + s], e = soff[(size_t)sp * (S + 1) + s + 1];
      for (int64_t t = b; t < e; t += 256) h->tiles.push_back(make_int4(sp, s, (int)t, (int)std::min<int64_t>(t + 256, e)));
    }
  if (total >= (int64_t)1 << 31) return fail(h, FELIS_UNSUPPORTED, "more than 2^31 particles per handle");
  if (h->d_soff) cudaFree(h->d_soff);
  if (h->d_tiles) cudaFree(h->d_tiles);
  if (h->d_part) cudaFree(h->d_part);
  h->d_soff = nullptr; h->d_tiles = nullptr; h->d_part = nullptr;
  CK(cudaMalloc(&h->d_soff, soff.size() * sizeof(int64_t)));
  CK(cudaMemcpy(h->d_soff, soff.data(), soff.size() * sizeof(int64_t), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&h->d_tiles, std::max<size_t>(h->tiles.size(), 1) * sizeof(int4)));
  if (!h->tiles.empty())
    CK(cudaMemcpy(h->d_tiles, h->tiles.data(), h->tiles.size() * sizeof(int4), cudaMemcpyHostToDevice));
  CK(cudaMalloc(&h->d_part, std::max<size_t>(h->tiles.size(), 1) * h->diag_stride * sizeof(double)));
  // deposit records
  if (total > h->dep_cap) {
    void* ptrs[] = {h->dep.key, h->dep.rkey, h->dep.wx1, h->dep.wy1, h->dep.wr1, h->dep.coef, h->dep.fx, h->dep.fy, h->dep.ez};
    for (void* q : ptrs) if (q) cudaFree(q);
    h->dep = DevDeposit{};
    const size_t n = std::max<int64_t>(total, 1);
    const int H = h->p.num_harmony, LF = h->p.scl_mode * h->p.scf_mode;
    CK(cudaMalloc(&h->dep.key, n * sizeof(int)));
    CK(cudaMalloc(&h->dep.rkey, n * sizeof(int)));
    CK(cudaMalloc(&h->dep.wx1, n * sizeof(double)));
    CK(cudaMalloc(&h->dep.wy1, n * sizeof(double)));
    CK(cudaMalloc(&h->dep.wr1, n * sizeof(double)));
    CK(cudaMalloc(&h->dep.coef, n * H * sizeof(double2)));
    if (h->has_even) {
      CK(cudaMalloc(&h->dep.fx, n * H * sizeof(double2)));
      CK(cudaMalloc(&h->dep.fy, n * H * sizeof(double2)));
    }
    CK(cudaMalloc(&h->dep.ez, n * LF * sizeof(double2)));
    h->dep_cap = n;
  }
  // deposit chunk: the largest power of two (<= 4096 particles) whose sort
  // buffers and records fit in ~100 KB of shared memory (two CTAs per SM)
  int dev_smem = 0;
  cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
  const size_t budget = std::min<size_t>(100 * 1024, (size_t)dev_smem);
  const int H = h->p.num_harmony, Lm = h->p.scl_mode, Fm = h->p.scf_mode, nr = h->p.nr;
  int neven = 0;
  for (int k = 0; k < H; ++k) neven += (h->p.harmony[k] % 2 == 0);
  int cap = 4096;
  while (cap > 64 && deposit_smem_bytes(cap, H, neven, Lm, Fm, nr) > budget) cap >>= 1;
  const size_t smem = deposit_smem_bytes(cap, H, neven, Lm, Fm, nr);
  if ((int)smem > dev_smem) return fail(h, FELIS_UNSUPPORTED, "deposit buffers do not fit in shared memory");
  int qb = 0;
  while ((1 << qb) < cap) ++qb;
  int kb = 0;
  while ((1 << kb) < h->p.nx * h->p.ny + 1) ++kb;
  if (kb + qb > 32) return fail(h, FELIS_UNSUPPORTED, "grid too large for 32-bit deposit keys");
  deposit_set_smem(smem);
  h->dep_pcap = cap;
  (void)maxslice;
  invalidate_particles(h);
  return FELIS_OK;
}

}  // namespace

extern "C" {

const char* felis_last_error(const felis_handle* h) { return h ? h->err.c_str() : "null handle"; }

felis_status felis_device_info(char* name, size_t name_len, int32_t* sm_count) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return FELIS_NO_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, 0) != cudaSuccess) return FELIS_CUDA_ERROR;
  if (name && name_len) snprintf(name, name_len, "%s", prop.name);
  if (sm_count) *sm_count = prop.multiProcessorCount;
  return FELIS_OK;
}

felis_status felis_create(const felis_params* p, felis_handle** out) {
  if (!p || !out) return FELIS_BAD_ARG;
  *out = nullptr;
  if (p->abi_version != FELIS_ABI_VERSION) return FELIS_BAD_ARG;
  if (p->dimension != 3 && p->dimension != 1) return FELIS_UNSUPPORTED;
  if (p->precision != FELIS_FP64) return FELIS_UNSUPPORTED;
  const bool one_d = p->dimension == 1;
  if (p->num_harmony < 1 || p->num_harmony > FELIS_MAX_HARMONY || p->num_species < 1 ||
      p->num_species > FELIS_MAX_SPECIES || p->slice_n < 1 || p->scl_mode < 1 || p->scf_mode < 1 ||
      p->scl_mode * p->scf_mode > 16 || p->scl_mode > 4 || p->bessel_rows < 2 || p->bessel_cols < 1 ||
      !p->bessel || p->num_undulators < 0 || (p->num_undulators > 0 && !p->undulators))
    return FELIS_BAD_ARG;
  if (one_d ? (p->nx != 1 || p->ny != 1 || p->nr != 1 || p->scf_mode != 1)
            : (p->nx < 4 || p->ny < 4 || p->nr < 3 || !p->abc_alpha || !p->abc_alpha_p || !p->abc_beta ||
               !p->abc_beta_p))
    return FELIS_BAD_ARG;
  if (one_d)
    for (int s = 0; s < p->num_species; ++s)
      if (!(p->beam_area[s] > 0.0)) return FELIS_BAD_ARG;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FELIS_NO_DEVICE;
  felis_handle* h = new felis_handle();
  h->p = *p;
  // own copies of the arrays felis_params points to
  const int nx = p->nx, ny = p->ny, S = p->slice_n, H = p->num_harmony;
  for (int u = 0; u < p->num_undulators; ++u) {
    const felis_undulator& U = p->undulators[u];
    HostUnd o;
    o.type = U.type; o.K0_alpha = U.K0_alpha; o.numbers = U.numbers; o.air = U.air;
    o.lambdaU = U.lambdaU; o.slopeK = U.slopeK; o.ue = U.ue;
    o.unitStart.assign(U.unit_start, U.unit_start + U.numbers);
    o.unitEnd.assign(U.unit_end, U.unit_end + U.numbers);
    o.undStart.assign(U.und_start, U.und_start + U.numbers);
    o.undEnd.assign(U.und_end, U.und_end + U.numbers);
    o.K0.assign(U.K0, U.K0 + U.numbers);
    h->und.push_back(o);
  }
  for (int q = 0; q < p->num_quads; ++q) {
    const felis_quad& Q = p->quads[q];
    HostQuad o;
    o.numbers = Q.numbers;
    o.qdStart.assign(Q.qd_start, Q.qd_start + Q.numbers);
    o.qdEnd.assign(Q.qd_end, Q.qd_end + Q.numbers);
    o.g.assign(Q.g, Q.g + Q.numbers);
    h->quad.push_back(o);
  }
  if (p->num_phase_shifts > 0) {
    h->ps_z.assign(p->phase_shift_z, p->phase_shift_z + p->num_phase_shifts);
    h->ps_phase.assign(p->phase_shift_phase, p->phase_shift_phase + p->num_phase_shifts);
  }
  h->p.num_phase_shifts = (int32_t)h->ps_z.size();
  h->p.phase_shift_z = nullptr;
  h->p.phase_shift_phase = nullptr;
  h->p.undulators = nullptr;
  h->p.quads = nullptr;
  h->bessel_host.assign(p->bessel, p->bessel + (size_t)p->bessel_rows * p->bessel_cols);
  h->p.bessel = h->bessel_host.data();  // host copy for the odd-harmonic constants
  h->lat.K0 = p->K0_init;
  h->lat.ue = p->ue_init;
  h->lat.lambdaU = p->lambdaU_init;
  h->lat.ku = 2.0 * M_PI / p->lambdaU_init;
  h->lat.g = 0.0;
  h->lat.K0_alpha = p->K0_alpha_init;
  h->lat.und_type = p->und_type_init;
  h->lat.current_flag = 0;
  h->lat.drift_flag = 0;
  h->counts.assign(p->num_species, 0);
  h->uploaded.assign(p->num_species, 0);
  h->weight.assign((size_t)p->num_species * S, 0.0);
  for (int k = 0; k < H; ++k) h->has_even |= (p->harmony[k] % 2 == 0);
  h->diag_stride = 7 + 2 * H + 1;
  felis_status st = FELIS_OK;
  auto bail = [&](felis_status s, const char* m) {
    st = s;
    h->err = m;
  };
  cudaError_t ce = cudaGetDevice(&h->device);
  if (ce == cudaSuccess) cudaDeviceGetAttribute(&h->sms, cudaDevAttrMultiProcessorCount, h->device);
  if (ce == cudaSuccess) ce = cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking);
  const size_t N = (size_t)nx * ny;
  if (ce == cudaSuccess) ce = cudaMalloc(&h->U, (size_t)H * 2 * S * N * sizeof(double2));
  if (ce == cudaSuccess) ce = cudaMemsetAsync(h->U, 0, (size_t)H * 2 * S * N * sizeof(double2), h->st);
  if (ce == cudaSuccess) ce = cudaMalloc(&h->Sc, (size_t)H * 2 * S * N * sizeof(double2));
  if (ce == cudaSuccess) ce = cudaMalloc(&h->box, (size_t)S * sizeof(int4));
  const size_t ezn = (size_t)p->scl_mode * (S + 2) * p->scf_mode * p->nr;
  if (ce == cudaSuccess) ce = cudaMalloc(&h->Ez, ezn * sizeof(double2));
  if (ce == cudaSuccess) ce = cudaMemsetAsync(h->Ez, 0, ezn * sizeof(double2), h->st);
  if (ce == cudaSuccess) ce = cudaMalloc(&h->d_bessel, (size_t)p->bessel_rows * p->bessel_cols * sizeof(double));
  if (ce == cudaSuccess) ce = cudaMemcpy(h->d_bessel, p->bessel, (size_t)p->bessel_rows * p->bessel_cols * sizeof(double), cudaMemcpyHostToDevice);
  std::vector<double> wake(std::max(p->global_slice_n, 1), 0.0);
  h->p.wake_e = nullptr;
  h->p.abc_alpha = h->p.abc_alpha_p = h->p.abc_beta = h->p.abc_beta_p = nullptr;
  if (p->wake_e) std::copy(p->wake_e, p->wake_e + p->global_slice_n, wake.begin());
  if (ce == cudaSuccess) ce = cudaMalloc(&h->d_wake, wake.size() * sizeof(double));
  if (ce == cudaSuccess) ce = cudaMemcpy(h->d_wake, wake.data(), wake.size() * sizeof(double), cudaMemcpyHostToDevice);
  std::vector<double> logtab(p->nr, 0.0);
  for (int j = 1; j < p->nr; ++j) logtab[j] = log((j + 0.5) / (j - 0.5));
  if (ce == cudaSuccess) ce = cudaMalloc(&h->d_log, logtab.size() * sizeof(double));
  if (ce == cudaSuccess) ce = cudaMemcpy(h->d_log, logtab.data(), logtab.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (ce == cudaSuccess) ce = cudaMalloc(&h->d_planes, (size_t)H * 2 * S * sizeof(double));
  if (ce == cudaSuccess) ce = cudaMalloc(&h->d_planes2, (size_t)H * 2 * S * sizeof(double));
  h->hist_n = std::max(p->max_step, 1) + 1;
  if (ce == cudaSuccess) ce = cudaMalloc(&h->d_hist_e, (size_t)h->hist_n * 2 * H * sizeof(double));
  if (ce == cudaSuccess) ce = cudaMalloc(&h->d_hist_t, (size_t)h->hist_n * 6 * p->num_species * sizeof(double));
  if (ce == cudaSuccess) ce = cudaMalloc(&h->d_hist_b, (size_t)h->hist_n * 2 * H * sizeof(double));
  if (ce == cudaSuccess) ce = cudaMalloc(&h->d_tmp, (size_t)(6 * FELIS_MAX_SPECIES + 4 * FELIS_MAX_HARMONY) * sizeof(double));
  if (ce == cudaSuccess) ce = cudaMalloc(&h->d_l1, (size_t)h->l1_blocks * (7 * FELIS_MAX_SPECIES + 2 * FELIS_MAX_HARMONY + 1) * sizeof(double));
  if (ce == cudaSuccess) ce = cudaMalloc(&h->d_err, ERR_SLOTS * sizeof(int));
  if (ce == cudaSuccess) ce = cudaMemsetAsync(h->d_err, 0, ERR_SLOTS * sizeof(int), h->st);
  if (ce == cudaSuccess) ce = cudaMallocHost(&h->h_err, ERR_SLOTS * sizeof(int));
  if (ce != cudaSuccess) {
    bail(FELIS_CUDA_ERROR, cudaGetErrorString(ce));
  }
  // ADI tables (3D; the 1D field has no transverse operator)
  if (st == FELIS_OK && one_d) {
    if (cudaMemsetAsync(h->box, 0, (size_t)S * sizeof(int4), h->st) != cudaSuccess ||
        cudaMemsetAsync(h->Sc, 0, (size_t)H * 2 * S * sizeof(double2), h->st) != cudaSuccess)
      bail(FELIS_CUDA_ERROR, "1D buffers");
  }
  if (st == FELIS_OK && !one_d) {
    std::vector<cd> al(nx), alP(nx), be(ny), beP(ny);
    for (int i = 0; i < nx; ++i) { al[i] = C(p->abc_alpha[2 * i], p->abc_alpha[2 * i + 1]); alP[i] = C(p->abc_alpha_p[2 * i], p->abc_alpha_p[2 * i + 1]); }
    for (int j = 0; j < ny; ++j) { be[j] = C(p->abc_beta[2 * j], p->abc_beta[2 * j + 1]); beP[j] = C(p->abc_beta_p[2 * j], p->abc_beta_p[2 * j + 1]); }
    std::vector<AdiTab> tabs(H);
    for (int k = 0; k < H && st == FELIS_OK; ++k) {
      std::vector<cd> cv;
      std::vector<double> dv;
      size_t oc[14], od[6];
      build_adi(h, k, al, alP, be, beP, cv, dv, oc, od);
      cd* dc = nullptr;
      double* dd = nullptr;
      if (cudaMalloc(&dc, cv.size() * sizeof(cd)) != cudaSuccess || cudaMalloc(&dd, dv.size() * sizeof(double)) != cudaSuccess ||
          cudaMemcpy(dc, cv.data(), cv.size() * sizeof(cd), cudaMemcpyHostToDevice) != cudaSuccess ||
          cudaMemcpy(dd, dv.data(), dv.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
        bail(FELIS_CUDA_ERROR, "ADI table upload failed");
        break;
      }
      h->adi_dev.push_back(dc);
      h->adi_dev.push_back(dd);
      AdiTab& T = tabs[k];
      T.rx_m = dc + oc[0]; T.rx_0 = dc + oc[1]; T.rx_p = dc + oc[2];
      T.ax_p = dc + oc[3]; T.ax_a = dc + oc[4]; T.ax_q = dc + oc[5]; T.ax_cc = dc + oc[6];
      T.ry_m = dc + oc[7]; T.ry_0 = dc + oc[8]; T.ry_p = dc + oc[9];
      T.ay_p = dc + oc[10]; T.ay_a = dc + oc[11]; T.ay_q = dc + oc[12]; T.ay_cc = dc + oc[13];
      T.ax_pinv = dd + od[0]; T.ax_qinv = dd + od[1]; T.ax_ccinv = dd + od[2];
      T.ay_pinv = dd + od[3]; T.ay_qinv = dd + od[4]; T.ay_ccinv = dd + od[5];
    }
    if (st == FELIS_OK) {
      if (cudaMalloc(&h->d_adi, H * sizeof(AdiTab)) != cudaSuccess ||
          cudaMemcpy(h->d_adi, tabs.data(), H * sizeof(AdiTab), cudaMemcpyHostToDevice) != cudaSuccess)
        bail(FELIS_CUDA_ERROR, "ADI table upload failed");
    }
    h->nxp = nx | 1;
    const size_t smem = adi_smem_bytes(nx, ny, h->nxp);
    int dev_smem = 0;
    cudaDeviceGetAttribute(&dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device);
    if (st == FELIS_OK && (int)smem <= dev_smem - 1024) {
      adi_set_smem(smem);
    } else if (st == FELIS_OK) {
      // plane larger than shared memory: global-memory sweeps, one scratch
      // plane per CTA of a persistent grid
      h->adi_big_grid = std::min(S * H * 2, h->sms * 2);
      if (cudaMalloc(&h->adi_scratch, (size_t)h->adi_big_grid * nx * ny * sizeof(double2)) != cudaSuccess)
        bail(FELIS_CUDA_ERROR, "ADI scratch allocation failed");
    }
    if (st == FELIS_OK && std::max(nx, ny) > 256) bail(FELIS_UNSUPPORTED, "grid wider than 256 points");
  }
  // geometry
  DevGeom& G = h->G;
  G.S = S; G.nx = nx; G.ny = ny; G.N = nx * ny; G.H = H; G.L = p->scl_mode; G.F = p->scf_mode; G.nr = p->nr;
  G.bn = p->bessel_rows; G.bcols = p->bessel_cols; G.nspecies = p->num_species; G.numSlice = p->num_slice;
  G.minI = p->min_i; G.wakeOn = p->wake_on; G.mode = p->mode;
  for (int k = 0; k < FELIS_MAX_HARMONY; ++k) G.harmony[k] = k < H ? p->harmony[k] : 1;
  G.ks = p->ks; G.lambda0 = p->lambda0; G.dz = p->dz; G.dx = p->dx; G.dy = p->dy; G.dr = p->dr;
  G.minX = p->min_x; G.minY = p->min_y; G.gamR = p->gam_r; G.dBessel = p->d_bessel;
  G.bessel = h->d_bessel; G.wakeE = h->d_wake; G.logtab = h->d_log;
  if (st == FELIS_OK) {
    cudaStreamSynchronize(h->st);
  }
  if (st != FELIS_OK) {
    fprintf(stderr, "felis_create: %s\n", h->err.c_str());
    felis_destroy(h);
    return st;
  }
  *out = h;
  return FELIS_OK;
}

void felis_destroy(felis_handle* h) {
  if (!h) return;
  if (h->st) cudaStreamSynchronize(h->st);
  void* ptrs[] = {h->x, h->y, h->px, h->py, h->th, h->ga, h->d_soff, h->d_weight, h->d_tiles, h->U, h->Sc, h->box,
                  h->Ez, h->d_bessel, h->d_wake, h->d_log, h->d_adi, h->d_part, h->d_planes, h->d_planes2,
                  h->d_hist_e, h->d_hist_t, h->d_hist_b, h->d_tmp, h->d_l1, h->d_err,
                  h->dep.key, h->dep.rkey, h->dep.wx1, h->dep.wy1, h->dep.wr1, h->dep.coef, h->dep.fx, h->dep.fy, h->dep.ez,
                  h->adi_scratch};
  for (void* q : ptrs) if (q) cudaFree(q);
  for (void* q : h->adi_dev) if (q) cudaFree(q);
  if (h->h_err) cudaFreeHost(h->h_err);
  for (cudaEvent_t e : h->ev) cudaEventDestroy(e);
  if (h->st) cudaStreamDestroy(h->st);
  delete h;
}

felis_status felis_upload_particles(felis_handle* h, int32_t species, const double* x, const double* y,
                                    const double* px, const double* py, const double* theta, const double* gamma,
                                    const int64_t* slice_offsets, const double* weights) {
  if (!h || species < 0 || species >= h->p.num_species || !slice_offsets || !weights) return fail(h, FELIS_BAD_ARG, "bad argument");
  const int S = h->p.slice_n, ns = h->p.num_species;
  if (slice_offsets[0] != 0) return fail(h, FELIS_BAD_ARG, "slice_offsets[0] must be 0");
  for (int s = 0; s < S; ++s)
    if (slice_offsets[s + 1] < slice_offsets[s]) return fail(h, FELIS_BAD_ARG, "slice_offsets must be non-decreasing");
  const int64_t cnt = slice_offsets[S];
  if (cnt > 0 && (!x || !y || !px || !py || !theta || !gamma)) return fail(h, FELIS_BAD_ARG, "null particle array");
  // per-slice counts of every species (keep the others)
  std::vector<int64_t> per((size_t)ns * S, 0);
  for (int sp = 0; sp < ns; ++sp)
    for (int s = 0; s < S; ++s)
      per[(size_t)sp * S + s] = h->soff.empty() ? 0 : h->soff[(size_t)sp * (S + 1) + s + 1] - h->soff[(size_t)sp * (S + 1) + s];
  bool changed = h->soff.empty();
  for (int s = 0; s < S; ++s) {
    const int64_t c = slice_offsets[s + 1] - slice_offsets[s];
    if (per[(size_t)species * S + s] != c) changed = true;
    per[(size_t)species * S + s] = c;
  }
  if (changed) {
    // keep the data of the other species across the relayout
    std::vector<std::vector<double>> keep;
    std::vector<int> kept;
    for (int sp = 0; sp < ns; ++sp) {
      if (sp == species || !h->uploaded[sp] || !h->x) continue;
      const int64_t b = h->soff[(size_t)sp * (S + 1)], e = h->soff[(size_t)sp * (S + 1) + S];
      std::vector<double> buf(6 * (e - b));
      double* arrs[6] = {h->x, h->y, h->px, h->py, h->th, h->ga};
      for (int k = 0; k < 6; ++k) CK(cudaMemcpy(buf.data() + k * (e - b), arrs[k] + b, (e - b) * sizeof(double), cudaMemcpyDeviceToHost));
      keep.push_back(std::move(buf));
      kept.push_back(sp);
    }
    felis_status st = relayout(h, per);
    if (st != FELIS_OK) return st;
    for (size_t k = 0; k < kept.size(); ++k) {
      const int sp = kept[k];
      const int64_t b = h->soff[(size_t)sp * (S + 1)], e = h->soff[(size_t)sp * (S + 1) + S];
      double* arrs[6] = {h->x, h->y, h->px, h->py, h->th, h->ga};
      for (int q = 0; q < 6; ++q) CK(cudaMemcpy(arrs[q] + b, keep[k].data() + q * (e - b), (e - b) * sizeof(double), cudaMemcpyHostToDevice));
      h->uploaded[sp] = 1;
    }
  }
  const int64_t b = h->soff[(size_t)species * (S + 1)];
  const double* src[6] = {x, y, px, py, theta, gamma};
  double* dst[6] = {h->x, h->y, h->px, h->py, h->th, h->ga};
  // host or device arrays (felis_config_load_beam_device writes device ones)
  for (int k = 0; k < 6; ++k)
    if (cnt > 0) CK(cudaMemcpyAsync(dst[k] + b, src[k], cnt * sizeof(double), cudaMemcpyDefault, h->st));
  for (int s = 0; s < S; ++s) h->weight[(size_t)species * S + s] = weights[s];
  if (!h->d_weight) CK(cudaMalloc(&h->d_weight, (size_t)ns * S * sizeof(double)));
  CK(cudaMemcpyAsync(h->d_weight, h->weight.data(), (size_t)ns * S * sizeof(double), cudaMemcpyHostToDevice, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->uploaded[species] = 1;
  h->counts[species] = cnt;
  invalidate_particles(h);
  return FELIS_OK;
}

felis_status felis_download_particles(felis_handle* h, int32_t species, double* x, double* y, double* px, double* py,
                                      double* theta, double* gamma) {
  if (!h || species < 0 || species >= h->p.num_species || !h->uploaded[species]) return fail(h, FELIS_BAD_ARG, "bad argument");
  const int S = h->p.slice_n;
  const int64_t b = h->soff[(size_t)species * (S + 1)], e = h->soff[(size_t)species * (S + 1) + S];
  double* dst[6] = {x, y, px, py, theta, gamma};
  const double* src[6] = {h->x, h->y, h->px, h->py, h->th, h->ga};
  for (int k = 0; k < 6; ++k)
    if (dst[k] && e > b) CK(cudaMemcpyAsync(dst[k], src[k] + b, (e - b) * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return FELIS_OK;
}

felis_status felis_upload_field(felis_handle* h, int32_t hidx, int32_t pol, const double* data) {
  if (!h || hidx < 0 || hidx >= h->p.num_harmony || pol < 0 || pol > 1 || !data) return fail(h, FELIS_BAD_ARG, "bad argument");
  const int S = h->p.slice_n;
  const size_t N = (size_t)h->p.nx * h->p.ny;
  for (int s = 0; s < S; ++s)
    CK(cudaMemcpyAsync(h->U + field_plane(S, hidx, pol, s, h->ring_base) * N, data + 2 * (size_t)(s + 1) * N,
                       N * sizeof(double2), cudaMemcpyHostToDevice, h->st));
  CK(cudaStreamSynchronize(h->st));
  h->diag_valid = false;
  return FELIS_OK;
}

felis_status felis_download_field(felis_handle* h, int32_t hidx, int32_t pol, double* data) {
  if (!h || hidx < 0 || hidx >= h->p.num_harmony || pol < 0 || pol > 1 || !data) return fail(h, FELIS_BAD_ARG, "bad argument");
  const int S = h->p.slice_n;
  const size_t N = (size_t)h->p.nx * h->p.ny;
  memset(data, 0, 2 * N * sizeof(double));
  memset(data + 2 * (size_t)(S + 1) * N, 0, 2 * N * sizeof(double));
  for (int s = 0; s < S; ++s)
    CK(cudaMemcpyAsync(data + 2 * (size_t)(s + 1) * N, h->U + field_plane(S, hidx, pol, s, h->ring_base) * N,
                       N * sizeof(double2), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return FELIS_OK;
}

felis_status felis_download_source(felis_handle* h, int32_t hidx, int32_t pol, double* data) {
  if (!h || hidx < 0 || hidx >= h->p.num_harmony || pol < 0 || pol > 1 || !data) return fail(h, FELIS_BAD_ARG, "bad argument");
  const int S = h->p.slice_n, nx = h->p.nx;
  const size_t N = (size_t)h->p.nx * h->p.ny;
  std::vector<int4> box(S);
  std::vector<double> plane(2 * N);
  CK(cudaMemcpy(box.data(), h->box, S * sizeof(int4), cudaMemcpyDeviceToHost));
  memset(data, 0, 2 * (size_t)(S + 2) * N * sizeof(double));
  for (int s = 0; s < S; ++s) {
    CK(cudaMemcpy(plane.data(), h->Sc + (((size_t)hidx * 2 + pol) * S + s) * N, N * sizeof(double2), cudaMemcpyDeviceToHost));
    const int4 b = box[s];
    for (int j = b.z; j <= b.w; ++j)
      for (int i = b.x; i <= b.y; ++i) {
        const size_t k = (size_t)j * nx + i;
        data[2 * ((size_t)(s + 1) * N + k)] = plane[2 * k];
        data[2 * ((size_t)(s + 1) * N + k) + 1] = plane[2 * k + 1];
      }
  }
  return FELIS_OK;
}

felis_status felis_download_ez(felis_handle* h, double* data) {
  if (!h || !data) return fail(h, FELIS_BAD_ARG, "bad argument");
  const size_t n = (size_t)h->p.scl_mode * (h->p.slice_n + 2) * h->p.scf_mode * h->p.nr;
  CK(cudaMemcpy(data, h->Ez, n * sizeof(double2), cudaMemcpyDeviceToHost));
  return FELIS_OK;
}

felis_status felis_update_lattice(felis_handle* h, int32_t it, double half) {
  if (!h) return FELIS_BAD_ARG;
  update_lattice(h, it, half);
  h->prep_valid = false;
  return FELIS_OK;
}
felis_status felis_get_lattice(felis_handle* h, felis_lattice* out) {
  if (!h || !out) return FELIS_BAD_ARG;
  *out = h->lat;
  return FELIS_OK;
}
felis_status felis_set_lattice(felis_handle* h, const felis_lattice* in) {
  if (!h || !in) return FELIS_BAD_ARG;
  h->lat = *in;
  h->prep_valid = false;
  return FELIS_OK;
}

felis_status felis_update_total_energy(felis_handle* h, int32_t it, double* out) {
  if (!h || !out) return FELIS_BAD_ARG;
  (void)it;
  {
    KernelScope ks(h, FELIS_KERNEL_REDUCE);
    launch_energy(h->G, h->U, h->ring_base, h->d_planes2, h->st);
    launch_sum_planes(h->d_planes2, h->p.num_harmony, h->p.slice_n, 0, h->d_tmp, h->st);
    h->launches[FELIS_KERNEL_REDUCE] += 1;
  }
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, h->d_tmp, 2 * h->p.num_harmony * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return FELIS_OK;
}

static felis_status diag_now(felis_handle* h, double* twiss_dev, double* bf_dev) {
  felis_status s = ensure_ready(h);
  if (s != FELIS_OK) return s;
  s = run_particles(h, OP_DIAG, nullptr, nullptr);
  if (s != FELIS_OK) return s;
  {
    KernelScope ks(h, FELIS_KERNEL_REDUCE);
    launch_diag_finalize(h->d_part, (int)h->tiles.size(), h->diag_stride, h->p.num_species, h->p.num_harmony,
                         h->d_tiles, h->d_l1, h->l1_blocks, twiss_dev, bf_dev, h->st);
  }
  CK(cudaGetLastError());
  return FELIS_OK;
}

felis_status felis_twiss(felis_handle* h, int32_t it, double* out) {
  if (!h || !out) return FELIS_BAD_ARG;
  (void)it;
  felis_status s = diag_now(h, h->d_tmp, h->d_tmp + 6 * FELIS_MAX_SPECIES);
  if (s != FELIS_OK) return s;
  CK(cudaMemcpyAsync(out, h->d_tmp, 6 * h->p.num_species * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return FELIS_OK;
}

felis_status felis_bfactor(felis_handle* h, int32_t it, double* out) {
  if (!h || !out) return FELIS_BAD_ARG;
  (void)it;
  felis_status s = diag_now(h, h->d_tmp, h->d_tmp + 6 * FELIS_MAX_SPECIES);
  if (s != FELIS_OK) return s;
  CK(cudaMemcpyAsync(out, h->d_tmp + 6 * FELIS_MAX_SPECIES, 2 * h->p.num_harmony * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  return FELIS_OK;
}

// Scalars of one 1D call (solveField.cpp:428-470, particlePush.cpp:390-436),
// formed on the host in the restatement's order.
static bool oned_setup(const felis_handle* h, const felis_lattice& L, OneDLaunch* a) {
  *a = OneDLaunch{};
  a->G = h->G;
  a->ns = h->p.num_species;
  a->ring_base = h->ring_base;
  a->soff = h->d_soff; a->weight = h->d_weight; a->th = h->th; a->ga = h->ga;
  a->U = h->U; a->Sc = h->Sc; a->Ez = h->Ez; a->err = h->d_err;
  if (!polarisation(L, &a->Phi, &a->etaX, &a->etaY)) return false;
  const double K0 = L.K0, ue = L.ue, ks = h->p.ks, dz = h->p.dz;
  const double bucket = h->p.lambda0 * h->p.num_slice;
  a->K0 = K0; a->ue = ue; a->ku = L.ku; a->dz = dz;
  a->K2 = 1.0 + K0 * K0 * 0.5 * (1.0 + ue * ue);
  a->dPhi = 2.0 * M_PI * h->p.num_slice;
  a->e_mc2 = K_ECHARGE / K_EMASS / K_VELOCITYC / K_VELOCITYC;
  a->sq = sqrt(ue * ue + 1.0);
  for (int sp = 0; sp < h->p.num_species; ++sp) {
    const double area = h->p.beam_area[sp];
    a->coefU[sp] = dz * K_ECHARGE * K_ECHARGE * K_MU0 * K0 * sqrt(1.0 + ue * ue) / (2.0 * ks * K_EMASS * bucket * area);
    a->coefE[sp] = K_ECHARGE * K_VELOCITYC * K_VELOCITYC * K_MU0 / ks / area / bucket;
  }
  const double xi = 0.25 * K0 * K0 * (1.0 - ue * ue) / (1.0 + (1.0 + ue * ue) * K0 * K0 * 0.5);
  const double K0a = L.K0_alpha;
  const double* B = h->p.bessel;
  const int bc = h->p.bessel_cols, rows = h->p.bessel_rows;
  for (int hh = 0; hh < h->p.num_harmony; ++hh) {
    const int H = h->p.harmony[hh];
    a->fsrc[hh][0] = a->fsrc[hh][1] = a->fpush[hh][0] = a->fpush[hh][1] = C(0.0, 0.0);
    if (H % 2 != 1) continue;
    const double sign = ((H - 1) / 2 % 2 == 0) ? 1.0 : -1.0;
    const int idx = (int)(H * xi / h->p.d_bessel);
    if (idx < 0 || idx + 1 >= rows) return false;
    double w[2];
    w[1] = (H * xi / h->p.d_bessel) - idx;
    w[0] = 1.0 - w[1];
    int order = (H - 1) / 2;
    const double J1 = B[(size_t)idx * bc + order] * w[0] + B[(size_t)(idx + 1) * bc + order] * w[1];
    order = (H + 1) / 2;
    const double J2 = B[(size_t)idx * bc + order] * w[0] + B[(size_t)(idx + 1) * bc + order] * w[1];
    a->fsrc[hh][0] = C(sign * (J1 - K0a * J2), 0.0);
    a->fsrc[hh][1] = C(sign * (J1 + K0a * J2), 0.0);
    a->fpush[hh][0] = C(sign * (K0a * J1 - J2), 0.0);
    a->fpush[hh][1] = C(sign * (K0a * J1 + J2), 0.0);
  }
  return true;
}

static felis_status run_1d_field(felis_handle* h) {
  OneDLaunch a;
  if (!oned_setup(h, h->lat, &a)) return fail(h, FELIS_BAD_ARG, "invalid K0_alpha or Bessel range (1D)");
  KernelScope ks(h, FELIS_KERNEL_ADI);
  CK(launch_1d_field(a, h->lat.current_flag, h->st));
  return FELIS_OK;
}

static felis_status run_1d_push(felis_handle* h, const felis_lattice& L) {
  OneDLaunch a;
  if (!oned_setup(h, L, &a)) return fail(h, FELIS_BAD_ARG, "invalid K0_alpha or Bessel range (1D)");
  KernelScope ks(h, FELIS_KERNEL_PARTICLES);
  CK(launch_1d_push(a, h->st));
  return FELIS_OK;
}

static felis_status solve_field_impl(felis_handle* h) {
  felis_status s = ensure_ready(h);
  if (s != FELIS_OK) return s;
  if (h->p.dimension == 1) return run_1d_field(h);
  if (h->lat.current_flag) {
    if (!h->prep_valid) {
      s = run_particles(h, OP_PREP, nullptr, &h->lat);
      if (s != FELIS_OK) return s;
    }
    s = run_deposit(h, h->lat);
    if (s != FELIS_OK) return s;
  }
  return run_adi(h, h->lat.current_flag);
}

felis_status felis_solve_field(felis_handle* h, int32_t it) {
  if (!h) return FELIS_BAD_ARG;
  (void)it;
  felis_status s = solve_field_impl(h);
  if (s != FELIS_OK) return s;
  h->diag_valid = false;
  return check_err(h);
}

felis_status felis_transverse_push(felis_handle* h, int32_t it) {
  if (!h) return FELIS_BAD_ARG;
  (void)it;
  felis_status s = ensure_ready(h);
  if (s != FELIS_OK) return s;
  if (h->p.dimension == 1) return FELIS_OK;  // main.cpp:133-140: 3D only
  s = run_particles(h, OP_T0, &h->lat, nullptr);
  if (s != FELIS_OK) return s;
  invalidate_particles(h);
  return check_err(h);
}

felis_status felis_push_theta_gamma(felis_handle* h, int32_t it) {
  if (!h) return FELIS_BAD_ARG;
  (void)it;
  felis_status s = ensure_ready(h);
  if (s != FELIS_OK) return s;
  s = h->p.dimension == 1 ? run_1d_push(h, h->lat) : run_particles(h, OP_PUSH, nullptr, &h->lat);
  if (s != FELIS_OK) return s;
  invalidate_particles(h);
  return check_err(h);
}

felis_status felis_drift_theta_gamma(felis_handle* h, int32_t it) {
  if (!h) return FELIS_BAD_ARG;
  (void)it;
  felis_status s = ensure_ready(h);
  if (s != FELIS_OK) return s;
  if (h->p.dimension == 1) return FELIS_OK;  // nx = 1: no particle passes particlePush.cpp:160
  s = run_particles(h, OP_DRIFT, nullptr, &h->lat);
  if (s != FELIS_OK) return s;
  invalidate_particles(h);
  return check_err(h);
}

felis_status felis_phase_shift(felis_handle* h, int32_t it) {
  if (!h) return FELIS_BAD_ARG;
  felis_status s = ensure_ready(h);
  if (s != FELIS_OK) return s;
  const double dth = theta_shift(h, it);
  if (dth == 0.0) return FELIS_OK;
  s = run_particles(h, OP_PHASE, nullptr, nullptr, dth);
  if (s != FELIS_OK) return s;
  invalidate_particles(h);
  return check_err(h);
}

felis_status felis_periodic_particles(felis_handle* h, int32_t it) {
  if (!h) return FELIS_BAD_ARG;
  (void)it;
  felis_status s = ensure_ready(h);
  if (s != FELIS_OK) return s;
  s = run_particles(h, OP_WRAP, nullptr, nullptr);
  if (s != FELIS_OK) return s;
  invalidate_particles(h);
  return check_err(h);
}

felis_status felis_shift_field(felis_handle* h, int32_t it) {
  if (!h) return FELIS_BAD_ARG;
  (void)it;
  felis_status s = do_shift(h);
  if (s != FELIS_OK) return s;
  h->diag_valid = false;
  CK(cudaStreamSynchronize(h->st));
  return FELIS_OK;
}

// One iteration of the 1D model (main.cpp:117-155 without the transverse
// pushes): diagnostics, field, push, wrap, shift.
static felis_status step_impl_1d(felis_handle* h, int it) {
  const int H = h->p.num_harmony, ns = h->p.num_species;
  if (it >= 0 && it < h->hist_n) {
    {
      KernelScope ks(h, FELIS_KERNEL_REDUCE);
      launch_energy(h->G, h->U, h->ring_base, h->d_planes2, h->st);
      launch_sum_planes(h->d_planes2, H, h->p.slice_n, 0, h->d_hist_e + (size_t)it * 2 * H, h->st);
      h->launches[FELIS_KERNEL_REDUCE] += 1;
    }
    felis_status s = diag_now(h, h->d_hist_t + (size_t)it * 6 * ns, h->d_hist_b + (size_t)it * 2 * H);
    if (s != FELIS_OK) return s;
  }
  felis_status s = run_1d_field(h);
  if (s != FELIS_OK) return s;
  update_lattice(h, it, 0);
  update_lattice(h, it, 0.5);
  const felis_lattice l1 = h->lat;
  if (!l1.drift_flag) {
    s = run_1d_push(h, l1);
    if (s != FELIS_OK) return s;
  }
  const double dth = theta_shift(h, it);
  s = run_particles(h, dth != 0.0 ? (OP_PHASE | OP_WRAP) : OP_WRAP, nullptr, nullptr, dth);
  if (s != FELIS_OK) return s;
  h->prep_valid = false;
  if (!l1.drift_flag && h->p.mode == FELIS_TIME_DEPENDENT) {
    s = do_shift(h);
    if (s != FELIS_OK) return s;
  }
  h->diag_valid = false;
  return FELIS_OK;
}

// One iteration of main.cpp:117-155 with the fused particle kernel.
static felis_status step_impl(felis_handle* h, int it) {
  if (h->p.dimension == 1) return step_impl_1d(h, it);
  const int H = h->p.num_harmony, ns = h->p.num_species;
  const bool rec = it >= 0 && it < h->hist_n;
  // diagnostics of this iteration (state before the step)
  if (!(h->diag_valid && h->diag_iter == it)) {
    if (rec) {
      {
        KernelScope ks(h, FELIS_KERNEL_REDUCE);
        launch_energy(h->G, h->U, h->ring_base, h->d_planes2, h->st);
        launch_sum_planes(h->d_planes2, H, h->p.slice_n, 0, h->d_hist_e + (size_t)it * 2 * H, h->st);
        h->launches[FELIS_KERNEL_REDUCE] += 1;
      }
      felis_status s = diag_now(h, h->d_hist_t + (size_t)it * 6 * ns, h->d_hist_b + (size_t)it * 2 * H);
      if (s != FELIS_OK) return s;
    }
  }
  // solveField with the flag left by the previous iteration
  felis_status s = solve_field_impl(h);
  if (s != FELIS_OK) return s;
  felis_lattice l0, l1;
  update_lattice(h, it, 0);
  l0 = h->lat;
  update_lattice(h, it, 0.5);
  l1 = h->lat;
  unsigned ops = OP_T0 | OP_T1 | OP_WRAP | OP_DIAG;
  ops |= l1.drift_flag ? OP_DRIFT : OP_PUSH;
  if (l1.current_flag) ops |= OP_PREP;
  const double dth = theta_shift(h, it);
  if (dth != 0.0) ops |= OP_PHASE;
  s = run_particles(h, ops, &l0, &l1, dth);
  if (s != FELIS_OK) return s;
  h->prep_valid = l1.current_flag != 0;
  const bool shift = !l1.drift_flag && h->p.mode == FELIS_TIME_DEPENDENT;
  if (shift) {
    s = do_shift(h);
    if (s != FELIS_OK) return s;
  }
  // diagnostics of the next iteration from the fused partials and the ADI planes
  if (it + 1 < h->hist_n) {
    {
      KernelScope ks(h, FELIS_KERNEL_REDUCE);
      launch_diag_finalize(h->d_part, (int)h->tiles.size(), h->diag_stride, ns, H, h->d_tiles, h->d_l1, h->l1_blocks,
                           h->d_hist_t + (size_t)(it + 1) * 6 * ns, h->d_hist_b + (size_t)(it + 1) * 2 * H, h->st);
      launch_sum_planes(h->d_planes, H, h->p.slice_n, shift ? 1 : 0, h->d_hist_e + (size_t)(it + 1) * 2 * H, h->st);
      h->launches[FELIS_KERNEL_REDUCE] += 1;
    }
    CK(cudaGetLastError());
    h->diag_valid = true;
    h->diag_iter = it + 1;
  } else {
    h->diag_valid = false;
  }
  return FELIS_OK;
}

felis_status felis_step(felis_handle* h, int32_t it) {
  if (!h) return FELIS_BAD_ARG;
  felis_status s = step_impl(h, it);
  if (s != FELIS_OK) return s;
  return check_err(h);
}

felis_status felis_run(felis_handle* h, int32_t it0, int32_t it1) {
  if (!h || it1 < it0) return FELIS_BAD_ARG;
  if (it1 == it0) return FELIS_OK;
  felis_status s = ensure_ready(h);
  if (s != FELIS_OK) return s;
  CK(cudaStreamSynchronize(h->st));
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  CK(cudaStreamBeginCapture(h->st, cudaStreamCaptureModeThreadLocal));
  h->capturing = true;
  for (int it = it0; it < it1 && s == FELIS_OK; ++it) s = step_impl(h, it);
  h->capturing = false;
  cudaError_t ce = cudaStreamEndCapture(h->st, &graph);
  if (s != FELIS_OK) {
    if (graph) cudaGraphDestroy(graph);
    return s;
  }
  if (ce != cudaSuccess) return fail(h, FELIS_CUDA_ERROR, std::string("graph capture: ") + cudaGetErrorString(ce));
  ce = cudaGraphInstantiate(&exec, graph, 0);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ce == cudaSuccess) ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
  if (ce == cudaSuccess) ce = cudaEventRecord(e0, h->st);
  if (ce == cudaSuccess) ce = cudaGraphLaunch(exec, h->st);
  if (ce == cudaSuccess) ce = cudaEventRecord(e1, h->st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(h->st);
  if (ce == cudaSuccess) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    h->last_run_ms = ms;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (exec) cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess) return fail(h, FELIS_CUDA_ERROR, std::string("graph run: ") + cudaGetErrorString(ce));
  return check_err(h);
}

felis_status felis_get_diagnostics(felis_handle* h, int32_t it0, int32_t it1, double* energy, double* twiss,
                                   double* bfactor) {
  if (!h || it0 < 0 || it1 < it0 || it1 > h->hist_n) return fail(h, FELIS_BAD_ARG, "bad iteration range");
  const int H = h->p.num_harmony, ns = h->p.num_species;
  const size_t n = it1 - it0;
  if (energy) CK(cudaMemcpy(energy, h->d_hist_e + (size_t)it0 * 2 * H, n * 2 * H * sizeof(double), cudaMemcpyDeviceToHost));
  if (twiss) CK(cudaMemcpy(twiss, h->d_hist_t + (size_t)it0 * 6 * ns, n * 6 * ns * sizeof(double), cudaMemcpyDeviceToHost));
  if (bfactor) CK(cudaMemcpy(bfactor, h->d_hist_b + (size_t)it0 * 2 * H, n * 2 * H * sizeof(double), cudaMemcpyDeviceToHost));
  return FELIS_OK;
}

felis_status felis_edge_deposit_count(felis_handle* h, int64_t* count) {
  if (!h || !count) return FELIS_BAD_ARG;
  felis_status s = check_err(h);
  *count = h->edge_total;
  return s;
}

felis_status felis_sync(felis_handle* h) {
  if (!h) return FELIS_BAD_ARG;
  return check_err(h);
}

felis_status felis_profile(felis_handle* h, int32_t enable, int32_t max_launches) {
  if (!h || max_launches < 0) return FELIS_BAD_ARG;
  CK(cudaStreamSynchronize(h->st));
  h->prof = enable != 0;
  h->marks.clear();
  h->ev_used = 0;
  for (int k = 0; k < FELIS_KERNEL_KINDS; ++k) h->launches[k] = 0;
  const size_t want = 2 * (size_t)max_launches;
  while (h->prof && h->ev.size() < want) {
    cudaEvent_t e;
    CK(cudaEventCreate(&e));
    h->ev.push_back(e);
  }
  return FELIS_OK;
}

felis_status felis_kernel_stats(felis_handle* h, int32_t kind, int64_t* launches, double* total_ms) {
  if (!h || kind < -1 || kind >= FELIS_KERNEL_KINDS) return FELIS_BAD_ARG;
  CK(cudaStreamSynchronize(h->st));
  int64_t n = 0;
  if (kind < 0) for (int k = 0; k < FELIS_KERNEL_KINDS; ++k) n += h->launches[k];
  else n = h->launches[kind];
  double ms = 0.0;
  for (const auto& m : h->marks) {
    if (kind >= 0 && m.first != kind) continue;
    float t = 0.f;
    if (cudaEventElapsedTime(&t, h->ev[m.second], h->ev[m.second + 1]) == cudaSuccess) ms += t;
  }
  if (launches) *launches = n;
  if (total_ms) *total_ms = ms;
  return FELIS_OK;
}

felis_status felis_set_slice_exchange(felis_handle* h, int32_t enable) {
  if (!h) return FELIS_BAD_ARG;
  h->exchange = enable != 0;
  h->diag_valid = false;
  return FELIS_OK;
}

// The first slice's planes of every harmonic and polarisation, [H][2][ny*nx]
// interleaved complex: after a shift in exchange mode, the slice that leaves
// this process's block (the packed slot of fieldShareZ.cpp:39-78).
felis_status felis_get_first_planes(felis_handle* h, double* out) {
  if (!h || !out) return FELIS_BAD_ARG;
  const int S = h->p.slice_n, H = h->p.num_harmony;
  const size_t N = (size_t)h->p.nx * h->p.ny;
  CK(cudaStreamSynchronize(h->st));
  for (int hh = 0; hh < H; ++hh)
    for (int pol = 0; pol < 2; ++pol)
      CK(cudaMemcpy(out + 2 * ((size_t)(hh * 2 + pol) * N), h->U + field_plane(S, hh, pol, 0, h->ring_base) * N,
                    N * sizeof(double2), cudaMemcpyDeviceToHost));
  return FELIS_OK;
}

// Device addresses of the first slice's planes, [h][pol] order (2H
// pointers to ny*nx interleaved complex): the same planes as
// felis_get_first_planes, for an exchange that stays in device memory.
felis_status felis_first_planes_device(felis_handle* h, double** planes) {
  if (!h || !planes) return FELIS_BAD_ARG;
  const int S = h->p.slice_n, H = h->p.num_harmony;
  const size_t N = (size_t)h->p.nx * h->p.ny;
  for (int hh = 0; hh < H; ++hh)
    for (int pol = 0; pol < 2; ++pol)
      planes[hh * 2 + pol] = reinterpret_cast<double*>(h->U + field_plane(S, hh, pol, 0, h->ring_base) * N);
  h->diag_valid = false;
  return FELIS_OK;
}

felis_status felis_get_stream(felis_handle* h, void** stream) {
  if (!h || !stream) return FELIS_BAD_ARG;
  *stream = static_cast<void*>(h->st);
  return FELIS_OK;
}

// Sets the first slice's planes (the slice received from the previous
// process; zeros on the first process).
felis_status felis_set_first_planes(felis_handle* h, const double* in) {
  if (!h || !in) return FELIS_BAD_ARG;
  const int S = h->p.slice_n, H = h->p.num_harmony;
  const size_t N = (size_t)h->p.nx * h->p.ny;
  CK(cudaStreamSynchronize(h->st));
  for (int hh = 0; hh < H; ++hh)
    for (int pol = 0; pol < 2; ++pol)
      CK(cudaMemcpy(h->U + field_plane(S, hh, pol, 0, h->ring_base) * N, in + 2 * ((size_t)(hh * 2 + pol) * N),
                    N * sizeof(double2), cudaMemcpyHostToDevice));
  h->diag_valid = false;
  return FELIS_OK;
}

// Unfinished diagnostic sums of the current state, for reductions across
// processes (twiss.cpp:46-64, saveFile.cpp:126-137): per species sum x^2,
// y^2, x'^2, y'^2, x x', y y', count; then per harmonic sum w cos(H theta),
// sum w sin(H theta); then sum w.
felis_status felis_diagnostic_sums(felis_handle* h, int32_t it, double* out) {
  if (!h || !out) return FELIS_BAD_ARG;
  (void)it;
  felis_status s = diag_now(h, h->d_tmp, h->d_tmp + 6 * FELIS_MAX_SPECIES);
  if (s != FELIS_OK) return s;
  const int nq = 7 * h->p.num_species + 2 * h->p.num_harmony + 1;
  std::vector<double> l1((size_t)h->l1_blocks * nq);
  CK(cudaMemcpyAsync(l1.data(), h->d_l1, l1.size() * sizeof(double), cudaMemcpyDeviceToHost, h->st));
  CK(cudaStreamSynchronize(h->st));
  for (int k = 0; k < nq; ++k) {
    double t = 0.0;
    for (int b = 0; b < h->l1_blocks; ++b) t += l1[(size_t)b * nq + k];
    out[k] = t;
  }
  return FELIS_OK;
}

felis_status felis_last_run_ms(felis_handle* h, double* ms) {
  if (!h || !ms) return FELIS_BAD_ARG;
  *ms = h->last_run_ms;
  return FELIS_OK;
}

void felis_detmath_sincos(double x, double* s, double* c) { fm::sincos(x, s, c); }
double felis_detmath_atan(double x) { return fm::atan(x); }
double felis_detmath_atan2(double y, double x) { return fm::atan2(y, x); }

}  // extern "C"
