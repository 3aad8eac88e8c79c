// Host side of the mixed-precision ensemble engine (felis_batch_*).
//
// An ensemble holds many FELIS instances (each one Domain: its own slices,
// grid, harmonics, lattice and beam) resident on one GPU.  All instances
// advance together; every iteration is two launches over all instances, the
// ADI over every field plane and the push (with the next deposit) over every
// slice, followed by a per-instance diagnostic reduction.  A run of
// iterations is captured as one CUDA graph.  The lattice
// (updateK_quadG.cpp:8-94) is evaluated on the host in FP64 for every
// instance and iteration and uploaded as a table.
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <sys/stat.h>
#include <mutex>
#include <array>
#include <cmath>
#include <initializer_list>
#include <complex>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "batch.cuh"

using namespace felis;

namespace {

struct HUnd {
  int type, K0_alpha, air;
  double lambdaU, slopeK, ue;
  std::vector<double> unitStart, unitEnd, undStart, undEnd, K0;
};
struct HQuad {
  std::vector<double> qdStart, qdEnd, g;
};

struct Inst {
  felis_params p{};
  std::vector<HUnd> und;
  std::vector<HQuad> quad;
  std::vector<double> ps_z, ps_phase;  // [Phase_shifter] positions [m] and phases [pi]
  felis_lattice lat{};
  int ring_base = 0;
  int64_t count = 0;
  bool uploaded = false;
  std::vector<double> bessel;
  // device
  float *x = nullptr, *y = nullptr, *px = nullptr, *py = nullptr, *dg = nullptr;
  double* th = nullptr;
  int64_t* soff = nullptr;
  float* weight = nullptr;
  float2* U = nullptr;
  float2* Ez = nullptr;
  float* d_bessel = nullptr;
  double* wake = nullptr;
  float2* adi = nullptr;
  float2* src = nullptr;
  int4* sbox = nullptr;
  int nsrc = 0;
  int src_plane[FELIS_MAX_HARMONY] = {0};
  int cx[5] = {0}, cy[5] = {0};  // ADI chunks of the interior columns / rows
  int adi_k[FELIS_MAX_HARMONY][8] = {};  // constant ranges and product lengths (adi_ranges)
  double* part_e = nullptr;
  double* part_b = nullptr;
  int* err = nullptr;
};

// Same state machine as updateK_quadG.cpp:8-94.
void update_lattice(Inst& I, int iteration, double half) {
  felis_lattice& D = I.lat;
  const double dz = I.p.dz, z = (iteration + half) * dz;
  double K0 = D.K0, ue = D.ue, lambdaU = D.lambdaU;
  int K0_alpha = D.K0_alpha, undType = D.und_type;
  bool inUnd = false, inInter = false, air = false;
  for (const HUnd& U : I.und)
    for (size_t n = 0; n < U.unitStart.size(); ++n)
      if (z >= U.unitStart[n] && z < U.unitEnd[n]) {
        if (z >= U.undStart[n] && z < U.undEnd[n]) {
          inUnd = true;
          K0 = U.K0[n] * (1 + U.slopeK * (z - U.undStart[n]));
          K0_alpha = U.K0_alpha; ue = U.ue; undType = U.type; lambdaU = U.lambdaU;
        } else {
          inInter = true;
          if (U.air) air = true;
        }
      }
  D.K0 = K0; D.ue = ue; D.K0_alpha = K0_alpha; D.lambdaU = lambdaU; D.ku = 2 * M_PI / lambdaU; D.und_type = undType;
  D.current_flag = 0;
  D.drift_flag = 0;
  if (K0 == 0.0) air = true;
  if (!inUnd && !inInter) air = true;
  if (inUnd) D.current_flag = 1;
  if (air) { D.ku = 0.0; D.drift_flag = 1; D.current_flag = 0; }
  double g = 0;
  const double x0 = z, x1 = z + dz * 0.5;
  for (const HQuad& Q : I.quad)
    for (size_t n = 0; n < Q.g.size(); ++n) {
      const double q0 = Q.qdStart[n], q1 = Q.qdEnd[n];
      if (q1 <= x0 || q0 >= x1) continue;
      if (x0 < q0 && q1 < x1) g = (q1 - q0) / dz * 2.0 * Q.g[n];
      else if (x0 < q0 && q0 < x1) g = (x1 - q0) / dz * 2.0 * Q.g[n];
      else if (x0 < q1 && q1 < x1) g = (q1 - x0) / dz * 2.0 * Q.g[n];
      else g = 1.0 * Q.g[n];
      break;
    }
  D.g = g;
}

bool phi_eta(const felis_lattice& L, double* Phi, double eta[4]) {
  const double ue = L.ue;
  *Phi = atan2(2.0 * ue / (1.0 + ue * ue), (1.0 - ue * ue) / (1.0 + ue * ue));
  const double c = cos(*Phi * 0.5), s = sin(*Phi * 0.5);
  if (L.K0_alpha == 1) { eta[0] = c; eta[1] = 0; eta[2] = 0; eta[3] = s; }
  else if (L.K0_alpha == -1) { eta[0] = 0; eta[1] = s; eta[2] = c; eta[3] = 0; }
  else return false;
  return true;
}

// Transverse half-push of particlePush.cpp:42-110 for lattice L: for a
// fixed a = 1/gamma the RK4 step of dz/2 is exact polynomial arithmetic on
// the linear system s' = A(a) s, s = (x, y, px, py):
//   x'  = a px - aa a^2 (K0a x + y)        y'  = a py + aa a^2 (K0a x - y)
//   px' = K0a dd (px - py) - fx x           py' = K0a dd (px + py) - fy y
// with dd = ku K0^2 ue a^2 / 4, fx = bb a xCoef + cc, fy = bb a yCoef - cc;
// the step multiplies s by P(hA) = I + hA + (hA)^2/2 + (hA)^3/6 + (hA)^4/24.
struct HalfPush {
  double h, K0, ue, ku, aa, bb, cc, xCoef, yCoef, K0a;
};

HalfPush half_push(const Inst& I, const felis_lattice& L) {
  HalfPush t;
  t.h = I.p.dz * 0.5;
  t.K0 = L.K0; t.ue = L.ue; t.ku = L.ku;
  t.aa = L.K0 * L.K0 * 0.25 * L.ue * L.ku;
  t.bb = L.K0 * L.K0 * 0.25 * (1.0 + L.ue * L.ue) * L.ku * L.ku;
  t.cc = K_ECHARGE * L.g / K_EMASS / K_VELOCITYC;
  t.xCoef = 0.0; t.yCoef = 0.0;
  if (L.und_type == FELIS_BIPOLAR) {
    if (L.K0_alpha == 1) t.xCoef = 1.0;
    else if (L.K0_alpha == -1) t.yCoef = 1.0;
  } else {
    t.xCoef = 1.0; t.yCoef = 1.0;
  }
  t.K0a = L.K0_alpha;
  return t;
}

typedef std::vector<double> Mat;  // 4 x 4, row-major

Mat matmul(const Mat& A, const Mat& B) {
  Mat C(16, 0.0);
  for (int r = 0; r < 4; ++r)
    for (int c = 0; c < 4; ++c)
      for (int k = 0; k < 4; ++k) C[r * 4 + c] += A[r * 4 + k] * B[k * 4 + c];
  return C;
}

Mat half_map(const HalfPush& t, double a) {
  const double dd = t.ku * t.K0 * t.K0 * 0.25 * a * a * t.ue;
  const double fx = t.bb * a * t.xCoef + t.cc, fy = t.bb * a * t.yCoef - t.cc;
  Mat X = {-t.aa * t.K0a * a * a, -t.aa * a * a, a, 0.0,
           t.aa * t.K0a * a * a, -t.aa * a * a, 0.0, a,
           -fx, 0.0, t.K0a * dd, -t.K0a * dd,
           0.0, -fy, t.K0a * dd, t.K0a * dd};
  for (double& v : X) v *= t.h;
  // Horner: I + X (I + X/2 (I + X/3 (I + X/4)))
  Mat P(16, 0.0);
  for (int k = 0; k < 4; ++k) P[k * 5] = 1.0;
  for (int d = 4; d >= 1; --d) {
    Mat Q = matmul(X, P);
    for (int k = 0; k < 16; ++k) P[k] = (k % 5 == 0 ? 1.0 : 0.0) + Q[k] / d;
  }
  return P;
}

// Both half pushes (lattices l0 then l1) to second order in a - 1/gamR.
void transverse_maps(const Inst& I, const felis_lattice& l0, const felis_lattice& l1, BStep& T) {
  const HalfPush t0 = half_push(I, l0), t1 = half_push(I, l1);
  const double aR = 1.0 / I.p.gam_r, eps = aR * 1e-3;
  auto full = [&](double a) { return matmul(half_map(t1, a), half_map(t0, a)); };
  const Mat M0 = full(aR), Mp = full(aR + eps), Mm = full(aR - eps);
  for (int k = 0; k < 16; ++k) {
    T.tD0[k] = (float)(M0[k] - (k % 5 == 0 ? 1.0 : 0.0));
    T.tM1[k] = (float)((Mp[k] - Mm[k]) / (2.0 * eps));
    T.tM2[k] = (float)((Mp[k] - 2.0 * M0[k] + Mm[k]) / (2.0 * eps * eps));
  }
}

// ADI tables of one harmonic in FP32 (the reference recurrence of
// solveField.cpp:138-180 rewritten with reciprocals): per direction p = 1/aP
// (last row 1), m = a/(aP CC[i-1]) (first row 0, last row 1/CC[i-1]),
// r = 1/CC, and the right-hand-side coefficients.
// Four equal chunks of an interior line of m points, for the partitioned
// recurrences of the ADI.  The kernel's lanes walk one chunk of 32
// neighbouring lines (odd row pitch), so any chunk start is free of
// shared-memory bank conflicts; equal chunks keep the four chunk groups
// equally long between the barriers.
void adi_chunks(int m, int out[5]) {
  for (int q = 0; q <= 4; ++q) out[q] = q * m / 4;
}

// Complex tables of the ADI of harmonic hidx (solveField.cpp:80-185), indexed
// by interior point c = i - 1, 16 tables of M entries:
//   0-4   x sweep: 1/alphaP (last: 1), alpha/(alphaP CC[i-1]) (first 0, last
//         1/CC[n-3]), 1/CC, and the chunk products
//         G_c = prod_{k = chunk start}^{c} (-m_k),  Q_c = prod_{k = c}^{chunk end} (-1/CC_k)
//         of the forward and backward recurrences (chunks cx)
//   5-9   the same for the y sweep (chunks cy)
//   10-12 right-hand side of the x sweep by row: -betaP, H+betaP+beta, beta
//   13-15 right-hand side of the y sweep by column: -alphaP, H+alphaP+alpha, alpha
void adi_tables(const felis_params& p, int hidx, int M, const int cx[5], const int cy[5], std::vector<float2>& out) {
  typedef std::complex<double> cd;
  const double H = p.harmony[hidx];
  out.assign((size_t)16 * M, make_float2(0.f, 0.f));
  auto put = [&](int t, int k, cd v) { out[(size_t)t * M + k] = make_float2((float)v.real(), (float)v.imag()); };
  for (int dir = 0; dir < 2; ++dir) {
    const int n = dir == 0 ? p.nx : p.ny, m = n - 2;
    const int* ch = dir == 0 ? cx : cy;
    const double* A = dir == 0 ? p.abc_alpha : p.abc_beta;
    const double* AP = dir == 0 ? p.abc_alpha_p : p.abc_beta_p;
    std::vector<cd> al(n), ap(n), CC(n), fw(m), rc(m);
    for (int i = 0; i < n; ++i) { al[i] = cd(A[2 * i], A[2 * i + 1]); ap[i] = cd(AP[2 * i], AP[2 * i + 1]); }
    CC[1] = (H - ap[1] - al[1]) / ap[1];
    for (int i = 2; i < n - 2; ++i) CC[i] = (H - ap[i] - al[i]) / ap[i] - al[i] / (ap[i] * CC[i - 1]);
    CC[n - 2] = H - ap[n - 2] - al[n - 2] - 1.0 / CC[n - 3];
    const int tp = dir == 0 ? 0 : 5;
    for (int i = 1; i < n - 1; ++i) {
      const int c = i - 1;
      const cd a = i < n - 2 ? 1.0 / ap[i] : cd(1.0, 0.0);
      fw[c] = i == 1 ? cd(0.0, 0.0) : (i < n - 2 ? al[i] / (ap[i] * CC[i - 1]) : 1.0 / CC[n - 3]);
      rc[c] = 1.0 / CC[i];
      put(tp + 0, c, a);
      put(tp + 1, c, fw[c]);
      put(tp + 2, c, rc[c]);
    }
    for (int q = 0; q < 4; ++q) {
      cd g(1.0, 0.0);
      for (int c = ch[q]; c < ch[q + 1]; ++c) { g *= -fw[c]; put(tp + 3, c, g); }
      g = cd(1.0, 0.0);
      for (int c = ch[q + 1] - 1; c >= ch[q]; --c) { g *= -rc[c]; put(tp + 4, c, g); }
    }
    // right-hand side of the other sweep
    const int tr = dir == 0 ? 13 : 10;
    for (int i = 1; i < n - 1; ++i) {
      put(tr + 0, i - 1, -ap[i]);
      put(tr + 1, i - 1, H + ap[i] + al[i]);
      put(tr + 2, i - 1, al[i]);
    }
  }
}

// Where the ADI kernel may use constants instead of table reads, and where
// it may skip the chunk products: out = {kx0, kx1, ky0, ky1, gx, qx, gy, qy}
// for the 16 tables t of one harmonic (layout of adi_tables).  [kx0, kx1) is
// the widest range of interior columns around the middle where the
// column-indexed tables (0-2: x sweep, 13-15: right-hand side of the y sweep)
// hold the same values bit for bit (they vary inside the absorbing layers,
// and the Thomas coefficients settle within a few cells of them); [ky0, ky1)
// likewise for the row-indexed tables (5-7, 10-12).  gx: over how many points
// from a chunk's start the forward product G of the x sweep has a component
// of magnitude >= 2^-40 (beyond, the carry it scales is far below FP32
// resolution); qx: the same for Q from a chunk's end; gy, qy for the y sweep.
void adi_ranges(const std::vector<float2>& t, int M, int mx, int my, const int cx[5], const int cy[5], int out[8]) {
  auto eq = [&](int tab, int a, int b) {
    const float2 u = t[(size_t)tab * M + a], v = t[(size_t)tab * M + b];
    return memcmp(&u, &v, sizeof(float2)) == 0;
  };
  auto range = [&](int m, std::initializer_list<int> tabs, int* o) {
    const int ref = m / 2;
    auto same = [&](int k) {
      for (int tab : tabs)
        if (!eq(tab, k, ref)) return false;
      return true;
    };
    int lo = ref, hi = ref + 1;
    while (lo > 0 && same(lo - 1)) --lo;
    while (hi < m && same(hi)) ++hi;
    o[0] = lo;
    o[1] = hi;
  };
  range(mx, {0, 1, 2, 13, 14, 15}, out);
  range(my, {5, 6, 7, 10, 11, 12}, out + 2);
  const float thr = 0x1p-40f;
  auto big = [&](int tab, int k) {
    const float2 v = t[(size_t)tab * M + k];
    return std::fabs(v.x) >= thr || std::fabs(v.y) >= thr;
  };
  auto lengths = [&](const int* ch, int tg, int tq, int* o) {
    int g = 0, q = 0;
    for (int c = 0; c < 4; ++c)
      for (int k = ch[c]; k < ch[c + 1]; ++k) {
        if (big(tg, k)) g = std::max(g, k - ch[c] + 1);
        if (big(tq, k)) q = std::max(q, ch[c + 1] - k);
      }
    o[0] = g;
    o[1] = q;
  };
  lengths(cx, 3, 4, out + 4);
  lengths(cy, 8, 9, out + 6);
}

}  // namespace

// ADI planes of one grid size: one launch each, so that small grids are not
// given the shared memory of the largest.
struct AdiClass {
  int nx, ny, offset, count, threads, smem;
};

struct felis_batch {
  std::vector<Inst> in;
  std::vector<AdiClass> adi_classes;
  // event-timed launches (felis_batch_profile)
  bool prof = false, capturing = false;
  std::vector<cudaEvent_t> ev;
  size_t ev_used = 0;
  std::vector<std::pair<int, size_t>> marks;
  int64_t launches[FELIS_BATCH_KERNEL_KINDS] = {0};
  int device = 0, sms = 0, dev_smem = 0;
  cudaStream_t st = nullptr;
  std::string err;
  int nx_max = 0, ny_max = 0, H_max = 1, L_max = 1, LF_max = 1, nr_max = 1, N_max = 0, nsrc_max = 1;
  BInst* d_inst = nullptr;
  int4* d_adi_work = nullptr;
  int4* d_push_work = nullptr;
  int n_adi = 0, n_push = 0;
  BStep* d_steps = nullptr;
  double* d_rad = nullptr;  // radial elimination tables of the run's steps (BStep::rad_off)
  int steps_cap = 0;
  double *d_he = nullptr, *d_ht = nullptr, *d_hb = nullptr;
  int hist_n = 0;
  int adi_smem_max = 0;
  // launch shape: source cells the push stages in shared memory (which sets
  // how many push CTAs share an SM) and ADI CTAs per SM
  int push_box = 3072, push_smem = 0, adi_ctas = 2;
  bool layout_ready = false;
  int src_valid_it = -1;  // iteration whose solveField source is in the buffers
  double last_run_ms = 0.0;
  int* h_err = nullptr;
  // device staging of host transfers (FP64 particles and field planes are
  // copied as they are and rounded or widened on the device)
  double* stage = nullptr;
  size_t stage_bytes = 0;
};

namespace {

#define BCK(call)                                                                    \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      b->err = std::string(#call) + ": " + cudaGetErrorString(e_);                   \
      return FELIS_CUDA_ERROR;                                                       \
    }                                                                                \
  } while (0)

felis_status bfail(felis_batch* b, felis_status s, const std::string& m) {
  if (b) b->err = m;
  return s;
}

struct BatchScope {
  felis_batch* b;
  int kind;
  size_t slot = (size_t)-1;
  BatchScope(felis_batch* bb, int k) : b(bb), kind(k) {
    b->launches[k] += 1;
    if (b->prof && b->ev_used + 2 <= b->ev.size()) {
      slot = b->ev_used;
      b->ev_used += 2;
      cudaEventRecordWithFlags(b->ev[slot], b->st, b->capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
    }
  }
  ~BatchScope() {
    if (slot != (size_t)-1) {
      cudaEventRecordWithFlags(b->ev[slot + 1], b->st, b->capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
      b->marks.emplace_back(kind, slot);
    }
  }
};

felis_status upload_inst_table(felis_batch* b) {
  std::vector<BInst> h(b->in.size());
  for (size_t k = 0; k < b->in.size(); ++k) {
    Inst& I = b->in[k];
    BInst& D = h[k];
    const felis_params& p = I.p;
    D.S = p.slice_n; D.nx = p.nx; D.ny = p.ny; D.N = p.nx * p.ny; D.H = p.num_harmony; D.L = p.scl_mode;
    D.F = p.scf_mode; D.nr = p.nr; D.bn = p.bessel_rows; D.bcols = p.bessel_cols;
    D.pitch = (p.nx - 2) | 1;
    for (int q = 0; q < 5; ++q) { D.cx[q] = I.cx[q]; D.cy[q] = I.cy[q]; }
    memcpy(D.adi_k, I.adi_k, sizeof(D.adi_k));
    D.numSlice = p.num_slice; D.minI = p.min_i; D.wakeOn = p.wake_on;
    D.nsrc = I.nsrc;
    for (int i = 0; i < FELIS_MAX_HARMONY; ++i) {
      D.harmony[i] = i < p.num_harmony ? p.harmony[i] : 1;
      D.src_plane[i] = I.src_plane[i];
    }
    D.ks = p.ks; D.dz = p.dz; D.dx = p.dx; D.dy = p.dy; D.dr = p.dr; D.minX = p.min_x; D.minY = p.min_y;
    D.gamR = p.gam_r; D.dBessel = p.d_bessel;
    D.x = I.x; D.y = I.y; D.px = I.px; D.py = I.py; D.dg = I.dg; D.th = I.th;
    D.soff = I.soff; D.weight = I.weight; D.U = I.U; D.Ez = I.Ez; D.src = I.src; D.sbox = I.sbox;
    D.bessel = I.d_bessel; D.wakeE = I.wake;
    D.adi_c = I.adi; D.part_e = I.part_e; D.part_b = I.part_b; D.err = I.err;
  }
  BCK(cudaMemcpy(b->d_inst, h.data(), h.size() * sizeof(BInst), cudaMemcpyHostToDevice));
  return FELIS_OK;
}

// Deposit constants of lattice L (solveField.cpp:209-301; the odd-harmonic
// fx, fy with the lattice's constant xi).
bool make_dep(const Inst& I, const felis_lattice& L, BDep* d) {
  double eta[4], Phi;
  if (!phi_eta(L, &Phi, eta)) return false;
  const felis_params& p = I.p;
  const double K0 = L.K0, ue = L.ue, ks = p.ks;
  d->K0 = (float)K0; d->ue = (float)ue; d->K0a = (float)L.K0_alpha; d->Phi_half = (float)(Phi * 0.5);
  d->coef_U = (float)(p.dz * K_ECHARGE * K_ECHARGE * K_MU0 * K0 * sqrt(1.0 + ue * ue) /
                      (4.0 * ks * K_EMASS * (p.lambda0 * p.num_slice) * p.dx * p.dy));
  const double xi = 0.25 * K0 * K0 * (1.0 - ue * ue) / (1.0 + (1.0 + ue * ue) * K0 * K0 * 0.5);
  d->xi = (float)xi;
  d->coef_Ez = (float)(K_ECHARGE * K_VELOCITYC * K_VELOCITYC * K_MU0 * ks * (1.0 + 0.5 * (1.0 + ue * ue) * K0 * K0) /
                       (2.0 * M_PI * p.lambda0 * p.num_slice * p.gam_r * p.gam_r));
  d->A = ks * ks * (1.0 + 0.5 * (1.0 + ue * ue) * K0 * K0) / (p.gam_r * p.gam_r) * p.dr * p.dr;
  d->etaX = make_float2((float)eta[0], (float)eta[1]);
  d->etaY = make_float2((float)eta[2], (float)eta[3]);
  for (int h = 0; h < FELIS_MAX_HARMONY; ++h) d->fconst[h][0] = d->fconst[h][1] = 0.f;
  for (int h = 0; h < p.num_harmony; ++h) {
    const int H = p.harmony[h];
    if (H % 2 == 1) {
      const double x = H * xi / p.d_bessel;
      const int i0 = std::max(0, std::min((int)x, p.bessel_rows - 1));
      const int i1 = std::min(i0 + 1, p.bessel_rows - 1);
      const double w1 = x - (int)x, w0 = 1.0 - w1;
      const int bc = p.bessel_cols;
      const double J1 = I.bessel[(size_t)i0 * bc + (H - 1) / 2] * w0 + I.bessel[(size_t)i1 * bc + (H - 1) / 2] * w1;
      const double J2 = I.bessel[(size_t)i0 * bc + (H + 1) / 2] * w0 + I.bessel[(size_t)i1 * bc + (H + 1) / 2] * w1;
      const double sign = ((H - 1) / 2 % 2 == 0) ? 1.0 : -1.0;
      d->fconst[h][0] = (float)(sign * (J1 - L.K0_alpha * J2));
      d->fconst[h][1] = (float)(sign * (J1 + L.K0_alpha * J2));
    }
  }
  return true;
}

// ADI source factors of a deposit made with lattice L: odd harmonics keep one
// plane m = sum w mc, the ADI adds -eta fx m (x) and -eta fy m (y); even
// harmonics deposit each polarisation directly.
void make_sfac(const Inst& I, const BDep& d, float2 sfac[FELIS_MAX_HARMONY][2]) {
  for (int h = 0; h < FELIS_MAX_HARMONY; ++h) {
    sfac[h][0] = sfac[h][1] = make_float2(1.f, 0.f);
    if (h < I.p.num_harmony && (I.p.harmony[h] & 1)) {
      const double fx = d.fconst[h][0], fy = d.fconst[h][1];
      sfac[h][0] = make_float2((float)(-d.etaX.x * fx), (float)(-d.etaX.y * fx));
      sfac[h][1] = make_float2((float)(-d.etaY.x * fy), (float)(-d.etaY.y * fy));
    }
  }
}

// The radial Ez elimination of solveField.cpp:361-397 for one deposit's
// coefficient A: per (l, f) mode and point j the multiplier w_j = c_j / b_{j-1}
// and the pivot b_j, in the order and FP64 arithmetic of the device solve,
// which then runs only the right-hand side's recurrence and the divisions.
void radial_elimination(const Inst& I, double depA, double* out) {
  const int L = I.p.scl_mode, F = I.p.scf_mode, nr = I.p.nr;
  for (int l = 0; l < L; ++l)
    for (int f = 0; f < F; ++f) {
      double* t = out + ((size_t)l * F + f) * nr * 2;
      double bprev = f == 0 ? -(1.0 + (l + 1.0) * (l + 1.0) * depA / 8.0) : 1.0;
      double aprev = f == 0 ? 1.0 : 0.0;
      t[0] = 0.0;
      t[1] = bprev;
      for (int j = 1; j < nr; ++j) {
        const bool last = j == nr - 1;
        const double aj = last ? 0.0 : j + 0.5, cj = last ? 0.0 : j - 0.5;
        double bj = last ? 1.0 : -2.0 * j - (l + 1.0) * (l + 1.0) * depA * j - f * f * log((j + 0.5) / (j - 0.5));
        const double ww = cj / bprev;
        bj -= ww * aprev;
        t[2 * j] = ww;
        t[2 * j + 1] = bj;
        bprev = bj;
        aprev = aj;
      }
    }
}

// Per-iteration scalars of every instance for iterations [it0, it1), plus
// one row (index it1 - it0) for a deposit-only launch at it0; `rad` receives
// every row's radial elimination table (rad_stride doubles per row).
felis_status build_steps(felis_batch* b, int it0, int it1, std::vector<BStep>& out, std::vector<double>& rad) {
  const int n = (int)b->in.size();
  out.assign((size_t)(it1 - it0 + 1) * n, BStep{});
  const size_t rs = (size_t)b->LF_max * b->nr_max * 2;
  rad.assign(out.size() * rs, 0.0);
  for (int k = 0; k < n; ++k) {
    Inst& I = b->in[k];
    const felis_params& p = I.p;
    {
      BStep& D0 = out[(size_t)(it1 - it0) * n + k];
      D0.ring_base = I.ring_base;
      D0.deposit = I.lat.current_flag;
      if (!make_dep(I, I.lat, &D0.dep)) return bfail(b, FELIS_BAD_ARG, "invalid K0_alpha");
      const size_t r = (size_t)(it1 - it0) * n + k;
      D0.rad_off = (int64_t)(r * rs);
      radial_elimination(I, D0.dep.A, rad.data() + r * rs);
    }
    for (int it = it0; it < it1; ++it) {
      BStep& T = out[(size_t)(it - it0) * n + k];
      const felis_lattice dl = I.lat;  // solveField uses the flag left by the previous iteration
      update_lattice(I, it, 0);
      const felis_lattice l0 = I.lat;
      update_lattice(I, it, 0.5);
      const felis_lattice l1 = I.lat;
      T.ring_base = I.ring_base;
      T.current = dl.current_flag;
      T.drift = l1.drift_flag;
      T.shift = !l1.drift_flag && p.mode == FELIS_TIME_DEPENDENT;
      T.theta_shift = phase_shift_of((int)I.ps_z.size(), I.ps_z.data(), I.ps_phase.data(), it, p.dz);
      if (T.shift) I.ring_base = (I.ring_base - 1 + p.slice_n) % p.slice_n;
      if (l0.und_type != FELIS_BIPOLAR && l0.und_type != FELIS_QUADPOLAR) return bfail(b, FELIS_BAD_ARG, "no undulator_mode");
      transverse_maps(I, l0, l1, T);
      BDep dd;
      if (!make_dep(I, dl, &dd)) return bfail(b, FELIS_BAD_ARG, "invalid K0_alpha");
      make_sfac(I, dd, T.sfac);
      T.deposit = l1.current_flag;
      if (!make_dep(I, l1, &T.dep)) return bfail(b, FELIS_BAD_ARG, "invalid K0_alpha");
      double eta[4], Phi;
      phi_eta(l1, &Phi, eta);
      const double ks = p.ks, K0 = l1.K0, ue = l1.ue, ku = l1.ku, gR = p.gam_r;
      const double A0 = ks / (2.0 * gR * gR), c1 = (1.0 + ue * ue) * K0 * K0 * 0.5, Q0 = 1.0 + c1;
      T.R0 = (float)(ku - A0 * Q0);
      T.A0 = (float)A0;
      T.AQ0 = (float)(A0 * Q0);
      T.c1 = (float)c1;
      T.c2 = (float)(ku * ku * 0.5);
      T.K0 = (float)K0; T.ue = (float)ue; T.K0a = (float)l1.K0_alpha; T.Phi_half = (float)(Phi * 0.5);
      T.cxi = ku != 0.0 ? (float)(ks / ku * K0 * K0 / 8.0 * (1.0 - ue * ue)) : 0.f;
      T.sq = (float)sqrt(ue * ue + 1.0);
      T.ksK0 = (float)(ks * K0);
      T.e_mc2 = (float)(K_ECHARGE / K_EMASS / K_VELOCITYC / K_VELOCITYC);
      T.dPhi = (float)(2 * M_PI * p.num_slice);
      T.ku = ku;
      T.A0d = A0;
      T.etaX = make_float2((float)eta[0], (float)eta[1]);
      T.etaY = make_float2((float)eta[2], (float)eta[3]);
      const size_t r = (size_t)(it - it0) * n + k;
      T.rad_off = (int64_t)(r * rs);
      radial_elimination(I, T.dep.A, rad.data() + r * rs);
    }
  }
  return FELIS_OK;
}

felis_status prepare(felis_batch* b) {
  if (b->layout_ready) return FELIS_OK;
  for (auto& I : b->in)
    if (!I.uploaded) return bfail(b, FELIS_BAD_ARG, "particles of every instance must be uploaded first");
  // work lists, longest items first (the hardware block scheduler then runs a
  // longest-processing-time schedule): ADI planes by their sweep length,
  // slices by their particle count
  std::vector<int4> push;
  std::vector<double> cp;
  std::map<std::pair<int, int>, std::vector<int4>> by_grid;
  for (size_t k = 0; k < b->in.size(); ++k) {
    const Inst& I = b->in[k];
    std::vector<int64_t> so(I.p.slice_n + 1);
    BCK(cudaMemcpy(so.data(), I.soff, so.size() * sizeof(int64_t), cudaMemcpyDeviceToHost));
    std::vector<int4>& g = by_grid[std::make_pair(I.p.nx, I.p.ny)];
    for (int s = 0; s < I.p.slice_n; ++s) {
      push.push_back(make_int4((int)k, s, 0, 0));
      cp.push_back((double)(so[s + 1] - so[s]));
      for (int hp = 0; hp < 2 * I.p.num_harmony; ++hp) g.push_back(make_int4((int)k, s, hp, 0));
    }
  }
  // largest grids first
  std::vector<int4> adi;
  b->adi_classes.clear();
  for (auto it = by_grid.rbegin(); it != by_grid.rend(); ++it) {
    AdiClass c{};
    c.nx = it->first.first;
    c.ny = it->first.second;
    c.offset = (int)adi.size();
    c.count = (int)it->second.size();
    adi.insert(adi.end(), it->second.begin(), it->second.end());
    b->adi_classes.push_back(c);
  }
  std::vector<double> ca(adi.size(), 0.0);
  auto sorted = [](std::vector<int4>& w, const std::vector<double>& c) {
    std::vector<int> o(w.size());
    for (size_t k = 0; k < o.size(); ++k) o[k] = (int)k;
    std::stable_sort(o.begin(), o.end(), [&](int a, int d) { return c[a] > c[d]; });
    std::vector<int4> r(w.size());
    for (size_t k = 0; k < o.size(); ++k) r[k] = w[o[k]];
    w.swap(r);
  };
  sorted(push, cp);
  b->n_adi = (int)adi.size();
  b->n_push = (int)push.size();
  if (b->d_adi_work) cudaFree(b->d_adi_work);
  if (b->d_push_work) cudaFree(b->d_push_work);
  b->d_adi_work = b->d_push_work = nullptr;
  BCK(cudaMalloc(&b->d_adi_work, adi.size() * sizeof(int4)));
  BCK(cudaMalloc(&b->d_push_work, push.size() * sizeof(int4)));
  BCK(cudaMemcpy(b->d_adi_work, adi.data(), adi.size() * sizeof(int4), cudaMemcpyHostToDevice));
  BCK(cudaMemcpy(b->d_push_work, push.data(), push.size() * sizeof(int4), cudaMemcpyHostToDevice));
  felis_status s = upload_inst_table(b);
  if (s != FELIS_OK) return s;
  b->layout_ready = true;
  return FELIS_OK;
}

// Shared memory of both launches: the ADI holds its interior plane, 16 tables and as
// much of the source box as fits beside adi_ctas CTAs per SM (more cells are
// read from global memory); the push holds the staged field and the
// accumulators of up to push_box source cells (the central window of larger
// boxes; the rest accumulates in the source buffer in global memory).  The
// push kernel's limit is set for the largest choice, 6144 cells.
felis_status ensure_launch(felis_batch* b) {
  b->adi_smem_max = 0;
  for (AdiClass& c : b->adi_classes) {
    if (std::max(c.nx, c.ny) > 256) return bfail(b, FELIS_UNSUPPORTED, "grid wider than 256 points");
    // four chunks of every interior row (x sweep) and column (y sweep)
    c.threads = batch_adi_threads(c.nx, c.ny);
    // 1 KB of every CTA's share stays for static shared memory
    const size_t cap = (size_t)b->dev_smem - 1024;
    const size_t base = batch_adi_smem(c.nx, c.ny, 0);
    if (base > cap) return bfail(b, FELIS_UNSUPPORTED, "field plane does not fit in shared memory");
    const size_t per = (size_t)(b->dev_smem / b->adi_ctas - 2048);
    size_t src_cells = 0;
    if (base <= per) src_cells = (per - base) / sizeof(float2);
    else src_cells = (cap - base) / sizeof(float2);
    src_cells = std::min(src_cells, (size_t)c.nx * c.ny);
    c.smem = (int)batch_adi_smem(c.nx, c.ny, (int)src_cells);
    b->adi_smem_max = std::max(b->adi_smem_max, c.smem);
  }
  b->push_smem = (int)batch_push_smem(b->nsrc_max, b->LF_max, b->nr_max, std::min(b->N_max, b->push_box));
  const int push_max = (int)batch_push_smem(b->nsrc_max, b->LF_max, b->nr_max, std::min(b->N_max, 6144));
  if (batch_set_smem(b->H_max, b->L_max, b->adi_smem_max, push_max) != cudaSuccess)
    return bfail(b, FELIS_UNSUPPORTED, "shared memory of the ensemble launches exceeds the device limit");
  return FELIS_OK;
}

felis_status enqueue_run(felis_batch* b, int it0, int it1, bool deposit0) {
  const int n = (int)b->in.size();
  const int se = 2 * b->H_max, stt = 6, sb = 2 * b->H_max;
  const int steps = it1 - it0;
  const BStep* row_d0 = b->d_steps + (size_t)steps * n;
  if (it0 < b->hist_n) {
    // diagnostics of the state at it0 (row d0 carries the ring offset, no shift)
    BatchScope ks(b, FELIS_BATCH_KERNEL_REDUCE);
    launch_batch_measure(b->d_inst, row_d0, b->d_push_work, b->n_push, b->st);
    launch_batch_reduce(b->d_inst, n, row_d0, b->d_he + (size_t)it0 * se, b->d_ht + (size_t)it0 * stt,
                        b->d_hb + (size_t)it0 * sb, se * b->hist_n, stt * b->hist_n, sb * b->hist_n, b->st);
  }
  if (deposit0) {
    BatchLaunch d{};
    d.inst = b->d_inst; d.step = row_d0; d.work = b->d_push_work; d.nwork = b->n_push;
    d.smem_bytes = b->push_smem; d.mode = BATCH_DEPOSIT_ONLY; d.rad = b->d_rad;
    BatchScope ks(b, FELIS_BATCH_KERNEL_PUSH);
    launch_batch_push(d, b->H_max, b->L_max, b->st);
  }
  for (int it = it0; it < it1; ++it) {
    const BStep* T = b->d_steps + (size_t)(it - it0) * n;
    for (const AdiClass& c : b->adi_classes) {
      BatchLaunch a{};
      a.inst = b->d_inst; a.step = T; a.work = b->d_adi_work + c.offset; a.nwork = c.count; a.smem_bytes = c.smem;
      BatchScope ks(b, FELIS_BATCH_KERNEL_ADI);
      launch_batch_adi(a, c.threads, b->st);
    }
    {
      BatchLaunch p{};
      p.inst = b->d_inst; p.step = T; p.work = b->d_push_work; p.nwork = b->n_push; p.smem_bytes = b->push_smem;
      p.mode = BATCH_PUSH;
      p.rad = b->d_rad;
      BatchScope ks(b, FELIS_BATCH_KERNEL_PUSH);
      launch_batch_push(p, b->H_max, b->L_max, b->st);
    }
    if (it + 1 < b->hist_n) {
      BatchScope ks(b, FELIS_BATCH_KERNEL_REDUCE);
      launch_batch_reduce(b->d_inst, n, T, b->d_he + (size_t)(it + 1) * se, b->d_ht + (size_t)(it + 1) * stt,
                          b->d_hb + (size_t)(it + 1) * sb, se * b->hist_n, stt * b->hist_n, sb * b->hist_n, b->st);
    }
  }
  BCK(cudaGetLastError());
  return FELIS_OK;
}

felis_status check_batch_err(felis_batch* b) {
  for (auto& I : b->in) {
    BCK(cudaMemcpy(b->h_err, I.err, ERR_SLOTS * sizeof(int), cudaMemcpyDeviceToHost));
    felis_status s = FELIS_OK;
    if (b->h_err[ERR_THETA_OVERFLOW]) s = bfail(b, FELIS_THETA_OVERFLOW, "push_theta_gamma: |dtheta| > 2 pi numSlice");
    else if (b->h_err[ERR_OUT_OF_RANGE]) s = bfail(b, FELIS_OUT_OF_RANGE, "theta outside [0, dTh] after the wrap");
    else if (b->h_err[ERR_NAN]) s = bfail(b, FELIS_NAN, "non-finite particle state");
    else if (b->h_err[ERR_RADIAL]) s = bfail(b, FELIS_UNSUPPORTED, "particle outside the radial Ez grid");
    else if (b->h_err[ERR_TIMEOUT]) s = bfail(b, FELIS_TIMEOUT, "a bounded device wait ran out");
    if (s != FELIS_OK) {
      BCK(cudaMemset(I.err, 0, ERR_SLOTS * sizeof(int)));
      return s;
    }
  }
  return FELIS_OK;
}

}  // namespace

extern "C" {

felis_status felis_batch_create(const felis_params* const* instances, int32_t n, felis_batch** out) {
  if (!instances || n < 1 || !out) return FELIS_BAD_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FELIS_NO_DEVICE;
  felis_batch* b = new felis_batch();
  cudaGetDevice(&b->device);
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device);
  cudaDeviceGetAttribute(&b->dev_smem, cudaDevAttrMaxSharedMemoryPerBlockOptin, b->device);
  auto bad = [&](felis_status s, const char* m) {
    fprintf(stderr, "felis_batch_create: %s\n", m);
    felis_batch_destroy(b);
    return s;
  };
  if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess) return bad(FELIS_CUDA_ERROR, "stream");
  if (cudaMallocHost(&b->h_err, ERR_SLOTS * sizeof(int)) != cudaSuccess) return bad(FELIS_CUDA_ERROR, "host buffer");
  b->in.resize(n);
  int max_step = 1;
  for (int k = 0; k < n; ++k) {
    const felis_params* p = instances[k];
    if (!p || p->abi_version != FELIS_ABI_VERSION || p->dimension != 3 || p->num_species != 1 || p->slice_n < 1 ||
        p->num_harmony < 1 || p->num_harmony > FELIS_MAX_HARMONY || p->nx < 6 || p->ny < 6 || p->scl_mode < 1 ||
        p->scl_mode > 4 || p->scf_mode < 1 || p->scl_mode * p->scf_mode > 16 || !p->bessel || !p->abc_alpha)
      return bad(FELIS_BAD_ARG, "instance parameters rejected (one species, 3D, L <= 4)");
    Inst& I = b->in[k];
    I.p = *p;
    for (int u = 0; u < p->num_undulators; ++u) {
      const felis_undulator& U = p->undulators[u];
      HUnd o;
      o.type = U.type; o.K0_alpha = U.K0_alpha; o.air = U.air; o.lambdaU = U.lambdaU; o.slopeK = U.slopeK; o.ue = U.ue;
      o.unitStart.assign(U.unit_start, U.unit_start + U.numbers);
      o.unitEnd.assign(U.unit_end, U.unit_end + U.numbers);
      o.undStart.assign(U.und_start, U.und_start + U.numbers);
      o.undEnd.assign(U.und_end, U.und_end + U.numbers);
      o.K0.assign(U.K0, U.K0 + U.numbers);
      I.und.push_back(o);
    }
    for (int q = 0; q < p->num_quads; ++q) {
      const felis_quad& Q = p->quads[q];
      HQuad o;
      o.qdStart.assign(Q.qd_start, Q.qd_start + Q.numbers);
      o.qdEnd.assign(Q.qd_end, Q.qd_end + Q.numbers);
      o.g.assign(Q.g, Q.g + Q.numbers);
      I.quad.push_back(o);
    }
    if (p->num_phase_shifts > 0) {
      I.ps_z.assign(p->phase_shift_z, p->phase_shift_z + p->num_phase_shifts);
      I.ps_phase.assign(p->phase_shift_phase, p->phase_shift_phase + p->num_phase_shifts);
    }
    I.p.num_phase_shifts = (int32_t)I.ps_z.size();
    I.p.phase_shift_z = nullptr;
    I.p.phase_shift_phase = nullptr;
    I.lat.K0 = p->K0_init; I.lat.ue = p->ue_init; I.lat.lambdaU = p->lambdaU_init;
    I.lat.ku = 2.0 * M_PI / p->lambdaU_init; I.lat.K0_alpha = p->K0_alpha_init; I.lat.und_type = p->und_type_init;
    I.bessel.assign(p->bessel, p->bessel + (size_t)p->bessel_rows * p->bessel_cols);
    b->nx_max = std::max(b->nx_max, p->nx);
    b->ny_max = std::max(b->ny_max, p->ny);
    b->N_max = std::max(b->N_max, p->nx * p->ny);
    b->H_max = std::max(b->H_max, p->num_harmony);
    b->LF_max = std::max(b->LF_max, p->scl_mode * p->scf_mode);
    b->L_max = std::max(b->L_max, p->scl_mode);
    b->nr_max = std::max(b->nr_max, p->nr);
    max_step = std::max(max_step, p->max_step);
    const int S = p->slice_n, N = p->nx * p->ny, H = p->num_harmony, M = std::max(p->nx, p->ny);
    I.nsrc = 0;
    for (int h = 0; h < H; ++h) {
      I.src_plane[h] = I.nsrc;
      I.nsrc += (p->harmony[h] & 1) ? 1 : 2;
    }
    b->nsrc_max = std::max(b->nsrc_max, I.nsrc);
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMalloc(&I.src, (size_t)S * I.nsrc * N * sizeof(float2));
    if (e == cudaSuccess) e = cudaMalloc(&I.sbox, (size_t)S * sizeof(int4));
    if (e == cudaSuccess) {
      std::vector<int4> empty(S, make_int4(1, 0, 1, 0));
      e = cudaMemcpy(I.sbox, empty.data(), S * sizeof(int4), cudaMemcpyHostToDevice);
    }
    const size_t un = (size_t)H * 2 * S * N;
    if (e == cudaSuccess) e = cudaMalloc(&I.U, un * sizeof(float2));
    if (e == cudaSuccess) e = cudaMemset(I.U, 0, un * sizeof(float2));
    const size_t ezn = (size_t)p->scl_mode * S * p->scf_mode * p->nr;
    if (e == cudaSuccess) e = cudaMalloc(&I.Ez, ezn * sizeof(float2));
    if (e == cudaSuccess) e = cudaMemset(I.Ez, 0, ezn * sizeof(float2));
    std::vector<float> bf(I.bessel.begin(), I.bessel.end());
    if (e == cudaSuccess) e = cudaMalloc(&I.d_bessel, bf.size() * sizeof(float));
    if (e == cudaSuccess) e = cudaMemcpy(I.d_bessel, bf.data(), bf.size() * sizeof(float), cudaMemcpyHostToDevice);
    std::vector<double> wk(std::max(p->global_slice_n, 1), 0.0);
    if (p->wake_e) std::copy(p->wake_e, p->wake_e + p->global_slice_n, wk.begin());
    if (e == cudaSuccess) e = cudaMalloc(&I.wake, wk.size() * sizeof(double));
    if (e == cudaSuccess) e = cudaMemcpy(I.wake, wk.data(), wk.size() * sizeof(double), cudaMemcpyHostToDevice);
    adi_chunks(p->nx - 2, I.cx);
    adi_chunks(p->ny - 2, I.cy);
    std::vector<float2> tabs;
    for (int h = 0; h < H; ++h) {
      std::vector<float2> t;
      adi_tables(*p, h, M, I.cx, I.cy, t);
      adi_ranges(t, M, p->nx - 2, p->ny - 2, I.cx, I.cy, I.adi_k[h]);
      tabs.insert(tabs.end(), t.begin(), t.end());
    }
    if (e == cudaSuccess) e = cudaMalloc(&I.adi, tabs.size() * sizeof(float2));
    if (e == cudaSuccess) e = cudaMemcpy(I.adi, tabs.data(), tabs.size() * sizeof(float2), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc(&I.part_e, (size_t)S * 2 * H * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&I.part_b, (size_t)S * (8 + 2 * H) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&I.err, ERR_SLOTS * sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(I.err, 0, ERR_SLOTS * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&I.soff, (size_t)(S + 1) * sizeof(int64_t));
    if (e == cudaSuccess) e = cudaMalloc(&I.weight, (size_t)S * sizeof(float));
    if (e != cudaSuccess) return bad(FELIS_CUDA_ERROR, cudaGetErrorString(e));
    I.p.undulators = nullptr; I.p.quads = nullptr; I.p.bessel = nullptr; I.p.wake_e = nullptr;
    // keep the ABC tables for later table rebuilds
  }
  b->hist_n = max_step + 1;
  cudaError_t e = cudaMalloc(&b->d_inst, (size_t)n * sizeof(BInst));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_he, (size_t)n * b->hist_n * 2 * b->H_max * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_ht, (size_t)n * b->hist_n * 6 * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_hb, (size_t)n * b->hist_n * 2 * b->H_max * sizeof(double));
  if (e != cudaSuccess) return bad(FELIS_CUDA_ERROR, cudaGetErrorString(e));
  for (auto& I : b->in) { I.p.abc_alpha = I.p.abc_alpha_p = I.p.abc_beta = I.p.abc_beta_p = nullptr; }
  if (std::max(b->nx_max, b->ny_max) > 256) return bad(FELIS_UNSUPPORTED, "grid wider than 256 points");
  b->push_box = 3072;
  b->adi_ctas = 2;
  *out = b;
  return FELIS_OK;
}

void felis_batch_destroy(felis_batch* b) {
  if (!b) return;
  if (b->st) cudaStreamSynchronize(b->st);
  for (auto& I : b->in) {
    void* ptrs[] = {I.x, I.y, I.px, I.py, I.dg, I.th, I.soff, I.weight, I.U, I.Ez, I.d_bessel, I.wake, I.adi,
                    I.src, I.sbox, I.part_e, I.part_b, I.err};
    for (void* q : ptrs) if (q) cudaFree(q);
  }
  void* ptrs[] = {b->d_inst, b->d_adi_work, b->d_push_work, b->d_steps, b->d_rad, b->d_he, b->d_ht, b->d_hb, b->stage};
  for (void* q : ptrs) if (q) cudaFree(q);
  if (b->h_err) cudaFreeHost(b->h_err);
  for (cudaEvent_t e : b->ev) cudaEventDestroy(e);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
}

const char* felis_batch_last_error(const felis_batch* b) { return b ? b->err.c_str() : "null ensemble"; }

namespace {
// The staging buffer holds at least `bytes`.
cudaError_t ensure_stage(felis_batch* b, size_t bytes) {
  if (b->stage_bytes >= bytes) return cudaSuccess;
  cudaError_t e = cudaStreamSynchronize(b->st);
  if (e == cudaSuccess && b->stage) e = cudaFree(b->stage);
  b->stage = nullptr;
  b->stage_bytes = 0;
  if (e == cudaSuccess) e = cudaMalloc(&b->stage, bytes);
  if (e == cudaSuccess) b->stage_bytes = bytes;
  return e;
}
}  // namespace

felis_status felis_batch_upload_particles(felis_batch* b, int32_t inst, const double* x, const double* y,
                                          const double* px, const double* py, const double* theta,
                                          const double* gamma, const int64_t* slice_offsets, const double* weights) {
  if (!b || inst < 0 || inst >= (int)b->in.size() || !slice_offsets || !weights) return bfail(b, FELIS_BAD_ARG, "bad argument");
  Inst& I = b->in[inst];
  const int S = I.p.slice_n;
  if (slice_offsets[0] != 0) return bfail(b, FELIS_BAD_ARG, "slice_offsets[0] must be 0");
  for (int s = 0; s < S; ++s)
    if (slice_offsets[s + 1] < slice_offsets[s]) return bfail(b, FELIS_BAD_ARG, "slice_offsets must be non-decreasing");
  const int64_t n = slice_offsets[S];
  if (n > 0 && (!x || !y || !px || !py || !theta || !gamma)) return bfail(b, FELIS_BAD_ARG, "null particle array");
  if (n != I.count || !I.x) {
    float** fa[5] = {&I.x, &I.y, &I.px, &I.py, &I.dg};
    for (auto a : fa) {
      if (*a) cudaFree(*a);
      *a = nullptr;
      BCK(cudaMalloc(a, std::max<int64_t>(n, 1) * sizeof(float)));
    }
    if (I.th) cudaFree(I.th);
    I.th = nullptr;
    BCK(cudaMalloc(&I.th, std::max<int64_t>(n, 1) * sizeof(double)));
    I.count = n;
  }
  b->layout_ready = false;    // work lists follow the particle counts
  b->src_valid_it = -1;       // the next run deposits first
  const double* src[5] = {x, y, px, py, gamma};
  float* dst[5] = {I.x, I.y, I.px, I.py, I.dg};
  // every array is rounded on the device; gamma is stored as gamma - gamR.
  // Device arrays (the device beam loader's) are read in place; host arrays
  // are copied as they are through the theta buffer (n doubles), which
  // receives theta itself last
  cudaPointerAttributes at{};
  const bool on_device = n > 0 && cudaPointerGetAttributes(&at, x) == cudaSuccess && at.type == cudaMemoryTypeDevice;
  for (int k = 0; k < 5 && n > 0; ++k) {
    const double off = k == 4 ? I.p.gam_r : 0.0;
    if (on_device) {
      BCK(launch_f64_to_f32(src[k], dst[k], n, off, b->st));
    } else {
      BCK(cudaMemcpyAsync(I.th, src[k], n * sizeof(double), cudaMemcpyDefault, b->st));
      BCK(launch_f64_to_f32(I.th, dst[k], n, off, b->st));
    }
  }
  if (n) BCK(cudaMemcpyAsync(I.th, theta, n * sizeof(double), cudaMemcpyDefault, b->st));
  BCK(cudaStreamSynchronize(b->st));
  BCK(cudaMemcpy(I.soff, slice_offsets, (S + 1) * sizeof(int64_t), cudaMemcpyHostToDevice));
  std::vector<float> w(weights, weights + S);
  BCK(cudaMemcpy(I.weight, w.data(), S * sizeof(float), cudaMemcpyHostToDevice));
  I.uploaded = true;
  return FELIS_OK;
}

felis_status felis_batch_download_particles(felis_batch* b, int32_t inst, double* x, double* y, double* px,
                                            double* py, double* theta, double* gamma) {
  if (!b || inst < 0 || inst >= (int)b->in.size() || !b->in[inst].uploaded) return bfail(b, FELIS_BAD_ARG, "bad argument");
  Inst& I = b->in[inst];
  const int64_t n = I.count;
  // widened on the device into the staging buffer, then copied as they are
  double* dst[5] = {x, y, px, py, gamma};
  const float* src[5] = {I.x, I.y, I.px, I.py, I.dg};
  if (n) BCK(ensure_stage(b, n * sizeof(double)));
  for (int k = 0; k < 5; ++k) {
    if (!dst[k] || !n) continue;
    BCK(launch_f32_to_f64(src[k], b->stage, n, k == 4 ? I.p.gam_r : 0.0, b->st));
    BCK(cudaMemcpyAsync(dst[k], b->stage, n * sizeof(double), cudaMemcpyDefault, b->st));
  }
  if (theta && n) BCK(cudaMemcpyAsync(theta, I.th, n * sizeof(double), cudaMemcpyDefault, b->st));
  BCK(cudaStreamSynchronize(b->st));
  return FELIS_OK;
}

felis_status felis_batch_upload_field(felis_batch* b, int32_t inst, int32_t hidx, int32_t pol, const double* data) {
  if (!b || inst < 0 || inst >= (int)b->in.size() || !data) return bfail(b, FELIS_BAD_ARG, "bad argument");
  Inst& I = b->in[inst];
  if (hidx < 0 || hidx >= I.p.num_harmony || pol < 0 || pol > 1) return bfail(b, FELIS_BAD_ARG, "bad harmonic/pol");
  const int S = I.p.slice_n;
  const int N = I.p.nx * I.p.ny;
  // the slices' planes (the reference layout's planes 1..S) copied as they
  // are into the staging buffer, in blocks of slices, and rounded into the ring
  const size_t plane_bytes = (size_t)N * 2 * sizeof(double);
  BCK(ensure_stage(b, std::max(plane_bytes, std::min((size_t)S * plane_bytes, (size_t)64 << 20))));
  const int per = (int)std::max<size_t>(1, b->stage_bytes / plane_bytes);
  float2* U = I.U + (size_t)(hidx * 2 + pol) * S * N;
  for (int s0 = 0; s0 < S; s0 += per) {
    const int ns = std::min(per, S - s0);
    BCK(cudaMemcpyAsync(b->stage, data + 2 * (size_t)(s0 + 1) * N, (size_t)ns * plane_bytes, cudaMemcpyDefault, b->st));
    BCK(launch_field_to_f32(b->stage, U, s0, ns, S, N, I.ring_base, b->st));
  }
  BCK(cudaStreamSynchronize(b->st));
  return FELIS_OK;
}

felis_status felis_batch_download_field(felis_batch* b, int32_t inst, int32_t hidx, int32_t pol, double* data) {
  if (!b || inst < 0 || inst >= (int)b->in.size() || !data) return bfail(b, FELIS_BAD_ARG, "bad argument");
  Inst& I = b->in[inst];
  if (hidx < 0 || hidx >= I.p.num_harmony || pol < 0 || pol > 1) return bfail(b, FELIS_BAD_ARG, "bad harmonic/pol");
  BCK(cudaStreamSynchronize(b->st));
  const int S = I.p.slice_n;
  const size_t N = (size_t)I.p.nx * I.p.ny;
  std::vector<float2> plane(N);
  memset(data, 0, 2 * (size_t)(S + 2) * N * sizeof(double));
  for (int s = 0; s < S; ++s) {
    const int phys = (s + I.ring_base) % S;
    BCK(cudaMemcpy(plane.data(), I.U + ((size_t)(hidx * 2 + pol) * S + phys) * N, N * sizeof(float2), cudaMemcpyDeviceToHost));
    double* dst = data + 2 * (size_t)(s + 1) * N;
    for (size_t k = 0; k < N; ++k) { dst[2 * k] = plane[k].x; dst[2 * k + 1] = plane[k].y; }
  }
  return FELIS_OK;
}

felis_status felis_batch_spectral_moments(felis_batch* b, int32_t hidx, double* out) {
  if (!b || !out || hidx < 0 || hidx >= FELIS_MAX_HARMONY) return bfail(b, FELIS_BAD_ARG, "bad argument");
  const int n = (int)b->in.size();
  std::vector<int> ring(n);
  for (int k = 0; k < n; ++k) ring[k] = b->in[k].ring_base;
  int* d_ring = nullptr;
  double* d_out = nullptr;
  BCK(cudaMalloc(&d_ring, n * sizeof(int)));
  cudaError_t e = cudaMalloc(&d_out, (size_t)3 * n * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_ring, ring.data(), n * sizeof(int), cudaMemcpyHostToDevice, b->st);
  if (e == cudaSuccess) {
    launch_batch_spectrum(b->d_inst, n, d_ring, hidx, d_out, b->st);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, (size_t)3 * n * sizeof(double), cudaMemcpyDeviceToHost, b->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(b->st);
  cudaFree(d_ring);
  if (d_out) cudaFree(d_out);
  if (e != cudaSuccess) return bfail(b, FELIS_CUDA_ERROR, cudaGetErrorString(e));
  return FELIS_OK;
}

felis_status felis_batch_set_launch(felis_batch* b, int32_t push_box, int32_t adi_ctas) {
  if (!b || push_box < 512 || push_box > 6144 || adi_ctas < 1 || adi_ctas > 2)
    return bfail(b, FELIS_BAD_ARG, "bad launch shape (push box 512..6144 cells, ADI CTAs per SM 1 or 2)");
  b->push_box = push_box;
  b->adi_ctas = adi_ctas;
  return FELIS_OK;
}

felis_status felis_batch_get_launch(felis_batch* b, int32_t* push_box, int32_t* adi_ctas) {
  if (!b) return FELIS_BAD_ARG;
  if (push_box) *push_box = b->push_box;
  if (adi_ctas) *adi_ctas = b->adi_ctas;
  return FELIS_OK;
}

felis_status felis_batch_run(felis_batch* b, int32_t it0, int32_t it1) {
  if (!b || it1 < it0) return FELIS_BAD_ARG;
  if (it1 == it0) return FELIS_OK;
  felis_status s = prepare(b);
  if (s != FELIS_OK) return s;
  s = ensure_launch(b);
  if (s != FELIS_OK) return s;
  const int n = (int)b->in.size();
  const int steps = it1 - it0;
  // snapshot of the host lattice state: a failed run leaves it unchanged
  std::vector<std::pair<felis_lattice, int>> saved;
  for (auto& I : b->in) saved.push_back(std::make_pair(I.lat, I.ring_base));
  auto restore = [&]() {
    for (size_t k = 0; k < b->in.size(); ++k) { b->in[k].lat = saved[k].first; b->in[k].ring_base = saved[k].second; }
  };
  std::vector<BStep> tab;
  std::vector<double> rad;
  s = build_steps(b, it0, it1, tab, rad);
  if (s != FELIS_OK) { restore(); return s; }
  if (steps > b->steps_cap) {
    if (b->d_steps) cudaFree(b->d_steps);
    if (b->d_rad) cudaFree(b->d_rad);
    b->d_steps = nullptr;
    b->d_rad = nullptr;
    b->steps_cap = steps;
    BCK(cudaMalloc(&b->d_steps, (size_t)(b->steps_cap + 1) * n * sizeof(BStep)));
    BCK(cudaMalloc(&b->d_rad, (size_t)(b->steps_cap + 1) * n * b->LF_max * b->nr_max * 2 * sizeof(double)));
  }
  BCK(cudaMemcpy(b->d_steps, tab.data(), tab.size() * sizeof(BStep), cudaMemcpyHostToDevice));
  BCK(cudaMemcpy(b->d_rad, rad.data(), rad.size() * sizeof(double), cudaMemcpyHostToDevice));
  BCK(cudaStreamSynchronize(b->st));
  const bool deposit0 = b->src_valid_it != it0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  BCK(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
  b->capturing = true;
  s = enqueue_run(b, it0, it1, deposit0);
  b->capturing = false;
  cudaError_t ce = cudaStreamEndCapture(b->st, &graph);
  if (s != FELIS_OK) { if (graph) cudaGraphDestroy(graph); restore(); return s; }
  if (ce != cudaSuccess) { restore(); return bfail(b, FELIS_CUDA_ERROR, std::string("capture: ") + cudaGetErrorString(ce)); }
  ce = cudaGraphInstantiate(&exec, graph, 0);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ce == cudaSuccess) ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
  if (ce == cudaSuccess) ce = cudaEventRecord(e0, b->st);
  if (ce == cudaSuccess) ce = cudaGraphLaunch(exec, b->st);
  if (ce == cudaSuccess) ce = cudaEventRecord(e1, b->st);
  if (ce == cudaSuccess) ce = cudaStreamSynchronize(b->st);
  if (ce == cudaSuccess) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    b->last_run_ms = ms;
  }
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (exec) cudaGraphExecDestroy(exec);
  cudaGraphDestroy(graph);
  if (ce != cudaSuccess) return bfail(b, FELIS_CUDA_ERROR, std::string("graph run: ") + cudaGetErrorString(ce));
  b->src_valid_it = it1;
  return check_batch_err(b);
}

namespace {
// Launch shapes found by felis_batch_tune, per ensemble geometry: in memory,
// and in a text file (FELIS_TUNE_CACHE, or $HOME/.cache/felis_b200_batch_tune_v2.txt)
// so that later processes on the same kind of GPU skip the trials.  One line
// per geometry: SMs nx ny H L LF nr instances particles/65536 push_box adi_ctas.
typedef std::array<long long, 9> TuneKey;
std::mutex g_tune_mu;
std::map<TuneKey, std::pair<int, int>> g_tune;
bool g_tune_loaded = false;

std::string tune_path() {
  const char* e = getenv("FELIS_TUNE_CACHE");
  if (e && *e) return e;
  const char* home = getenv("HOME");
  return std::string(home && *home ? home : "/tmp") + "/.cache/felis_b200_batch_tune_v2.txt";
}

void tune_load() {
  if (g_tune_loaded) return;
  g_tune_loaded = true;
  FILE* f = fopen(tune_path().c_str(), "r");
  if (!f) return;
  TuneKey k;
  int box, adi;
  while (fscanf(f, "%lld %lld %lld %lld %lld %lld %lld %lld %lld %d %d", &k[0], &k[1], &k[2], &k[3], &k[4], &k[5],
                &k[6], &k[7], &k[8], &box, &adi) == 11)
    if (box >= 512 && box <= 6144 && adi >= 1 && adi <= 2) g_tune[k] = std::make_pair(box, adi);
  fclose(f);
}

void tune_store(const TuneKey& k, std::pair<int, int> v) {
  const std::string path = tune_path();
  const size_t slash = path.rfind('/');
  if (slash != std::string::npos && slash > 0) mkdir(path.substr(0, slash).c_str(), 0755);
  FILE* f = fopen(path.c_str(), "a");
  if (!f) return;  // the cache is optional
  fprintf(f, "%lld %lld %lld %lld %lld %lld %lld %lld %lld %d %d\n", k[0], k[1], k[2], k[3], k[4], k[5], k[6], k[7],
          k[8], v.first, v.second);
  fclose(f);
}
}  // namespace

// Launch shapes are tuned on the running ensemble: the push's staged source
// area (3072 cells: seven one-harmonic CTAs per SM; 6144: four, fewer cells
// through global memory on wide beams) and the ADI's CTAs per SM (1: more of
// the source box beside the plane; 2: more planes in flight).  Results do
// not depend on the shape, so the tuner advances the ensemble through real
// iterations, each candidate for `steps` of them, and keeps the fastest.
felis_status felis_batch_tune(felis_batch* b, int32_t it0, int32_t steps, int32_t* next_it) {
  if (!b || steps < 1 || !next_it) return FELIS_BAD_ARG;
  *next_it = it0;
  int64_t total = 0;
  for (auto& I : b->in) total += I.count;
  int dev = 0, sms = 0;
  BCK(cudaGetDevice(&dev));
  BCK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  const TuneKey key = {sms, b->nx_max, b->ny_max, b->H_max, b->L_max, b->LF_max, b->nr_max, (long long)b->in.size(),
                       (long long)(total >> 16)};
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    tune_load();
    auto hit = g_tune.find(key);
    if (hit != g_tune.end()) {
      std::tie(b->push_box, b->adi_ctas) = hit->second;
      return FELIS_OK;
    }
  }
  double best = 1e300;
  std::pair<int, int> pick(b->push_box, b->adi_ctas);
  int it = it0;
  // the first run after an upload also deposits: spend it outside the timing
  if (b->src_valid_it != it) {
    felis_status s = felis_batch_run(b, it, it + 1);
    if (s != FELIS_OK) return s;
    it += 1;
  }
  for (int box : {3072, 6144}) {
    if (box > 3072 && b->N_max <= 3072) continue;  // the same launch as 3072
    for (int c : {1, 2}) {
      b->push_box = box;
      b->adi_ctas = c;
      felis_status s = felis_batch_run(b, it, it + steps);
      if (s != FELIS_OK) return s;
      it += steps;
      const double per = b->last_run_ms / steps;
      if (per < best) { best = per; pick = std::make_pair(box, c); }
    }
  }
  std::tie(b->push_box, b->adi_ctas) = pick;
  {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[key] = pick;
    tune_store(key, pick);
  }
  *next_it = it;
  return FELIS_OK;
}

felis_status felis_batch_profile(felis_batch* b, int32_t enable, int32_t max_launches) {
  if (!b || max_launches < 0) return FELIS_BAD_ARG;
  BCK(cudaStreamSynchronize(b->st));
  b->prof = enable != 0;
  b->marks.clear();
  b->ev_used = 0;
  for (int k = 0; k < FELIS_BATCH_KERNEL_KINDS; ++k) b->launches[k] = 0;
  while (b->prof && b->ev.size() < 2 * (size_t)max_launches) {
    cudaEvent_t e;
    BCK(cudaEventCreate(&e));
    b->ev.push_back(e);
  }
  return FELIS_OK;
}

felis_status felis_batch_kernel_stats(felis_batch* b, int32_t kind, int64_t* launches, double* total_ms) {
  if (!b || kind < -1 || kind >= FELIS_BATCH_KERNEL_KINDS) return FELIS_BAD_ARG;
  BCK(cudaStreamSynchronize(b->st));
  int64_t n = 0;
  if (kind < 0) for (int k = 0; k < FELIS_BATCH_KERNEL_KINDS; ++k) n += b->launches[k];
  else n = b->launches[kind];
  double ms = 0.0;
  for (const auto& m : b->marks) {
    if (kind >= 0 && m.first != kind) continue;
    float t = 0.f;
    if (cudaEventElapsedTime(&t, b->ev[m.second], b->ev[m.second + 1]) == cudaSuccess) ms += t;
  }
  if (launches) *launches = n;
  if (total_ms) *total_ms = ms;
  return FELIS_OK;
}

felis_status felis_batch_last_run_ms(felis_batch* b, double* ms) {
  if (!b || !ms) return FELIS_BAD_ARG;
  *ms = b->last_run_ms;
  return FELIS_OK;
}

felis_status felis_batch_get_diagnostics(felis_batch* b, int32_t inst, int32_t it0, int32_t it1, double* energy,
                                         double* twiss, double* bfactor) {
  if (!b || inst < 0 || inst >= (int)b->in.size() || it0 < 0 || it1 < it0 || it1 > b->hist_n)
    return bfail(b, FELIS_BAD_ARG, "bad range");
  if (it1 == it0) return FELIS_OK;
  BCK(cudaStreamSynchronize(b->st));
  const int H = b->in[inst].p.num_harmony, se = 2 * b->H_max, sb = 2 * b->H_max;
  const size_t rows = (size_t)(it1 - it0);
  // history rows of one instance are contiguous: one strided copy per array
  if (energy)
    BCK(cudaMemcpy2D(energy, 2 * H * sizeof(double), b->d_he + (size_t)inst * se * b->hist_n + (size_t)it0 * se,
                     se * sizeof(double), 2 * H * sizeof(double), rows, cudaMemcpyDeviceToHost));
  if (twiss)
    BCK(cudaMemcpy(twiss, b->d_ht + (size_t)inst * 6 * b->hist_n + (size_t)it0 * 6, rows * 6 * sizeof(double),
                   cudaMemcpyDeviceToHost));
  if (bfactor)
    BCK(cudaMemcpy2D(bfactor, 2 * H * sizeof(double), b->d_hb + (size_t)inst * sb * b->hist_n + (size_t)it0 * sb,
                     sb * sizeof(double), 2 * H * sizeof(double), rows, cudaMemcpyDeviceToHost));
  return FELIS_OK;
}

}  // extern "C"
