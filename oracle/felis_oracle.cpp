// felis_oracle.cpp — CPU restatement of FELIS's per-step slice loop.
//
// TEST INFRASTRUCTURE ONLY.  This file is the test oracle of the GPU library:
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
// it; the product never does.
//
// Parity status: PINNED to the reference itself.  oracle/_ref/felis_ref is
// the reference's setup and step loop compiled from its unmodified sources
// (with project-written single-rank MPI and GSL stand-ins, oracle/ref_shim/);
// tests/test_ref_pin.py runs both builds of this restatement against it from
// the same initial state (static, SASE, QuadPolar with harmonics 1-3, quads,
// taper, wake, Gaussian current, 1D) and tests/test_golden_ref.py against its
// golden outputs for config 1 complete and config 2's leading slices (1539
// steps).  Measured differences: 1e-16 .. 4e-13 relative, from glibc's
// sin/cos/atan versus the deterministic ones below and from the reference's
// two-division complex quotients.  Analytic checks remain in
// tests/test_oracle_pins.py (ADI against a dense solve, Gaussian diffraction,
// energy balance, theta-wrap edges, the 1D gain length).
//
// What it restates (file:line in the reference):
//   updateK_quadG         updateK_quadG.cpp:8-94
//   transversePush        particlePush.cpp:32-117
//   drift_theta_gamma     particlePush.cpp:119-195
//   push_theta_gamma_3D   particlePush.cpp:198-386
//   push_theta_gamma_1D   particlePush.cpp:388-524
//   solve_Sc_1D, solve_Field_U_1D  solveField.cpp:409-549
//   solveField            solveField.cpp:49-78
//   solve_Field_U_3D      solveField.cpp:80-185
//   solve_Sc_3D           solveField.cpp:187-403
//   shiftField            solveField.cpp:19-47 (+ fieldShareZ.cpp:39-78, a no-op at one rank)
//   periodicParticles     rearrangeParticles.cpp:77-114
//   [Phase_shifter]       README.md:57-70 (the block the reference documents
//                         but does not read; the project's reading of it)
//   updateTotalEnergy     updateTotalEnergy.cpp:7-45
//   calculate_twiss       twiss.cpp:7-99
//   updatebFactor         saveFile.cpp:109-172
//   ABC coefficients      boundary.cpp:73-106
//   the loop order        main.cpp:117-155
//
// Arithmetic conventions (kept identical in the GPU library so the two agree
// bit for bit):
//   * every std::complex<double> expression of the reference is written out
//     with the same operand order; complex division uses the expansion that
//     the reference's -ffast-math build selects (limited range, reciprocal):
//     inv = 1/(c^2+d^2); ((a c + b d) inv, (b c - a d) inv);
//   * the per-particle elementary functions (std::exp(I*phase), std::atan,
//     std::atan2) come from the deterministic library in
//     felis_b200/csrc/detmath.h, unless ORACLE_SYSTEM_LIBM is defined, in
//     which case the C library is used (that build measures how far the
//     trajectories move when only the libm changes: the noise floor);
//   * per-step scalars (Phi, eta) use the C library, as the GPU library's
//     host code does;
//   * built with -ffp-contract=off for the parity golden.
// The Bessel table, wake energy loss and initial particles/field are inputs
// (they come from GSL and the beam loader in the reference, outside the loop).

#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../felis_b200/csrc/detmath.h"
#include "../include/felis_b200.h"

#include <atomic>
#include <thread>

namespace {

// constants.h:1-10
const double kMu0 = 1.2566370614e-6;
const double kVelocityC = 299792458.0;
const double kEMass = 9.10938291e-31;
const double kECharge = 1.60217662e-19;
const double kMc2 = 0.510998918;

struct cd {
  double re, im;
};
inline cd C(double r, double i) { return cd{r, i}; }
inline cd cadd(cd a, cd b) { return C(a.re + b.re, a.im + b.im); }
inline cd csub(cd a, cd b) { return C(a.re - b.re, a.im - b.im); }
inline cd cneg(cd a) { return C(-a.re, -a.im); }
inline cd cmul(cd a, cd b) { return C(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
inline cd cscale(cd a, double s) { return C(a.re * s, a.im * s); }  // complex * double
inline cd cdivr(cd a, double s) { return C(a.re / s, a.im / s); }   // complex / double
inline cd cdiv(cd a, cd b) {
  const double inv = 1.0 / (b.re * b.re + b.im * b.im);
  return C((a.re * b.re + a.im * b.im) * inv, (a.im * b.re - a.re * b.im) * inv);
}
inline cd cradd(double d, cd c) { return C(d + c.re, c.im); }   // double + complex
inline cd crsub(double d, cd c) { return C(d - c.re, -c.im); }  // double - complex
inline double cnorm(cd a) { return a.re * a.re + a.im * a.im; }
inline cd cconj(cd a) { return C(a.re, -a.im); }

inline void osincos(double x, double* s, double* c) {
#ifdef ORACLE_SYSTEM_LIBM
  *s = ::sin(x);
  *c = ::cos(x);
#else
  if (!(x - x == 0.0)) { *s = x - x; *c = x - x; return; }  // inf/nan -> nan
  fm::sincos(x, s, c);
#endif
}
inline double oatan(double x) {
#ifdef ORACLE_SYSTEM_LIBM
  return ::atan(x);
#else
  return fm::atan(x);
#endif
}
inline double oatan2(double y, double x) {
#ifdef ORACLE_SYSTEM_LIBM
  return ::atan2(y, x);
#else
  return fm::atan2(y, x);
#endif
}
// std::exp(z) for z = (+-0, phase): exp(+-0) = 1, so (cos phase, sin phase).
inline cd cexpi(double phase) {
  double s, c;
  osincos(phase, &s, &c);
  return C(c, s);
}

struct Und {
  int type, K0_alpha, numbers, air;
  double lambdaU, slopeK, ue;
  std::vector<double> unitStart, unitEnd, undStart, undEnd, K0;
};
struct Quad {
  int numbers;
  std::vector<double> unitStart, unitEnd, qdStart, qdEnd, g;
};

struct Species {
  std::vector<int64_t> off;  // slice_n + 1
  std::vector<double> weight;
  std::vector<double> x, y, px, py, theta, gamma;
};

// Static contiguous split of [n0, n1) over `threads` workers, the same
// block decomposition boundary.cpp:33-46 gives MPI ranks.
template <class Fn>
void pfor(int64_t n0, int64_t n1, int threads, Fn&& fn) {
  const int64_t n = n1 - n0;
  if (threads <= 1 || n < 2) {
    if (n > 0) fn(n0, n1);
    return;
  }
  const int64_t T = std::min<int64_t>(threads, n);
  std::vector<std::thread> pool;
  const int64_t base = n / T, rem = n % T;
  int64_t lo = n0;
  for (int64_t t = 0; t < T; ++t) {
    const int64_t hi = lo + base + (t < rem ? 1 : 0);
    pool.emplace_back([&fn, lo, hi] { fn(lo, hi); });
    lo = hi;
  }
  for (auto& th : pool) th.join();
}

}  // namespace

struct orc {
  // Domain scalars
  int dimension, mode, numHarmony, sliceN, subSliceN, minI, nx, ny, N, numSlice, nSpecies;
  double area[FELIS_MAX_SPECIES];  // 1D: 2 pi sigX sigY per species
  int L, F, nr, bn, bcols, abcN, wakeON, maxStep;
  double ks, lambda0, dz, dx, dy, dr, minX, minY, minZ, maxZ, gamma0, gamR, dBessel, abcSig;
  std::vector<int> harmony;
  // lattice state (Domain fields written by updateK_quadG)
  double K0, ue, lambdaU, ku, g;
  int K0_alpha, undType;
  bool currentFlag, driftFlag;
  std::vector<Und> und;
  std::vector<Quad> quad;
  std::vector<double> psZ, psPhase;  // [Phase_shifter] positions [m], phases [pi]
  // tables
  std::vector<cd> alpha, alphaP, beta, betaP;
  std::vector<double> bessel;  // [bn][bcols]
  std::vector<double> wakeE;
  // state
  std::vector<std::vector<cd>> Ux, Uy, ScUx, ScUy, Ez;
  std::vector<Species> sp;
  int threads;
  int err;  // first error code of the last call
  char msg[256];
  double BJ(int row, int col) const { return bessel[(size_t)row * bcols + col]; }
};

static void push_theta_gamma_1d(orc* D);

static void set_err(orc* D, int code, const char* m) {
  if (D->err == 0) {
    D->err = code;
    snprintf(D->msg, sizeof D->msg, "%s", m);
  }
}

// boundary.cpp:73-106
static void build_abc(orc* D) {
  const int nx = D->nx, ny = D->ny;
  const double dx = D->dx, dy = D->dy, dz = D->dz, ks = D->ks;
  std::vector<double> sigX(nx, 0.0), sigY(ny, 0.0);
  std::vector<cd> sX(nx), sY(ny);
  D->alpha.assign(nx, C(0, 0));
  D->alphaP.assign(nx, C(0, 0));
  D->beta.assign(ny, C(0, 0));
  D->betaP.assign(ny, C(0, 0));
  const int Lx = D->abcN, Ly = D->abcN;
  const double sig0 = D->abcSig;
  for (int i = 0; i < Lx; ++i) sigX[i] = sig0 * (Lx - i) * (Lx - i) / (1.0 * Lx * Lx);
  for (int i = nx - Lx; i < nx; ++i) sigX[i] = sig0 * (i - nx + Lx) * (i - nx + Lx) / (1.0 * Lx * Lx);
  for (int j = 0; j < Ly; ++j) sigY[j] = sig0 * (Ly - j) * (Ly - j) / (1.0 * Ly * Ly);
  for (int j = ny - Ly; j < ny; ++j) sigY[j] = sig0 * (j - ny + Ly) * (j - ny + Ly) / (1.0 * Ly * Ly);
  // 1.0 + I*sig = (1.0 + 0*sig, sig)
  for (int i = 0; i < nx; ++i) sX[i] = C(1.0 + 0.0 * sigX[i], sigX[i]);
  for (int j = 0; j < ny; ++j) sY[j] = C(1.0 + 0.0 * sigY[j], sigY[j]);
  const cd mIdz = C(-0.0 * dz, -1.0 * dz);  // -I*dz
  for (int i = 1; i < nx - 1; ++i) {
    const double k2 = 2.0 * ks * dx * dx;
    D->alpha[i] = cdiv(mIdz, cmul(cscale(sX[i], k2), cadd(sX[i], sX[i - 1])));
    D->alphaP[i] = cdiv(mIdz, cmul(cscale(sX[i], k2), cadd(sX[i], sX[i + 1])));
  }
  for (int j = 1; j < ny - 1; ++j) {
    const double k2 = 2.0 * ks * dy * dy;
    D->beta[j] = cdiv(mIdz, cmul(cscale(sY[j], k2), cadd(sY[j], sY[j - 1])));
    D->betaP[j] = cdiv(mIdz, cmul(cscale(sY[j], k2), cadd(sY[j], sY[j + 1])));
  }
}

// updateK_quadG.cpp:8-94
static void update_lattice(orc* D, int iteration, double half) {
  const double dz = D->dz;
  const double z = (iteration + half) * dz;
  double K0 = D->K0, ue = D->ue, lambdaU = D->lambdaU;
  int K0_alpha = D->K0_alpha, undType = D->undType;
  bool inUnd = false, inInter = false, airPosition = false;
  D->currentFlag = false;
  D->driftFlag = false;
  for (const Und& UL : D->und) {
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
  }
  D->K0 = K0;
  D->ue = ue;
  D->K0_alpha = K0_alpha;
  D->lambdaU = lambdaU;
  D->ku = 2 * M_PI / lambdaU;
  D->undType = undType;
  if (K0 == 0.0) airPosition = true;
  if (!inUnd && !inInter) airPosition = true;
  if (inUnd) D->currentFlag = true;
  if (airPosition) {
    D->ku = 0.0;
    D->driftFlag = true;
    D->currentFlag = false;
  }
  double g = 0;
  const double x0 = z, x1 = z + dz * 0.5;
  for (const Quad& QD : D->quad) {
    for (int n = 0; n < QD.numbers; ++n) {
      const double q0 = QD.qdStart[n], q1 = QD.qdEnd[n];
      if (q1 <= x0 || q0 >= x1) {
      } else {
        if (x0 < q0 && q1 < x1) {
          g = (q1 - q0) / dz * 2.0 * QD.g[n];
          n = QD.numbers;
        } else if (x0 < q0 && q0 < x1) {
          g = (x1 - q0) / dz * 2.0 * QD.g[n];
          n = QD.numbers;
        } else if (x0 < q1 && q1 < x1) {
          g = (q1 - x0) / dz * 2.0 * QD.g[n];
          n = QD.numbers;
        } else {
          g = 1.0 * QD.g[n];
          n = QD.numbers;
        }
      }
    }
  }
  D->g = g;
}

// particlePush.cpp:32-117
static void transverse_push(orc* D) {
  if (D->dimension == 1) return;  // main.cpp:133-140 pushes transversely in 3D only
  const double dz = D->dz * 0.5;
  const double ku = D->ku, K0 = D->K0, ue = D->ue;
  const double aa = D->K0 * D->K0 * 0.25 * ue * D->ku;
  const double bb = D->K0 * D->K0 * 0.25 * (1.0 + ue * ue) * D->ku * D->ku;
  const double cc = kECharge * D->g / kEMass / kVelocityC;
  double xCoef = 0.0, yCoef = 0.0;
  const int K0_alpha = D->K0_alpha;
  if (D->undType == FELIS_BIPOLAR) {
    if (K0_alpha == 1) { xCoef = 1; yCoef = 0; }
    else if (K0_alpha == -1) { xCoef = 0; yCoef = 1; }
  } else if (D->undType == FELIS_QUADPOLAR) {
    xCoef = 1; yCoef = 1;
  } else {
    set_err(D, FELIS_BAD_ARG, "transversePush: no undulator_mode");
    return;
  }
  const double coefList[5] = {0, 0, 0.5, 0.5, 1};
  for (int s = 0; s < D->nSpecies; ++s) {
    Species& P = D->sp[s];
    const int64_t cnt = P.off[D->subSliceN];
    pfor(0, cnt, D->threads, [&](int64_t lo_, int64_t hi_) {
    for (int64_t n = (int64_t)lo_; n < (int64_t)hi_; ++n) {
      double k_xL[5] = {0, 0, 0, 0, 0}, k_yL[5] = {0, 0, 0, 0, 0};
      double k_pxL[5] = {0, 0, 0, 0, 0}, k_pyL[5] = {0, 0, 0, 0, 0};
      const double gam = P.gamma[n];
      const double x0 = P.x[n], y0 = P.y[n], px0 = P.px[n], py0 = P.py[n];
      const double dd = ku * K0 * K0 / (4.0 * gam * gam) * ue;
      for (int m = 1; m < 5; ++m) {
        const double x = x0 + dz * k_xL[m - 1] * coefList[m];
        const double y = y0 + dz * k_yL[m - 1] * coefList[m];
        const double px = px0 + dz * k_pxL[m - 1] * coefList[m];
        const double py = py0 + dz * k_pyL[m - 1] * coefList[m];
        k_xL[m] = px / gam - aa * (K0_alpha * x + y) / (gam * gam);
        k_yL[m] = py / gam + aa * (K0_alpha * x - y) / (gam * gam);
        k_pxL[m] = K0_alpha * (px - py) * dd - (bb / gam * xCoef + cc) * x;
        k_pyL[m] = K0_alpha * (px + py) * dd - (bb / gam * yCoef - cc) * y;
      }
      P.x[n] += dz / 6.0 * (k_xL[1] + 2 * k_xL[2] + 2 * k_xL[3] + k_xL[4]);
      P.y[n] += dz / 6.0 * (k_yL[1] + 2 * k_yL[2] + 2 * k_yL[3] + k_yL[4]);
      P.px[n] += dz / 6.0 * (k_pxL[1] + 2 * k_pxL[2] + 2 * k_pxL[3] + k_pxL[4]);
      P.py[n] += dz / 6.0 * (k_pyL[1] + 2 * k_pyL[2] + 2 * k_pyL[3] + k_pyL[4]);
    }
    });
  }
}

// Phi and eta of particlePush.cpp:222-238 / solveField.cpp:216-231.
static bool polarisation(orc* D, double* Phi, cd* etaX, cd* etaY) {
  const double ue = D->ue;
  // (1.0-ue*ue + I*2.0*ue)/(1.0+ue*ue): I*2.0 = (0, 2); *ue = (0*ue, 2*ue)
  const double re = (1.0 - ue * ue + 0.0 * ue) / (1.0 + ue * ue);
  const double im = (2.0 * ue) / (1.0 + ue * ue);
  *Phi = ::atan2(im, re);
  const double K0_alpha = D->K0_alpha;
  if (K0_alpha == 1) {
    *etaX = C(::cos(*Phi * 0.5), 0.0);
    *etaY = C(0.0, ::sin(*Phi * 0.5));
  } else if (K0_alpha == -1) {
    *etaX = C(0.0, ::sin(*Phi * 0.5));
    *etaY = C(::cos(*Phi * 0.5), 0.0);
  } else {
    set_err(D, FELIS_BAD_ARG, "invalid K0_alpha");
    return false;
  }
  return true;
}

// particlePush.cpp:119-195
static void drift_theta_gamma(orc* D) {
  if (D->dimension == 1) return;  // nx = 1: no particle passes the grid test of particlePush.cpp:160
  const int nx = D->nx, ny = D->ny, N = D->N;
  const double dz = D->dz, ks = D->ks, ku = D->ku, gamR = D->gamR;
  const double dx = D->dx, dy = D->dy, minX = D->minX, minY = D->minY;
  const int H_n = D->numHarmony;
  for (int s = 0; s < D->nSpecies; ++s) {
    Species& P = D->sp[s];
    pfor(0, D->subSliceN, D->threads, [&](int64_t lo_, int64_t hi_) {
    for (int sl = (int)lo_; sl < (int)hi_; ++sl) {
      const int sliceI = sl + 1;
      double wakeE = 0.0;
      if (D->wakeON) wakeE = D->wakeE[sliceI - 1 + D->minI] / (kMc2 * 1.0e6);
      std::vector<cd> Ux(H_n), Uy(H_n);
      double wx[2], wy[2];
      for (int64_t n = P.off[sl]; n < P.off[sl + 1]; ++n) {
        const double x0 = P.x[n], y0 = P.y[n];
        const double px = P.px[n], py = P.py[n];
        const double pr2 = px * px + py * py;
        const double K2 = 1.0 + pr2;
        const int idxI = (int)((x0 - minX) / dx);
        const int idxJ = (int)((y0 - minY) / dy);
        wx[1] = (x0 - minX) / dx - idxI; wx[0] = 1.0 - wx[1];
        wy[1] = (y0 - minY) / dy - idxJ; wy[0] = 1.0 - wy[1];
        if (idxI >= 0 && idxI < nx - 1 && idxJ >= 0 && idxJ < ny - 1) {
          for (int h = 0; h < H_n; ++h) {
            Ux[h] = C(0, 0); Uy[h] = C(0, 0);
            for (int ii = 0; ii < 2; ++ii)
              for (int jj = 0; jj < 2; ++jj) {
                const size_t id = (size_t)sliceI * N + (idxJ + jj) * nx + (idxI + ii);
                Ux[h] = cadd(Ux[h], cscale(cscale(D->Ux[h][id], wx[ii]), wy[jj]));
                Uy[h] = cadd(Uy[h], cscale(cscale(D->Uy[h][id], wx[ii]), wy[jj]));
              }
          }
          double sumU2 = 0.0;
          for (int h = 0; h < H_n; ++h) {
            const int H = D->harmony[h];
            sumU2 += (cnorm(Ux[h]) + cnorm(Uy[h])) / (2.0 * H * H);
          }
          const double tmp = ku - ks / (2.0 * gamR * gamR) * (K2 + sumU2);
          P.theta[n] += tmp * dz;
          P.theta[n] -= dz * wakeE;
        }
      }
    }
    });
  }
}

// particlePush.cpp:198-386
static void push_theta_gamma(orc* D) {
  if (D->dimension == 1) { push_theta_gamma_1d(D); return; }  // particlePush.cpp:15-29
  const int nx = D->nx, ny = D->ny, nr = D->nr, N = D->N, L = D->L, F = D->F;
  const double dz = D->dz, dx = D->dx, dy = D->dy, dr = D->dr;
  const double ku = D->ku, ks = D->ks, K0 = D->K0, dBessel = D->dBessel;
  const double minX = D->minX, minY = D->minY;
  const double dPhi = 2 * M_PI * D->numSlice;
  const double e_mc2 = kECharge / kEMass / kVelocityC / kVelocityC;
  const double ue = D->ue;
  double Phi;
  cd etaX, etaY;
  if (!polarisation(D, &Phi, &etaX, &etaY)) return;
  const double K0_alpha = D->K0_alpha;
  const int H_n = D->numHarmony;
  const double coefList[5] = {0, 0, 0.5, 0.5, 1};
  // Em persists from one particle to the next (particlePush.cpp:248, 290-304):
  // a particle outside the radial grid reuses the previous particle's Em.
  // Slices run in order here so that this carries over exactly.
  std::vector<cd> Em(L, C(0, 0));
  double wakeE = 0.0;
  for (int s = 0; s < D->nSpecies; ++s) {
    Species& P = D->sp[s];
    for (int sl = 0; sl < D->subSliceN; ++sl) {
      const int sliceI = sl + 1;
      if (D->wakeON) wakeE = D->wakeE[sliceI - 1 + D->minI] / (kMc2 * 1.0e6);
      const int64_t n0 = P.off[sl], n1 = P.off[sl + 1];
      // Particles are independent except for the Em carry-over; run the
      // slice in parallel when no in-grid particle can leave the radial grid
      // (checked first), sequentially otherwise.
      bool independent = true;
      for (int64_t n = n0; n < n1 && independent; ++n) {
        const double x0 = P.x[n], y0 = P.y[n];
        const int idxI = (int)((x0 - minX) / dx), idxJ = (int)((y0 - minY) / dy);
        if (idxI >= 0 && idxI < nx - 1 && idxJ >= 0 && idxJ < ny - 1) {
          const int idxR = sqrt(x0 * x0 + y0 * y0) / dr + 0.5;
          if (!(idxR >= 0 && idxR < nr)) independent = false;
        }
      }
      const int nthreads = independent ? D->threads : 1;
      std::atomic<int> overflow{0};
      std::vector<cd> EmChunk0 = Em;
      pfor(n0, n1, nthreads, [&](int64_t lo_, int64_t hi_) {
      std::vector<cd> Em = EmChunk0;
      for (int64_t n = (int64_t)lo_; n < (int64_t)hi_; ++n) {
        double k_th[5] = {0, 0, 0, 0, 0}, k_gam[5] = {0, 0, 0, 0, 0};
        double w[2], wx[2], wy[2], wr[2];
        cd Ux[FELIS_MAX_HARMONY], Uy[FELIS_MAX_HARMONY];
        cd fx = C(0, 0), fy = C(0, 0);
        const double x0 = P.x[n], y0 = P.y[n];
        const double r2 = x0 * x0 + y0 * y0;
        const double px = P.px[n], py = P.py[n];
        const double pr2 = px * px + py * py;
        const double th0 = P.theta[n], gam0 = P.gamma[n];
        const double K2 = 1.0 + pr2 + (1.0 + ue * ue) * K0 * K0 * 0.5 * (1.0 + ku * ku * 0.5 * r2);
        const double xi = ks / ku * K0 * K0 / (8.0 * gam0 * gam0) * (1.0 - ue * ue);
        const double xi2 = sqrt(2.0) * K0 / (1.0 + K0 * K0 * 0.5 * (1.0 + ue * ue)) *
                           sqrt((1 + K0_alpha) * (px * px + ue * ue * py * py) +
                                (1 - K0_alpha) * (px * px * ue * ue + py * py));
        const double B = oatan(2.0 * K0_alpha * ue * (px - py) /
                               ((1.0 + K0_alpha) * (px + ue * ue * py) + (1 - K0_alpha) * (px * ue * ue + py)));
        const cd expP = cexpi(B - Phi * 0.5);
        const cd expM = cconj(expP);
        const int idxI = (int)((x0 - minX) / dx);
        const int idxJ = (int)((y0 - minY) / dy);
        wx[1] = (x0 - minX) / dx - idxI; wx[0] = 1.0 - wx[1];
        wy[1] = (y0 - minY) / dy - idxJ; wy[0] = 1.0 - wy[1];
        if (idxI >= 0 && idxI < nx - 1 && idxJ >= 0 && idxJ < ny - 1) {
          const double r = sqrt(r2);
          const int idxR = r / dr + 0.5;
          wr[1] = (r * r / (dr * dr) - idxR * idxR) / (2.0 * idxR);
          wr[0] = 1.0 - wr[1];
          if (idxR > 0 && idxR < nr) {
            for (int ll = 0; ll < L; ++ll) {
              Em[ll] = C(0, 0);
              for (int f = 0; f < F; ++f)
                for (int jj = 0; jj < 2; ++jj)
                  Em[ll] = cadd(Em[ll], cscale(D->Ez[ll][(size_t)sliceI * nr * F + nr * f + idxR + jj], wr[jj]));
            }
          } else if (idxR == 0) {
            for (int ll = 0; ll < L; ++ll) {
              Em[ll] = C(0, 0);
              for (int f = 0; f < F; ++f)
                for (int jj = 0; jj < 2; ++jj)
                  Em[ll] = cadd(Em[ll], D->Ez[ll][(size_t)sliceI * nr * F + nr * f + idxR + jj]);
            }
          }
          for (int h = 0; h < H_n; ++h) {
            Ux[h] = C(0, 0); Uy[h] = C(0, 0);
            for (int ii = 0; ii < 2; ++ii)
              for (int jj = 0; jj < 2; ++jj) {
                const size_t id = (size_t)sliceI * N + (idxJ + jj) * nx + (idxI + ii);
                Ux[h] = cadd(Ux[h], cscale(cscale(D->Ux[h][id], wx[ii]), wy[jj]));
                Uy[h] = cadd(Uy[h], cscale(cscale(D->Uy[h][id], wx[ii]), wy[jj]));
              }
          }
          double sumU2 = 0.0;
          for (int h = 0; h < H_n; ++h) {
            const int H = D->harmony[h];
            sumU2 += (cnorm(Ux[h]) + cnorm(Uy[h])) / (2.0 * H * H);
          }
          for (int m = 1; m < 5; ++m) {
            const double th = th0 + dz * k_th[m - 1] * coefList[m];
            const double gam = gam0 + dz * k_gam[m - 1] * coefList[m];
            double sumTh = 0.0, sumG = 0.0;
            double sumEzPart = 0.0;
            for (int ll = 0; ll < L; ++ll) {
              const cd e = cexpi((ll + 1.0) * th);
              sumEzPart += 2.0 * (Em[ll].re * e.re - Em[ll].im * e.im);
            }
            for (int h = 0; h < H_n; ++h) {
              const int H = D->harmony[h];
              int idx = (1.0 * H * xi) / dBessel;
              w[1] = (H * xi / dBessel) - idx; w[0] = 1.0 - w[1];
              if (H % 2 == 1) {
                const double sign = ((H - 1) / 2 % 2 == 0) ? 1.0 : -1.0;
                int order = (H - 1) / 2;
                const double J1 = D->BJ(idx, order) * w[0] + D->BJ(idx + 1, order) * w[1];
                order = (H + 1) / 2;
                const double J2 = D->BJ(idx, order) * w[0] + D->BJ(idx + 1, order) * w[1];
                fx = C(sign * (K0_alpha * J1 - J2), 0.0);
                fy = C(sign * (K0_alpha * J1 + J2), 0.0);
              } else {
                const double sign = (H / 2 % 2 == 0) ? 1.0 : -1.0;
                idx = (H * xi) / dBessel;
                w[1] = (H * xi / dBessel) - idx; w[0] = 1.0 - w[1];
                int order = (H - 2) / 2;
                const double J1 = D->BJ(idx, order) * w[0] + D->BJ(idx + 1, order) * w[1];
                order = H / 2;
                const double J2 = D->BJ(idx, order) * w[0] + D->BJ(idx + 1, order) * w[1];
                order = (H + 2) / 2;
                const double J3 = D->BJ(idx, order) * w[0] + D->BJ(idx + 1, order) * w[1];
                const double sx = sign * xi2 * H * 0.5;
                fx = cscale(cadd(cscale(expP, K0_alpha * J1 - J2), cscale(expM, K0_alpha * J2 - J3)), sx);
                fy = cscale(cadd(cscale(expP, K0_alpha * J1 + J2), cscale(expM, K0_alpha * J2 + J3)), sx);
              }
              const cd e = cexpi((1.0 * H) * (th + Phi * 0.5));
              const cd tmpComp = cmul(e, csub(cmul(cmul(etaX, fx), Ux[h]), cmul(cmul(etaY, fy), Uy[h])));
              // std::real(I*tmpComp) = 0*re - 1*im
              sumTh += (0.0 * tmpComp.re - 1.0 * tmpComp.im) / (1.0 * H);
              sumG += tmpComp.re / (2.0 * gam);
            }
            k_th[m] = ku - ks / (2.0 * gam * gam) * (K2 + sumU2 + K0 * sqrt(ue * ue + 1.0) * sumTh);
            k_gam[m] = ks * K0 * sqrt(ue * ue + 1.0) * sumG + e_mc2 * sumEzPart;
          }
          const double tmpTh = dz / 6.0 * (k_th[1] + 2.0 * k_th[2] + 2.0 * k_th[3] + k_th[4]);
          if (tmpTh > dPhi || tmpTh < -dPhi) overflow = 1;
          P.theta[n] += tmpTh;
          const double tmpGam = dz / 6.0 * (k_gam[1] + 2.0 * k_gam[2] + 2.0 * k_gam[3] + k_gam[4]) - dz * wakeE;
          P.gamma[n] += tmpGam;
        }
      }
      });
      if (overflow) set_err(D, FELIS_THETA_OVERFLOW, "push_theta_gamma: |dtheta| > 2 pi numSlice");
      // Em carried to the next slice: the value left by the last particle of
      // this slice that took one of the two radial-grid branches (x, y and Ez
      // are unchanged by this push, so it can be recomputed here).
      for (int64_t n = n1 - 1; n >= n0; --n) {
        const double x0 = P.x[n], y0 = P.y[n];
        const int idxI = (int)((x0 - minX) / dx), idxJ = (int)((y0 - minY) / dy);
        if (!(idxI >= 0 && idxI < nx - 1 && idxJ >= 0 && idxJ < ny - 1)) continue;
        const double r = sqrt(x0 * x0 + y0 * y0);
        const int idxR = r / dr + 0.5;
        const double wr1 = (r * r / (dr * dr) - idxR * idxR) / (2.0 * idxR), wr0 = 1.0 - wr1;
        if (!(idxR >= 0 && idxR < nr)) continue;
        for (int ll = 0; ll < L; ++ll) {
          Em[ll] = C(0, 0);
          for (int f = 0; f < F; ++f) {
            const size_t b0 = (size_t)sliceI * nr * F + nr * f;
            if (idxR > 0) {
              Em[ll] = cadd(Em[ll], cscale(D->Ez[ll][b0 + idxR], wr0));
              Em[ll] = cadd(Em[ll], cscale(D->Ez[ll][b0 + idxR + 1], wr1));
            } else {
              Em[ll] = cadd(Em[ll], D->Ez[ll][b0 + 0]);
              Em[ll] = cadd(Em[ll], D->Ez[ll][b0 + 1]);
            }
          }
        }
        break;
      }
    }
  }
}

// solveField.cpp:80-185 for one field (Un, Sc) pair.
static void solve_field_U(orc* D, std::vector<std::vector<cd>>& Un, std::vector<std::vector<cd>>& Sc) {
  const int nx = D->nx, ny = D->ny, N = D->N;
  const double currentFlag = D->currentFlag ? 1.0 : 0.0;
  for (int h = 0; h < D->numHarmony; ++h) {
    const double H = (double)D->harmony[h];
    pfor(0, D->subSliceN, D->threads, [&](int64_t lo_, int64_t hi_) {
    for (int sl = (int)lo_; sl < (int)hi_; ++sl) {
      const size_t sliceI = sl + 1;
      std::vector<cd> CCx(nx, C(0, 0)), DDx(nx, C(0, 0)), ddx(nx, C(0, 0));
      std::vector<cd> CCy(ny, C(0, 0)), DDy(ny, C(0, 0)), ddy(ny, C(0, 0));
      std::vector<cd> Uc((size_t)N, C(0, 0));
      const std::vector<cd>& al = D->alpha;
      const std::vector<cd>& alP = D->alphaP;
      const std::vector<cd>& be = D->beta;
      const std::vector<cd>& beP = D->betaP;
      for (int j = 0; j < ny; ++j) { Uc[j * nx + 0] = C(0, 0); Uc[j * nx + (nx - 1)] = C(0, 0); }
      for (int i = 0; i < nx; ++i) { Uc[0 * nx + i] = C(0, 0); Uc[(ny - 1) * nx + i] = C(0, 0); }
      for (int j = 1; j < ny - 1; ++j) {
        for (int i = 1; i < nx - 1; ++i) {
          const size_t idx = sliceI * N + j * nx + i;
          // - bP*U[+nx] + (H + bP + b)*U - b*U[-nx] + Sc*flag
          cd t = cmul(cneg(beP[j]), Un[h][idx + nx]);
          t = cadd(t, cmul(cadd(cradd(H, beP[j]), be[j]), Un[h][idx]));
          t = csub(t, cmul(be[j], Un[h][idx - nx]));
          ddx[i] = cadd(t, cscale(Sc[h][idx], currentFlag));
        }
        const cd Hx1 = csub(crsub(H, alP[1]), al[1]);
        CCx[1] = cdiv(Hx1, alP[1]);
        DDx[1] = cdiv(ddx[1], alP[1]);
        for (int i = 2; i < nx - 2; ++i) {
          const cd Hx = csub(crsub(H, alP[i]), al[i]);
          const cd Q = cmul(alP[i], CCx[i - 1]);
          CCx[i] = csub(cdiv(Hx, alP[i]), cdiv(al[i], Q));
          DDx[i] = csub(cdiv(ddx[i], alP[i]), cdiv(cmul(al[i], DDx[i - 1]), Q));
        }
        CCx[nx - 2] = csub(csub(crsub(H, alP[nx - 2]), al[nx - 2]), cdiv(C(1.0, 0.0), CCx[nx - 3]));
        DDx[nx - 2] = csub(ddx[nx - 2], cdiv(DDx[nx - 3], CCx[nx - 3]));
        Uc[j * nx + (nx - 2)] = cdiv(DDx[nx - 2], CCx[nx - 2]);
        for (int i = nx - 3; i > 0; --i) Uc[j * nx + i] = cdiv(csub(DDx[i], Uc[j * nx + (i + 1)]), CCx[i]);
      }
      for (int i = 1; i < nx - 1; ++i) {
        for (int j = 1; j < ny - 1; ++j) {
          const size_t idx = j * nx + i;
          cd t = cmul(cneg(alP[i]), Uc[idx + 1]);
          t = cadd(t, cmul(cadd(cradd(H, alP[i]), al[i]), Uc[idx]));
          t = csub(t, cmul(al[i], Uc[idx - 1]));
          ddy[j] = cadd(t, cscale(Sc[h][sliceI * N + j * nx + i], currentFlag));
        }
        const cd Hy1 = csub(crsub(H, beP[1]), be[1]);
        CCy[1] = cdiv(Hy1, beP[1]);
        DDy[1] = cdiv(ddy[1], beP[1]);
        for (int j = 2; j < ny - 1; ++j) {
          const cd Hy = csub(crsub(H, beP[j]), be[j]);
          const cd Q = cmul(beP[j], CCy[j - 1]);
          CCy[j] = csub(cdiv(Hy, beP[j]), cdiv(be[j], Q));
          DDy[j] = csub(cdiv(ddy[j], beP[j]), cdiv(cmul(be[j], DDy[j - 1]), Q));
        }
        CCy[ny - 2] = csub(csub(crsub(H, beP[ny - 2]), be[ny - 2]), cdiv(C(1.0, 0.0), CCy[ny - 3]));
        DDy[ny - 2] = csub(ddy[ny - 2], cdiv(DDy[ny - 3], CCy[ny - 3]));
        Un[h][sliceI * N + (ny - 2) * nx + i] = cdiv(DDy[ny - 2], CCy[ny - 2]);
        for (int j = ny - 3; j > 0; --j)
          Un[h][sliceI * N + j * nx + i] = cdiv(csub(DDy[j], Un[h][sliceI * N + (j + 1) * nx + i]), CCy[j]);
      }
    }
    });
  }
}

// solveField.cpp:187-403
static void solve_Sc(orc* D) {
  const int H_n = D->numHarmony, L = D->L, F = D->F;
  const double minX = D->minX, minY = D->minY;
  const int nx = D->nx, ny = D->ny, nr = D->nr, N = D->N;
  const double dx = D->dx, dy = D->dy, dz = D->dz, dr = D->dr;
  const double K0 = D->K0, ks = D->ks, dBessel = D->dBessel, ue = D->ue, gamR = D->gamR;
  double Phi;
  cd etaX, etaY;
  if (!polarisation(D, &Phi, &etaX, &etaY)) return;
  const double K0_alpha = D->K0_alpha;
  const int endI = D->subSliceN + 1;
  for (int h = 0; h < H_n; ++h)
    for (int sliceI = 0; sliceI <= endI; ++sliceI)
      for (int j = 0; j < N; ++j) {
        D->ScUx[h][(size_t)sliceI * N + j] = C(0, 0);
        D->ScUy[h][(size_t)sliceI * N + j] = C(0, 0);
      }
  const double coef_U = dz * kECharge * kECharge * kMu0 * K0 * sqrt(1.0 + ue * ue) /
                        (4.0 * ks * kEMass * (D->lambda0 * D->numSlice) * dx * dy);
  const double xi = 0.25 * K0 * K0 * (1.0 - ue * ue) / (1.0 + (1.0 + ue * ue) * K0 * K0 * 0.5);
  const double coef_Ez = kECharge * kVelocityC * kVelocityC * kMu0 * ks * (1.0 + 0.5 * (1.0 + ue * ue) * K0 * K0) /
                         (2.0 * M_PI * D->lambda0 * D->numSlice * gamR * gamR);
  for (int s = 0; s < D->nSpecies; ++s) {
    Species& P = D->sp[s];
    pfor(0, D->subSliceN, D->threads, [&](int64_t lo_, int64_t hi_) {
    for (int sl = (int)lo_; sl < (int)hi_; ++sl) {
      const int sliceI = sl + 1;
      double w[2], wx[2], wy[2];
      cd fx, fy;
      const double macro = P.weight[sl];
      for (int64_t n = P.off[sl]; n < P.off[sl + 1]; ++n) {
        const double x = P.x[n], y = P.y[n], theta = P.theta[n], gam = P.gamma[n];
        const double px = P.px[n], py = P.py[n];
        const double xi2 = sqrt(2.0) * K0 / (1.0 + K0 * K0 * 0.5 * (1.0 + ue * ue)) *
                           sqrt((1 + K0_alpha) * (px * px + ue * ue * py * py) +
                                (1 - K0_alpha) * (px * px * ue * ue + py * py));
        const double B = oatan(2.0 * K0_alpha * ue * (px - py) /
                               ((1.0 + K0_alpha) * (px + ue * ue * py) + (1 - K0_alpha) * (px * ue * ue + py)));
        const cd expP = cexpi(B - Phi * 0.5);
        const cd expM = cconj(expP);
        const int idxI = (x - minX) / dx;
        const int idxJ = (y - minY) / dy;
        const int64_t idx = (int64_t)sliceI * N + (int64_t)idxJ * nx + idxI;
        wx[1] = (x - minX) / dx - idxI; wx[0] = 1.0 - wx[1];
        wy[1] = (y - minY) / dy - idxJ; wy[0] = 1.0 - wy[1];
        if (idxI >= 0 && idxI < nx && idxJ >= 0 && idxJ < ny) {
          for (int h = 0; h < H_n; ++h) {
            const int H = D->harmony[h];
            const double dbH = (double)H;
            if (H % 2 == 1) {
              const double sign = ((H - 1) / 2 % 2 == 0) ? 1.0 : -1.0;
              const int ib = (dbH * xi) / dBessel;
              w[1] = (dbH * xi / dBessel) - ib; w[0] = 1.0 - w[1];
              int order = (H - 1) / 2;
              const double J1 = D->BJ(ib, order) * w[0] + D->BJ(ib + 1, order) * w[1];
              order = (H + 1) / 2;
              const double J2 = D->BJ(ib, order) * w[0] + D->BJ(ib + 1, order) * w[1];
              fx = C(sign * (J1 - K0_alpha * J2), 0.0);
              fy = C(sign * (J1 + K0_alpha * J2), 0.0);
            } else {
              const double sign = (H / 2 % 2 == 0) ? 1.0 : -1.0;
              const int ib = (dbH * xi) / dBessel;
              w[1] = (dbH * xi / dBessel) - ib; w[0] = 1.0 - w[1];
              int order = (H - 2) / 2;
              const double J1 = D->BJ(ib, order) * w[0] + D->BJ(ib + 1, order) * w[1];
              order = H / 2;
              const double J2 = D->BJ(ib, order) * w[0] + D->BJ(ib + 1, order) * w[1];
              order = (H + 2) / 2;
              const double J3 = D->BJ(ib, order) * w[0] + D->BJ(ib + 1, order) * w[1];
              const double sx = sign * xi2 * dbH * 0.5;
              fx = cscale(cadd(cscale(expM, J1 - K0_alpha * J2), cscale(expP, J2 - K0_alpha * J3)), sx);
              fy = cscale(cadd(cscale(expM, J1 + K0_alpha * J2), cscale(expP, J2 + K0_alpha * J3)), sx);
            }
            // dbH*macro*coef_U*exp(-I*dbH*(theta+Phi*0.5))/gam
            const cd e = cexpi((-1.0 * dbH) * (theta + Phi * 0.5));
            const cd mc = cdivr(cscale(e, dbH * macro * coef_U), gam);
            for (int ii = 0; ii < 2; ++ii)
              for (int jj = 0; jj < 2; ++jj) {
                const int64_t t = idx + jj * nx + ii;
                const cd ax = cmul(cmul(cscale(cscale(etaX, wx[ii]), wy[jj]), fx), mc);
                const cd ay = cmul(cmul(cscale(cscale(etaY, wx[ii]), wy[jj]), fy), mc);
                // The reference can write one cell past a row (q6); such
                // writes stay inside the (slice_n+2)-plane array.
                if (t >= 0 && t < (int64_t)(D->subSliceN + 2) * N) {
                  D->ScUx[h][t] = csub(D->ScUx[h][t], ax);
                  D->ScUy[h][t] = csub(D->ScUy[h][t], ay);
                }
              }
          }
        }
      }
    }
    });
    // Ez space charge (solveField.cpp:315-399); D->Ez keeps the last species' solve.
    const double A = ks * ks * (1.0 + 0.5 * (1.0 + ue * ue) * K0 * K0) / (gamR * gamR) * dr * dr;
    pfor(0, D->subSliceN, D->threads, [&](int64_t lo_, int64_t hi_) {
    for (int sl = (int)lo_; sl < (int)hi_; ++sl) {
      const int sliceI = sl + 1;
      std::vector<std::vector<cd>> Sc(L, std::vector<cd>((size_t)F * nr + 1, C(0, 0)));
      std::vector<double> a(nr), b(nr), c(nr);
      std::vector<cd> d(nr);
      double wr[2];
      const double macro = P.weight[sl];
      for (int64_t n = P.off[sl]; n < P.off[sl + 1]; ++n) {
        const double x = P.x[n], y = P.y[n], theta = P.theta[n];
        const double phi = (x == 0.0) ? 0.0 : oatan2(y, x);
        const double r = sqrt(x * x + y * y);
        const int idxR = r / dr + 0.5;
        wr[1] = (r * r / (dr * dr) - idxR * idxR) / (2.0 * idxR);
        wr[0] = 1.0 - wr[1];
        if (idxR > 0 && idxR < nr) {
          for (int l = 0; l < L; ++l)
            for (int f = 0; f < F; ++f) {
              const cd e = cexpi(-1.0 * ((l + 1) * theta + f * phi));
              // I*coef_Ez*(l+1.0) = (0*c*(l+1)..., c*(l+1))
              const cd ic = C(0.0 * coef_Ez * (l + 1.0), 1.0 * coef_Ez * (l + 1.0));
              const cd coefComp = cdivr(cscale(cmul(ic, e), macro), 1.0 * idxR);
              for (int jj = 0; jj < 2; ++jj) {
                const size_t t = (size_t)f * nr + idxR + jj;
                // t == F*nr is the reference's one-past-the-end write (q6 for Ez)
                Sc[l][t] = cadd(Sc[l][t], cscale(coefComp, wr[jj]));
              }
            }
        } else if (idxR == 0) {
          for (int l = 0; l < L; ++l) {
            const cd e = cexpi(-1.0 * ((l + 1) * theta));
            const cd ic = C(0.0 * coef_Ez * (l + 1.0), 1.0 * coef_Ez * (l + 1.0));
            const cd coefComp = cscale(cmul(ic, e), macro);
            Sc[l][idxR] = cadd(Sc[l][idxR], coefComp);
            for (int f = 1; f < F; ++f) Sc[l][(size_t)f * nr + idxR] = C(0, 0);
          }
        }
      }
      for (int f = 0; f < F; ++f)
        for (int l = 0; l < L; ++l) {
          if (f == 0) {
            a[0] = 1.0; b[0] = -(1.0 + (l + 1.0) * (l + 1.0) * A / 8.0); c[0] = 0.0; d[0] = Sc[l][0];
          } else {
            a[0] = 0.0; b[0] = 1.0; c[0] = 0.0; d[0] = C(0, 0);
          }
          for (int j = 1; j < nr - 1; ++j) {
            a[j] = j + 0.5;
            b[j] = -2.0 * j - (l + 1.0) * (l + 1.0) * A * j - f * f * ::log((j + 0.5) / (j - 0.5));
            c[j] = j - 0.5;
            d[j] = Sc[l][(size_t)f * nr + j];
          }
          a[nr - 1] = 0.0; b[nr - 1] = 1.0; c[nr - 1] = 0.0; d[nr - 1] = C(0, 0);
          for (int j = 1; j < nr; ++j) {
            const double ww = c[j] / b[j - 1];
            b[j] -= ww * a[j - 1];
            d[j] = csub(d[j], cscale(d[j - 1], ww));
          }
          // Back-substitution reads slice 0's storage (q2), which is always zero.
          D->Ez[l][(size_t)f * nr + nr - 1] = C(0, 0);
          for (int j = nr - 2; j >= 0; --j) {
            const cd ez0 = D->Ez[l][(size_t)f * nr + j + 1];
            D->Ez[l][(size_t)sliceI * F * nr + (size_t)f * nr + j] = cdivr(csub(d[j], cscale(ez0, a[j])), b[j]);
          }
        }
    }
    });
  }
}

// solveField.cpp:422-549 (1D): per slice, the source of every harmonic and
// the longitudinal space-charge modes, summed over the slice's particles in
// order (species by species).
static void solve_sc_1d(orc* D) {
  const int H_n = D->numHarmony, L = D->L;
  double Phi;
  cd etaX, etaY;
  if (!polarisation(D, &Phi, &etaX, &etaY)) return;
  const double K0_alpha = D->K0_alpha;
  const int endI = D->subSliceN + 1;
  const double dz = D->dz, ks = D->ks, K0 = D->K0, dBessel = D->dBessel, ue = D->ue;
  const double xi = 0.25 * K0 * K0 * (1.0 - ue * ue) / (1.0 + (1.0 + ue * ue) * K0 * K0 * 0.5);
  for (int s = 0; s < D->nSpecies; ++s) {
    Species& P = D->sp[s];
    const double area = D->area[s];
    const double coef = dz * kECharge * kECharge * kMu0 * K0 * sqrt(1.0 + ue * ue) /
                        (2.0 * ks * kEMass * (D->lambda0 * D->numSlice) * area);
    pfor(0, D->subSliceN, D->threads, [&](int64_t lo_, int64_t hi_) {
    for (int sl = (int)lo_; sl < (int)hi_; ++sl) {
      const int sliceI = sl + 1;
      const double macro = P.weight[sl];
      for (int64_t n = P.off[sl]; n < P.off[sl + 1]; ++n) {
        const double th = P.theta[n], gam = P.gamma[n];
        for (int h = 0; h < H_n; ++h) {
          const int H = D->harmony[h];
          cd fx = C(0, 0), fy = C(0, 0);
          if (H % 2 == 1) {
            const double sign = ((H - 1) / 2 % 2 == 0) ? 1.0 : -1.0;
            const int idx = (int)(H * xi / dBessel);
            double w[2];
            w[1] = (H * xi / dBessel) - idx; w[0] = 1.0 - w[1];
            int order = (H - 1) / 2;
            const double J1 = D->BJ(idx, order) * w[0] + D->BJ(idx + 1, order) * w[1];
            order = (H + 1) / 2;
            const double J2 = D->BJ(idx, order) * w[0] + D->BJ(idx + 1, order) * w[1];
            fx = C(sign * (J1 - K0_alpha * J2), 0.0);
            fy = C(sign * (J1 + K0_alpha * J2), 0.0);
          }
          // macro*coef*exp((-1.0*H)*I*(th+Phi*0.5))/gam
          const cd m = cdivr(cscale(cexpi((-1.0 * H) * (th + Phi * 0.5)), macro * coef), gam);
          D->ScUx[h][sliceI] = csub(D->ScUx[h][sliceI], cmul(cmul(etaX, fx), m));
          D->ScUy[h][sliceI] = csub(D->ScUy[h][sliceI], cmul(cmul(etaY, fy), m));
        }
      }
    }
    });
  }
  for (int l = 0; l < L; ++l)
    for (int sliceI = 0; sliceI <= endI; ++sliceI) D->Ez[l][sliceI] = C(0, 0);
  for (int s = 0; s < D->nSpecies; ++s) {
    Species& P = D->sp[s];
    const double area = D->area[s];
    const double coef = kECharge * kVelocityC * kVelocityC * kMu0 / ks / area / (D->lambda0 * D->numSlice);
    pfor(0, D->subSliceN, D->threads, [&](int64_t lo_, int64_t hi_) {
    for (int sl = (int)lo_; sl < (int)hi_; ++sl) {
      const int sliceI = sl + 1;
      const double macro = P.weight[sl];
      for (int64_t n = P.off[sl]; n < P.off[sl + 1]; ++n) {
        const double th = P.theta[n];
        for (int l = 0; l < L; ++l) {
          // -1.0*I*coef/(1.0+l)*macro*exp(-I*(l+1.0)*th), left to right
          cd t = C(-0.0, -1.0);
          t = cscale(t, coef);
          t = cdivr(t, 1.0 + l);
          t = cscale(t, macro);
          t = cmul(t, cexpi(-((l + 1.0) * th)));
          D->Ez[l][sliceI] = cadd(D->Ez[l][sliceI], t);
        }
      }
    }
    });
  }
}

// particlePush.cpp:388-524 (1D): RK4 of (theta, gamma) in the slice's field
// value and space-charge modes, with the constant xi of the 1D model.
static void push_theta_gamma_1d(orc* D) {
  const int L = D->L, H_n = D->numHarmony;
  const double ue = D->ue, ks = D->ks, ku = D->ku, K0 = D->K0, dz = D->dz, dBessel = D->dBessel;
  const double dPhi = 2.0 * M_PI * D->numSlice;
  const double e_mc2 = kECharge / kEMass / kVelocityC / kVelocityC;
  double Phi;
  cd etaX, etaY;
  if (!polarisation(D, &Phi, &etaX, &etaY)) return;
  const double K0_alpha = D->K0_alpha;
  const double K2 = 1.0 + K0 * K0 * 0.5 * (1.0 + ue * ue);
  const double coefList[5] = {0, 0, 0.5, 0.5, 1};
  const double xi = 0.25 * K0 * K0 * (1.0 - ue * ue) / (1.0 + (1.0 + ue * ue) * K0 * K0 * 0.5);
  for (int s = 0; s < D->nSpecies; ++s) {
    Species& P = D->sp[s];
    for (int sl = 0; sl < D->subSliceN; ++sl) {
      const int sliceI = sl + 1;
      const double wakeE = D->wakeON ? D->wakeE[sliceI - 1 + D->minI] / (kMc2 * 1.0e6) : 0.0;
      cd Em[4], Ux[FELIS_MAX_HARMONY], Uy[FELIS_MAX_HARMONY];
      for (int ll = 0; ll < L; ++ll) Em[ll] = D->Ez[ll][sliceI];
      for (int h = 0; h < H_n; ++h) { Ux[h] = D->Ux[h][sliceI]; Uy[h] = D->Uy[h][sliceI]; }
      double sumU2 = 0.0;
      for (int h = 0; h < H_n; ++h) {
        const int H = D->harmony[h];
        sumU2 += (cnorm(Ux[h]) + cnorm(Uy[h])) / (2.0 * H * H);
      }
      std::atomic<int> overflow{0};
      pfor(P.off[sl], P.off[sl + 1], D->threads, [&](int64_t lo_, int64_t hi_) {
      for (int64_t n = lo_; n < hi_; ++n) {
        const double th0 = P.theta[n], gam0 = P.gamma[n];
        double k_th[5] = {0, 0, 0, 0, 0}, k_gam[5] = {0, 0, 0, 0, 0};
        for (int m = 1; m < 5; ++m) {
          const double th = th0 + dz * k_th[m - 1] * coefList[m];
          const double gam = gam0 + dz * k_gam[m - 1] * coefList[m];
          double sumTh = 0.0, sumG = 0.0, sumEzPart = 0.0;
          for (int ll = 0; ll < L; ++ll) {
            const cd e = cexpi((ll + 1.0) * th);
            sumEzPart += 2.0 * (Em[ll].re * e.re - Em[ll].im * e.im);
          }
          for (int h = 0; h < H_n; ++h) {
            const int H = D->harmony[h];
            const double sign = ((H - 1) / 2 % 2 == 0) ? 1.0 : -1.0;
            const int idx = (1.0 * H * xi) / dBessel;
            double w[2];
            w[1] = (H * xi / dBessel) - idx; w[0] = 1.0 - w[1];
            cd fx = C(0, 0), fy = C(0, 0);
            if (H % 2 == 1) {
              int order = (H - 1) * 0.5;
              const double J1 = D->BJ(idx, order) * w[0] + D->BJ(idx + 1, order) * w[1];
              order = (H + 1) * 0.5;
              const double J2 = D->BJ(idx, order) * w[0] + D->BJ(idx + 1, order) * w[1];
              fx = C(sign * (K0_alpha * J1 - J2), 0.0);
              fy = C(sign * (K0_alpha * J1 + J2), 0.0);
            }
            const cd e = cexpi((1.0 * H) * (th + Phi * 0.5));
            const cd tmpComp = cmul(e, csub(cmul(cmul(etaX, fx), Ux[h]), cmul(cmul(etaY, fy), Uy[h])));
            sumTh += (0.0 * tmpComp.re - 1.0 * tmpComp.im) / (1.0 * H);
            sumG += tmpComp.re / (2.0 * gam);
          }
          k_th[m] = ku - ks / (2.0 * gam * gam) * (K2 + sumU2 + K0 * sqrt(ue * ue + 1.0) * sumTh);
          k_gam[m] = ks * K0 * sqrt(ue * ue + 1.0) * sumG + e_mc2 * sumEzPart;
        }
        const double tmpTh = dz / 6.0 * (k_th[1] + 2.0 * k_th[2] + 2.0 * k_th[3] + k_th[4]);
        if (tmpTh > dPhi || tmpTh <= -dPhi) overflow = 1;
        P.theta[n] += tmpTh;
        const double tmpGam = dz / 6.0 * (k_gam[1] + 2 * k_gam[2] + 2 * k_gam[3] + k_gam[4]) - dz * wakeE;
        P.gamma[n] += tmpGam;
      }
      });
      if (overflow) set_err(D, FELIS_THETA_OVERFLOW, "push_theta_gamma: |dtheta| > 2 pi numSlice");
    }
  }
}

// solveField.cpp:49-78
static void solve_field(orc* D) {
  for (int h = 0; h < D->numHarmony; ++h)
    for (int sliceI = 0; sliceI < D->subSliceN + 2; ++sliceI) {
      D->ScUx[h][sliceI] = C(0, 0);
      D->ScUy[h][sliceI] = C(0, 0);
    }
  if (D->dimension == 1) {
    // solveField.cpp:61-66, 409-416: U += ScU per slice
    if (D->currentFlag) solve_sc_1d(D);
    for (int h = 0; h < D->numHarmony; ++h)
      for (int sliceI = 1; sliceI < D->subSliceN + 1; ++sliceI) {
        D->Ux[h][sliceI] = cadd(D->Ux[h][sliceI], D->ScUx[h][sliceI]);
        D->Uy[h][sliceI] = cadd(D->Uy[h][sliceI], D->ScUy[h][sliceI]);
      }
    return;
  }
  if (D->currentFlag) solve_Sc(D);
  solve_field_U(D, D->Ux, D->ScUx);
  solve_field_U(D, D->Uy, D->ScUy);
}

// [Phase_shifter] (README.md:57-70; the reference's parser does not read the
// block, so this follows the project's reading of it): the shifters whose z
// lies in [it dz, (it+1) dz) delay every electron by phase * pi of theta,
// applied after the push or drift and before the wrap.
static void phase_shift(orc* D, int it) {
  double d = 0.0;
  const double z0 = it * D->dz, z1 = (it + 1) * D->dz;
  for (size_t k = 0; k < D->psZ.size(); ++k)
    if (D->psZ[k] >= z0 && D->psZ[k] < z1) d -= M_PI * D->psPhase[k];
  if (d == 0.0) return;
  for (int s = 0; s < D->nSpecies; ++s) {
    Species& P = D->sp[s];
    const int64_t cnt = P.off[D->subSliceN];
    for (int64_t n = 0; n < cnt; ++n) P.theta[n] += d;
  }
}

// rearrangeParticles.cpp:77-114
static void periodic_particles(orc* D) {
  const double dTh = D->numSlice * 2 * M_PI;
  for (int s = 0; s < D->nSpecies; ++s) {
    Species& P = D->sp[s];
    const int64_t cnt = P.off[D->subSliceN];
    std::atomic<int> bad{0};
    pfor(0, cnt, D->threads, [&](int64_t lo_, int64_t hi_) {
    for (int64_t n = (int64_t)lo_; n < (int64_t)hi_; ++n) {
      double delTh = 0.0;
      const double theta = P.theta[n];
      int intTh = 0;
      if (theta >= dTh) {
        intTh = theta / dTh;
        delTh = dTh * intTh;
      } else if (theta < 0) {
        intTh = theta / dTh - 1.0;
        delTh = dTh * intTh;
      }
      P.theta[n] -= delTh;
      if (P.theta[n] > dTh || P.theta[n] < 0) bad = 1;
    }
    });
    if (bad) set_err(D, FELIS_OUT_OF_RANGE, "periodicParticles: theta outside [0, dTh] after wrap");
  }
}

// solveField.cpp:19-47
static void shift_field(orc* D) {
  const size_t N = D->N;
  for (int h = 0; h < D->numHarmony; ++h)
    for (int sliceI = D->subSliceN + 1; sliceI >= 1; --sliceI) {
      memcpy(&D->Ux[h][sliceI * N], &D->Ux[h][(sliceI - 1) * N], N * sizeof(cd));
      memcpy(&D->Uy[h][sliceI * N], &D->Uy[h][(sliceI - 1) * N], N * sizeof(cd));
    }
}

// updateTotalEnergy.cpp:25-36
static void total_energy(orc* D, double* out) {
  const size_t N = D->N;
  for (int h = 0; h < D->numHarmony; ++h) {
    double totalX = 0.0, totalY = 0.0;
    for (int sliceI = 1; sliceI < D->subSliceN + 1; ++sliceI)
      for (size_t j = 0; j < N; ++j) {
        totalX += cnorm(D->Ux[h][sliceI * N + j]);
        totalY += cnorm(D->Uy[h][sliceI * N + j]);
      }
    out[2 * h] = totalX;
    out[2 * h + 1] = totalY;
  }
}

// twiss.cpp:138-192
static void twiss(orc* D, double* out) {
  for (int s = 0; s < D->nSpecies; ++s) {
    Species& P = D->sp[s];
    double aveX2 = 0, aveY2 = 0, aveXPrime = 0, aveYPrime = 0, aveCrsX = 0, aveCrsY = 0, cnt = 0;
    const int64_t n1 = P.off[D->subSliceN];
    for (int64_t n = 0; n < n1; ++n) {
      const double x = P.x[n], y = P.y[n], px = P.px[n], py = P.py[n], gam = P.gamma[n];
      const double invGam = 1.0 / gam;
      const double xPrime = px * invGam, yPrime = py * invGam;
      aveX2 += x * x; aveY2 += y * y;
      aveXPrime += xPrime * xPrime; aveYPrime += yPrime * yPrime;
      aveCrsX += x * xPrime; aveCrsY += y * yPrime;
      cnt += 1.0;
    }
    double* o = out + 6 * s;
    for (int k = 0; k < 6; ++k) o[k] = 0.0;
    if (cnt > 0.0) {
      const double avgX2 = aveX2 / cnt, avgY2 = aveY2 / cnt;
      const double avgXPrime = aveXPrime / cnt, avgYPrime = aveYPrime / cnt;
      const double avgCrsX = aveCrsX / cnt, avgCrsY = aveCrsY / cnt;
      const double emitX = sqrt(avgX2 * avgXPrime - avgCrsX * avgCrsX);
      const double emitY = sqrt(avgY2 * avgYPrime - avgCrsY * avgCrsY);
      o[0] = emitX; o[1] = avgX2 / emitX; o[2] = -avgCrsX / emitX;
      o[3] = emitY; o[4] = avgY2 / emitY; o[5] = -avgCrsY / emitY;
    }
  }
}

// saveFile.cpp:109-154 (b / totalN)
static void bfactor(orc* D, double* out) {
  double totalN = 0.0;
  for (int h = 0; h < D->numHarmony; ++h) {
    const double H = D->harmony[h];
    cd b = C(0, 0);
    for (int sl = 0; sl < D->subSliceN; ++sl)
      for (int s = 0; s < D->nSpecies; ++s) {
        Species& P = D->sp[s];
        const double weight = P.weight[sl];
        for (int64_t n = P.off[sl]; n < P.off[sl + 1]; ++n) {
          b = cadd(b, cscale(cexpi(H * P.theta[n]), weight));
          if (h == 0) totalN += weight;
        }
      }
    out[2 * h] = b.re / totalN;
    out[2 * h + 1] = b.im / totalN;
  }
}

// The unfinished sums behind twiss() and bfactor(), for reductions across
// processes (twiss.cpp:46-64 before MPI_Allreduce; saveFile.cpp:126-137):
// per species sum x^2, y^2, x'^2, y'^2, x x', y y', count; per harmonic
// sum w cos(H theta), sum w sin(H theta); sum w.
static void diagnostic_sums(orc* D, double* out) {
  int k = 0;
  for (int s = 0; s < D->nSpecies; ++s) {
    Species& P = D->sp[s];
    double a[7] = {0, 0, 0, 0, 0, 0, 0};
    const int64_t n1 = P.off[D->subSliceN];
    for (int64_t n = 0; n < n1; ++n) {
      const double x = P.x[n], y = P.y[n], invGam = 1.0 / P.gamma[n];
      const double xPrime = P.px[n] * invGam, yPrime = P.py[n] * invGam;
      a[0] += x * x; a[1] += y * y; a[2] += xPrime * xPrime; a[3] += yPrime * yPrime;
      a[4] += x * xPrime; a[5] += y * yPrime; a[6] += 1.0;
    }
    for (int j = 0; j < 7; ++j) out[k++] = a[j];
  }
  double totalN = 0.0;
  for (int h = 0; h < D->numHarmony; ++h) {
    cd b = C(0, 0);
    for (int sl = 0; sl < D->subSliceN; ++sl)
      for (int s = 0; s < D->nSpecies; ++s) {
        Species& P = D->sp[s];
        for (int64_t n = P.off[sl]; n < P.off[sl + 1]; ++n) {
          b = cadd(b, cscale(cexpi(D->harmony[h] * P.theta[n]), P.weight[sl]));
          if (h == 0) totalN += P.weight[sl];
        }
      }
    out[k++] = b.re;
    out[k++] = b.im;
  }
  out[k] = totalN;
}

extern "C" {

orc* orc_create(const felis_params* p, int threads) {
  if (!p || (p->dimension != 3 && p->dimension != 1) || p->num_harmony < 1 || p->num_harmony > FELIS_MAX_HARMONY)
    return nullptr;
  orc* D = new orc();
  D->err = 0;
  D->msg[0] = 0;
  D->threads = threads > 0 ? threads : 1;
  D->dimension = p->dimension;
  for (int k = 0; k < FELIS_MAX_SPECIES; ++k) D->area[k] = p->beam_area[k];
  D->mode = p->mode;
  D->numHarmony = p->num_harmony;
  D->harmony.assign(p->harmony, p->harmony + p->num_harmony);
  D->sliceN = p->global_slice_n;
  D->subSliceN = p->slice_n;
  D->minI = p->min_i;
  D->nx = p->nx; D->ny = p->ny; D->N = p->nx * p->ny;
  D->numSlice = p->num_slice;
  D->nSpecies = p->num_species;
  D->L = p->scl_mode; D->F = p->scf_mode; D->nr = p->nr;
  D->bn = p->bessel_rows; D->bcols = p->bessel_cols;
  D->abcN = p->abc_n; D->abcSig = p->abc_sig;
  D->wakeON = p->wake_on; D->maxStep = p->max_step;
  if (p->num_phase_shifts > 0) {
    D->psZ.assign(p->phase_shift_z, p->phase_shift_z + p->num_phase_shifts);
    D->psPhase.assign(p->phase_shift_phase, p->phase_shift_phase + p->num_phase_shifts);
  }
  D->ks = p->ks; D->lambda0 = p->lambda0; D->dz = p->dz; D->dx = p->dx; D->dy = p->dy; D->dr = p->dr;
  D->minX = p->min_x; D->minY = p->min_y; D->minZ = p->min_z; D->maxZ = p->max_z;
  D->gamma0 = p->gamma0; D->gamR = p->gam_r; D->dBessel = p->d_bessel;
  D->K0 = p->K0_init; D->ue = p->ue_init; D->lambdaU = p->lambdaU_init;
  D->ku = 2.0 * M_PI / p->lambdaU_init;
  D->g = 0.0;
  D->K0_alpha = p->K0_alpha_init; D->undType = p->und_type_init;
  D->currentFlag = false; D->driftFlag = false;
  for (int u = 0; u < p->num_undulators; ++u) {
    const felis_undulator& U = p->undulators[u];
    Und o;
    o.type = U.type; o.K0_alpha = U.K0_alpha; o.numbers = U.numbers; o.air = U.air;
    o.lambdaU = U.lambdaU; o.slopeK = U.slopeK; o.ue = U.ue;
    o.unitStart.assign(U.unit_start, U.unit_start + U.numbers);
    o.unitEnd.assign(U.unit_end, U.unit_end + U.numbers);
    o.undStart.assign(U.und_start, U.und_start + U.numbers);
    o.undEnd.assign(U.und_end, U.und_end + U.numbers);
    o.K0.assign(U.K0, U.K0 + U.numbers);
    D->und.push_back(o);
  }
  for (int q = 0; q < p->num_quads; ++q) {
    const felis_quad& Q = p->quads[q];
    Quad o;
    o.numbers = Q.numbers;
    o.unitStart.assign(Q.unit_start, Q.unit_start + Q.numbers);
    o.unitEnd.assign(Q.unit_end, Q.unit_end + Q.numbers);
    o.qdStart.assign(Q.qd_start, Q.qd_start + Q.numbers);
    o.qdEnd.assign(Q.qd_end, Q.qd_end + Q.numbers);
    o.g.assign(Q.g, Q.g + Q.numbers);
    D->quad.push_back(o);
  }
  if (D->dimension == 3) build_abc(D);
  D->bessel.assign(p->bessel, p->bessel + (size_t)p->bessel_rows * p->bessel_cols);
  if (p->wake_e) D->wakeE.assign(p->wake_e, p->wake_e + p->global_slice_n);
  else D->wakeE.assign(p->global_slice_n, 0.0);
  const size_t fs = (size_t)(D->subSliceN + 2) * D->N;
  D->Ux.assign(D->numHarmony, std::vector<cd>(fs, C(0, 0)));
  D->Uy = D->Ux; D->ScUx = D->Ux; D->ScUy = D->Ux;
  D->Ez.assign(D->L, std::vector<cd>((size_t)(D->subSliceN + 2) * D->nr * D->F, C(0, 0)));
  D->sp.resize(D->nSpecies);
  for (auto& s : D->sp) {
    s.off.assign(D->subSliceN + 1, 0);
    s.weight.assign(D->subSliceN, 0.0);
  }
  return D;
}

void orc_destroy(orc* D) { delete D; }
const char* orc_error(orc* D) { return D->msg; }
void orc_set_threads(orc* D, int threads) { D->threads = threads > 0 ? threads : 1; }

int orc_set_particles(orc* D, int s, const double* x, const double* y, const double* px, const double* py,
                      const double* theta, const double* gamma, const int64_t* off, const double* weight) {
  if (s < 0 || s >= D->nSpecies) return FELIS_BAD_ARG;
  Species& P = D->sp[s];
  P.off.assign(off, off + D->subSliceN + 1);
  P.weight.assign(weight, weight + D->subSliceN);
  const int64_t n = off[D->subSliceN];
  P.x.assign(x, x + n); P.y.assign(y, y + n); P.px.assign(px, px + n); P.py.assign(py, py + n);
  P.theta.assign(theta, theta + n); P.gamma.assign(gamma, gamma + n);
  return 0;
}

int orc_get_particles(orc* D, int s, double* x, double* y, double* px, double* py, double* theta, double* gamma) {
  if (s < 0 || s >= D->nSpecies) return FELIS_BAD_ARG;
  Species& P = D->sp[s];
  const size_t n = P.x.size() * sizeof(double);
  memcpy(x, P.x.data(), n); memcpy(y, P.y.data(), n); memcpy(px, P.px.data(), n);
  memcpy(py, P.py.data(), n); memcpy(theta, P.theta.data(), n); memcpy(gamma, P.gamma.data(), n);
  return 0;
}

static std::vector<std::vector<cd>>* field_of(orc* D, int which) {
  switch (which) {
    case 0: return &D->Ux;
    case 1: return &D->Uy;
    case 2: return &D->ScUx;
    case 3: return &D->ScUy;
    default: return nullptr;
  }
}

int orc_set_field(orc* D, int h, int which, const double* data) {
  auto* f = field_of(D, which);
  if (!f || h < 0 || h >= D->numHarmony) return FELIS_BAD_ARG;
  memcpy((*f)[h].data(), data, (*f)[h].size() * sizeof(cd));
  return 0;
}
int orc_get_field(orc* D, int h, int which, double* data) {
  auto* f = field_of(D, which);
  if (!f || h < 0 || h >= D->numHarmony) return FELIS_BAD_ARG;
  memcpy(data, (*f)[h].data(), (*f)[h].size() * sizeof(cd));
  return 0;
}
int orc_get_ez(orc* D, double* data) {
  const size_t n = (size_t)(D->subSliceN + 2) * D->nr * D->F;
  for (int l = 0; l < D->L; ++l) memcpy(data + 2 * n * l, D->Ez[l].data(), n * sizeof(cd));
  return 0;
}
int orc_set_ez(orc* D, const double* data) {
  const size_t n = (size_t)(D->subSliceN + 2) * D->nr * D->F;
  for (int l = 0; l < D->L; ++l) memcpy(D->Ez[l].data(), data + 2 * n * l, n * sizeof(cd));
  return 0;
}
void orc_get_abc(orc* D, double* alpha, double* alphaP, double* beta, double* betaP) {
  memcpy(alpha, D->alpha.data(), D->nx * sizeof(cd));
  memcpy(alphaP, D->alphaP.data(), D->nx * sizeof(cd));
  memcpy(beta, D->beta.data(), D->ny * sizeof(cd));
  memcpy(betaP, D->betaP.data(), D->ny * sizeof(cd));
}

int orc_update_lattice(orc* D, int it, double half) {
  update_lattice(D, it, half);
  return 0;
}
void orc_get_lattice(orc* D, felis_lattice* o) {
  o->K0 = D->K0; o->ue = D->ue; o->lambdaU = D->lambdaU; o->ku = D->ku; o->g = D->g;
  o->K0_alpha = D->K0_alpha; o->und_type = D->undType;
  o->current_flag = D->currentFlag; o->drift_flag = D->driftFlag;
}
void orc_set_lattice(orc* D, const felis_lattice* o) {
  D->K0 = o->K0; D->ue = o->ue; D->lambdaU = o->lambdaU; D->ku = o->ku; D->g = o->g;
  D->K0_alpha = o->K0_alpha; D->undType = o->und_type;
  D->currentFlag = o->current_flag != 0; D->driftFlag = o->drift_flag != 0;
}

#define ORC_CALL(expr) do { D->err = 0; D->msg[0] = 0; expr; return D->err; } while (0)
int orc_transverse_push(orc* D) { ORC_CALL(transverse_push(D)); }
int orc_push_theta_gamma(orc* D) { ORC_CALL(push_theta_gamma(D)); }
int orc_drift_theta_gamma(orc* D) { ORC_CALL(drift_theta_gamma(D)); }
int orc_solve_field(orc* D) { ORC_CALL(solve_field(D)); }
int orc_periodic_particles(orc* D) { ORC_CALL(periodic_particles(D)); }
int orc_phase_shift(orc* D, int it) { ORC_CALL(phase_shift(D, it)); }
int orc_shift_field(orc* D) { ORC_CALL(shift_field(D)); }
void orc_total_energy(orc* D, double* out) { total_energy(D, out); }
void orc_twiss(orc* D, double* out) { twiss(D, out); }
void orc_bfactor(orc* D, double* out) { bfactor(D, out); }
void orc_diagnostic_sums(orc* D, double* out) { diagnostic_sums(D, out); }

// main.cpp:117-155 for iterations [it0, it1).  Diagnostics per iteration are
// written when the pointers are non-null (2H energy, 6*species twiss, 2H bfactor).
int orc_run(orc* D, int it0, int it1, double* energy, double* tw, double* bf) {
  const int H2 = 2 * D->numHarmony, T6 = 6 * D->nSpecies;
  for (int it = it0; it < it1; ++it) {
    D->err = 0;
    D->msg[0] = 0;
    if (energy) total_energy(D, energy + (size_t)(it - it0) * H2);
    if (tw) twiss(D, tw + (size_t)(it - it0) * T6);
    if (bf) bfactor(D, bf + (size_t)(it - it0) * H2);
    solve_field(D);
    update_lattice(D, it, 0);
    transverse_push(D);
    update_lattice(D, it, 0.5);
    transverse_push(D);
    if (!D->driftFlag) push_theta_gamma(D);
    else drift_theta_gamma(D);
    phase_shift(D, it);
    periodic_particles(D);
    if (!D->driftFlag && D->mode == FELIS_TIME_DEPENDENT) shift_field(D);
    if (D->err) return D->err;
  }
  return 0;
}

int orc_build_flags(void) {
  int f = 0;
#ifdef ORACLE_SYSTEM_LIBM
  f |= 1;
#endif
#ifdef __FAST_MATH__
  f |= 2;
#endif
#ifdef _OPENMP
  f |= 4;
#endif
  return f;
}

}  // extern "C"
