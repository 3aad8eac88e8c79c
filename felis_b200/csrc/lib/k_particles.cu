// Particle kernels of the FELIS slice loop, FP64 plain path.
//
// Compiled with --fmad=false: every expression below is evaluated with the
// operand order of the reference (particlePush.cpp, solveField.cpp,
// rearrangeParticles.cpp) and no contraction, so the results equal the CPU
// restatement bit for bit.  One thread owns one particle; a block owns one
// tile of <= 256 consecutive particles of one (species, slice), so the
// slice's field plane, weight and wake term are uniform per block.
//
// Data layout in HBM: six FP64 structure-of-arrays (x, y, px, py, theta,
// gamma), species-major then slice-major; loads and stores are coalesced
// 8-byte accesses, 2 KB per array per block.
#include "particles.cuh"

namespace felis {

namespace {

// Bessel table lookup with the row clamped to the table (the reference reads
// past the table when H*xi approaches its end; the clamp is flagged).
__device__ __forceinline__ double BJ(const DevGeom& G, int row, int col, int* err) {
  if (row < 0 || row >= G.bn) {
    set_flag(err, ERR_RADIAL);
    row = row < 0 ? 0 : G.bn - 1;
  }
  return __ldg(G.bessel + (size_t)row * G.bcols + col);
}

// particlePush.cpp:82-110 for one particle.
__device__ __forceinline__ void transverse_one(const TransCoef& t, double& x_, double& y_, double& px_, double& py_,
                                               double gam) {
  const double coefList[5] = {0, 0, 0.5, 0.5, 1};
  double k_xL[5] = {0, 0, 0, 0, 0}, k_yL[5] = {0, 0, 0, 0, 0};
  double k_pxL[5] = {0, 0, 0, 0, 0}, k_pyL[5] = {0, 0, 0, 0, 0};
  const double dz = t.dz, ku = t.ku, K0 = t.K0, ue = t.ue, aa = t.aa, bb = t.bb, cc = t.cc;
  const int K0_alpha = t.K0_alpha;
  const double x0 = x_, y0 = y_, px0 = px_, py0 = py_;
  const double dd = ku * K0 * K0 / (4.0 * gam * gam) * ue;
#pragma unroll
  for (int m = 1; m < 5; ++m) {
    const double x = x0 + dz * k_xL[m - 1] * coefList[m];
    const double y = y0 + dz * k_yL[m - 1] * coefList[m];
    const double px = px0 + dz * k_pxL[m - 1] * coefList[m];
    const double py = py0 + dz * k_pyL[m - 1] * coefList[m];
    k_xL[m] = px / gam - aa * (K0_alpha * x + y) / (gam * gam);
    k_yL[m] = py / gam + aa * (K0_alpha * x - y) / (gam * gam);
    k_pxL[m] = K0_alpha * (px - py) * dd - (bb / gam * t.xCoef + cc) * x;
    k_pyL[m] = K0_alpha * (px + py) * dd - (bb / gam * t.yCoef - cc) * y;
  }
  x_ = x0 + dz / 6.0 * (k_xL[1] + 2 * k_xL[2] + 2 * k_xL[3] + k_xL[4]);
  y_ = y0 + dz / 6.0 * (k_yL[1] + 2 * k_yL[2] + 2 * k_yL[3] + k_yL[4]);
  px_ = px0 + dz / 6.0 * (k_pxL[1] + 2 * k_pxL[2] + 2 * k_pxL[3] + k_pxL[4]);
  py_ = py0 + dz / 6.0 * (k_pyL[1] + 2 * k_pyL[2] + 2 * k_pyL[3] + k_pyL[4]);
}

// Bilinear field gather of particlePush.cpp:306-321 (shared with the drift).
__device__ __forceinline__ double gather_sumU2(const ParticleLaunch& a, int s, int idxI, int idxJ,
                                               const double wx[2], const double wy[2], cd* Ux, cd* Uy) {
  const DevGeom& G = a.G;
  const int nx = G.nx;
  for (int h = 0; h < G.H; ++h) {
    const double2* px_ = a.U + field_plane(G.S, h, 0, s, a.ring_base) * G.N;
    const double2* py_ = a.U + field_plane(G.S, h, 1, s, a.ring_base) * G.N;
    cd ux = C(0, 0), uy = C(0, 0);
#pragma unroll
    for (int ii = 0; ii < 2; ++ii)
#pragma unroll
      for (int jj = 0; jj < 2; ++jj) {
        const int id = (idxJ + jj) * nx + (idxI + ii);
        const double2 vx = __ldg(px_ + id), vy = __ldg(py_ + id);
        ux = cadd(ux, cscale(cscale(C(vx.x, vx.y), wx[ii]), wy[jj]));
        uy = cadd(uy, cscale(cscale(C(vy.x, vy.y), wx[ii]), wy[jj]));
      }
    Ux[h] = ux;
    Uy[h] = uy;
  }
  double sumU2 = 0.0;
  for (int h = 0; h < G.H; ++h) {
    const int H = G.harmony[h];
    sumU2 += (cnorm(Ux[h]) + cnorm(Uy[h])) / (2.0 * H * H);
  }
  return sumU2;
}

// Odd-harmonic / even-harmonic coupling factors fx, fy of the push
// (particlePush.cpp:336-360).
__device__ __forceinline__ void push_f(const ParticleLaunch& a, int H, double xi, double xi2, double K0_alpha,
                                       cd expP, cd expM, cd* fx, cd* fy) {
  const DevGeom& G = a.G;
  double w[2];
  int idx = (1.0 * H * xi) / G.dBessel;
  w[1] = (H * xi / G.dBessel) - idx;
  w[0] = 1.0 - w[1];
  if (H % 2 == 1) {
    const double sign = ((H - 1) / 2 % 2 == 0) ? 1.0 : -1.0;
    int order = (H - 1) / 2;
    const double J1 = BJ(G, idx, order, a.err) * w[0] + BJ(G, idx + 1, order, a.err) * w[1];
    order = (H + 1) / 2;
    const double J2 = BJ(G, idx, order, a.err) * w[0] + BJ(G, idx + 1, order, a.err) * w[1];
    *fx = C(sign * (K0_alpha * J1 - J2), 0.0);
    *fy = C(sign * (K0_alpha * J1 + J2), 0.0);
  } else {
    const double sign = (H / 2 % 2 == 0) ? 1.0 : -1.0;
    idx = (H * xi) / G.dBessel;
    w[1] = (H * xi / G.dBessel) - idx;
    w[0] = 1.0 - w[1];
    int order = (H - 2) / 2;
    const double J1 = BJ(G, idx, order, a.err) * w[0] + BJ(G, idx + 1, order, a.err) * w[1];
    order = H / 2;
    const double J2 = BJ(G, idx, order, a.err) * w[0] + BJ(G, idx + 1, order, a.err) * w[1];
    order = (H + 2) / 2;
    const double J3 = BJ(G, idx, order, a.err) * w[0] + BJ(G, idx + 1, order, a.err) * w[1];
    const double sx = sign * xi2 * H * 0.5;
    *fx = cscale(cadd(cscale(expP, K0_alpha * J1 - J2), cscale(expM, K0_alpha * J2 - J3)), sx);
    *fy = cscale(cadd(cscale(expP, K0_alpha * J1 + J2), cscale(expM, K0_alpha * J2 + J3)), sx);
  }
}

// xi2 and the polarisation phase B of particlePush.cpp:272-279 and
// solveField.cpp:259-266 (identical expressions in both).
__device__ __forceinline__ void pol_terms(double K0, double ue, double K0_alpha, double Phi, double px, double py,
                                          double* xi2, cd* expP) {
  *xi2 = sqrt(2.0) * K0 / (1.0 + K0 * K0 * 0.5 * (1.0 + ue * ue)) *
         sqrt((1 + K0_alpha) * (px * px + ue * ue * py * py) + (1 - K0_alpha) * (px * px * ue * ue + py * py));
  const double B = fm::atan(2.0 * K0_alpha * ue * (px - py) /
                            ((1.0 + K0_alpha) * (px + ue * ue * py) + (1 - K0_alpha) * (px * ue * ue + py)));
  const double ph = B - Phi * 0.5;
  if (ph - ph == 0.0) *expP = cexpi(ph);
  else *expP = C(ph - ph, ph - ph);  // nan in, nan out
}

// particlePush.cpp:261-378 for one particle; returns false when the particle
// is outside the push grid (theta, gamma untouched).
__device__ __forceinline__ void push_one(const ParticleLaunch& a, int s, double wakeE, double x0, double y0,
                                         double px, double py, double& th_, double& ga_) {
  const DevGeom& G = a.G;
  const PushCoef& c = a.pc;
  const int nx = G.nx, ny = G.ny, nr = G.nr, L = G.L, F = G.F;
  const double dz = c.dz, ku = c.ku, ks = c.ks, K0 = c.K0, ue = c.ue, K0_alpha = c.K0_alpha;
  const double coefList[5] = {0, 0, 0.5, 0.5, 1};
  const int sliceI = s + 1;
  const double r2 = x0 * x0 + y0 * y0;
  const double pr2 = px * px + py * py;
  const double th0 = th_, gam0 = ga_;
  const double K2 = 1.0 + pr2 + (1.0 + ue * ue) * K0 * K0 * 0.5 * (1.0 + ku * ku * 0.5 * r2);
  const double xi = ks / ku * K0 * K0 / (8.0 * gam0 * gam0) * (1.0 - ue * ue);
  const int idxI = (int)((x0 - G.minX) / G.dx);
  const int idxJ = (int)((y0 - G.minY) / G.dy);
  double wx[2], wy[2], wr[2];
  wx[1] = (x0 - G.minX) / G.dx - idxI;
  wx[0] = 1.0 - wx[1];
  wy[1] = (y0 - G.minY) / G.dy - idxJ;
  wy[0] = 1.0 - wy[1];
  if (!(idxI >= 0 && idxI < nx - 1 && idxJ >= 0 && idxJ < ny - 1)) return;
  double xi2;
  cd expP;
  bool has_even = false;
  for (int h = 0; h < G.H; ++h) has_even |= (G.harmony[h] % 2 == 0);
  if (has_even) pol_terms(K0, ue, K0_alpha, c.Phi, px, py, &xi2, &expP);
  else { xi2 = 0.0; expP = C(1.0, 0.0); }
  const cd expM = cconj(expP);
  const double r = sqrt(r2);
  const int idxR = r / G.dr + 0.5;
  wr[1] = (r * r / (G.dr * G.dr) - idxR * idxR) / (2.0 * idxR);
  wr[0] = 1.0 - wr[1];
  cd Em[4];
  const double2* Ez = a.Ez;
  const size_t ezs = (size_t)(G.S + 2) * nr * F;
  if (idxR > 0 && idxR < nr) {
    for (int ll = 0; ll < L; ++ll) {
      cd e = C(0, 0);
      for (int f = 0; f < F; ++f)
        for (int jj = 0; jj < 2; ++jj) {
          const double2 v = Ez[ll * ezs + (size_t)sliceI * nr * F + nr * f + idxR + jj];
          e = cadd(e, cscale(C(v.x, v.y), wr[jj]));
        }
      Em[ll] = e;
    }
  } else if (idxR == 0) {
    for (int ll = 0; ll < L; ++ll) {
      cd e = C(0, 0);
      for (int f = 0; f < F; ++f)
        for (int jj = 0; jj < 2; ++jj) {
          const double2 v = Ez[ll * ezs + (size_t)sliceI * nr * F + nr * f + idxR + jj];
          e = cadd(e, C(v.x, v.y));
        }
      Em[ll] = e;
    }
  } else {
    // The reference reuses the previous particle's Em here (carry-over across
    // particles); that sequential dependence is not reproduced: flag it.
    set_flag(a.err, ERR_RADIAL);
    for (int ll = 0; ll < L; ++ll) Em[ll] = C(0, 0);
  }
  cd Ux[FELIS_MAX_HARMONY], Uy[FELIS_MAX_HARMONY];
  const double sumU2 = gather_sumU2(a, s, idxI, idxJ, wx, wy, Ux, Uy);
  double k_th[5] = {0, 0, 0, 0, 0}, k_gam[5] = {0, 0, 0, 0, 0};
  const double sq = sqrt(ue * ue + 1.0);
  for (int m = 1; m < 5; ++m) {
    const double th = th0 + dz * k_th[m - 1] * coefList[m];
    const double gam = gam0 + dz * k_gam[m - 1] * coefList[m];
    double sumTh = 0.0, sumG = 0.0, sumEzPart = 0.0;
    for (int ll = 0; ll < L; ++ll) {
      const cd e = cexpi((ll + 1.0) * th);
      sumEzPart += 2.0 * (Em[ll].re * e.re - Em[ll].im * e.im);
    }
    for (int h = 0; h < G.H; ++h) {
      const int H = G.harmony[h];
      cd fx, fy;
      push_f(a, H, xi, xi2, K0_alpha, expP, expM, &fx, &fy);
      const cd e = cexpi((1.0 * H) * (th + c.Phi * 0.5));
      const cd tmpComp = cmul(e, csub(cmul(cmul(c.etaX, fx), Ux[h]), cmul(cmul(c.etaY, fy), Uy[h])));
      sumTh += (0.0 * tmpComp.re - 1.0 * tmpComp.im) / (1.0 * H);
      sumG += tmpComp.re / (2.0 * gam);
    }
    k_th[m] = ku - ks / (2.0 * gam * gam) * (K2 + sumU2 + K0 * sq * sumTh);
    k_gam[m] = ks * K0 * sq * sumG + c.e_mc2 * sumEzPart;
  }
  const double tmpTh = dz / 6.0 * (k_th[1] + 2.0 * k_th[2] + 2.0 * k_th[3] + k_th[4]);
  if (tmpTh > c.dPhi || tmpTh < -c.dPhi) set_flag(a.err, ERR_THETA_OVERFLOW);
  th_ = th0 + tmpTh;
  const double tmpGam = dz / 6.0 * (k_gam[1] + 2.0 * k_gam[2] + 2.0 * k_gam[3] + k_gam[4]) - dz * wakeE;
  ga_ = gam0 + tmpGam;
}

// particlePush.cpp:150-184 for one particle.
__device__ __forceinline__ void drift_one(const ParticleLaunch& a, int s, double wakeE, double x0, double y0,
                                          double px, double py, double& th_) {
  const DevGeom& G = a.G;
  const PushCoef& c = a.pc;
  const double pr2 = px * px + py * py;
  const double K2 = 1.0 + pr2;
  const int idxI = (int)((x0 - G.minX) / G.dx);
  const int idxJ = (int)((y0 - G.minY) / G.dy);
  double wx[2], wy[2];
  wx[1] = (x0 - G.minX) / G.dx - idxI;
  wx[0] = 1.0 - wx[1];
  wy[1] = (y0 - G.minY) / G.dy - idxJ;
  wy[0] = 1.0 - wy[1];
  if (!(idxI >= 0 && idxI < G.nx - 1 && idxJ >= 0 && idxJ < G.ny - 1)) return;
  cd Ux[FELIS_MAX_HARMONY], Uy[FELIS_MAX_HARMONY];
  const double sumU2 = gather_sumU2(a, s, idxI, idxJ, wx, wy, Ux, Uy);
  const double tmp = c.ku - c.ks / (2.0 * c.gamR * c.gamR) * (K2 + sumU2);
  double th = th_;
  th += tmp * c.dz;
  th -= c.dz * wakeE;
  th_ = th;
}

// rearrangeParticles.cpp:301-320 for one particle.
__device__ __forceinline__ void wrap_one(double dTh, double& theta_, int* err) {
  double delTh = 0.0;
  const double theta = theta_;
  int intTh = 0;
  if (theta >= dTh) {
    intTh = theta / dTh;
    delTh = dTh * intTh;
  } else if (theta < 0) {
    intTh = theta / dTh - 1.0;
    delTh = dTh * intTh;
  }
  theta_ = theta - delTh;
  if (theta_ > dTh || theta_ < 0) set_flag(err, ERR_OUT_OF_RANGE);
}

// solveField.cpp:252-301 and 331-357: per-particle deposit records.
__device__ __forceinline__ void prep_one(const ParticleLaunch& a, int64_t n, double macro, double x, double y,
                                         double px, double py, double theta, double gam) {
  const DevGeom& G = a.G;
  const PrepCoef& c = a.prep;
  const DevDeposit& D = a.dep;
  const int nx = G.nx, ny = G.ny, nr = G.nr, L = G.L, F = G.F;
  const size_t tot = (size_t)a.P.total;
  bool has_even = false;
  for (int h = 0; h < G.H; ++h) has_even |= (G.harmony[h] % 2 == 0);
  double xi2 = 0.0;
  cd expP = C(1.0, 0.0);
  if (has_even) pol_terms(c.K0, c.ue, c.K0_alpha, c.Phi, px, py, &xi2, &expP);
  const cd expM = cconj(expP);
  const int idxI = (x - G.minX) / G.dx;
  const int idxJ = (y - G.minY) / G.dy;
  D.wx1[n] = (x - G.minX) / G.dx - idxI;
  D.wy1[n] = (y - G.minY) / G.dy - idxJ;
  const bool in = idxI >= 0 && idxI < nx && idxJ >= 0 && idxJ < ny;
  D.key[n] = in ? idxJ * nx + idxI : -1;
  if (in && (idxI == nx - 1 || idxJ == ny - 1)) atomicAdd(a.err + ERR_EDGE_DEPOSIT, 1);
  if (in) {
    for (int h = 0; h < G.H; ++h) {
      const int H = G.harmony[h];
      const double dbH = (double)H;
      if (H % 2 == 0) {
        double w[2];
        const double sign = (H / 2 % 2 == 0) ? 1.0 : -1.0;
        const int ib = (dbH * c.xi) / G.dBessel;
        w[1] = (dbH * c.xi / G.dBessel) - ib;
        w[0] = 1.0 - w[1];
        int order = (H - 2) / 2;
        const double J1 = BJ(G, ib, order, a.err) * w[0] + BJ(G, ib + 1, order, a.err) * w[1];
        order = H / 2;
        const double J2 = BJ(G, ib, order, a.err) * w[0] + BJ(G, ib + 1, order, a.err) * w[1];
        order = (H + 2) / 2;
        const double J3 = BJ(G, ib, order, a.err) * w[0] + BJ(G, ib + 1, order, a.err) * w[1];
        const double sx = sign * xi2 * dbH * 0.5;
        const cd fx = cscale(cadd(cscale(expM, J1 - c.K0_alpha * J2), cscale(expP, J2 - c.K0_alpha * J3)), sx);
        const cd fy = cscale(cadd(cscale(expM, J1 + c.K0_alpha * J2), cscale(expP, J2 + c.K0_alpha * J3)), sx);
        D.fx[(size_t)h * tot + n] = make_double2(fx.re, fx.im);
        D.fy[(size_t)h * tot + n] = make_double2(fy.re, fy.im);
      }
      const cd e = cexpi((-1.0 * dbH) * (theta + c.Phi * 0.5));
      const cd mc = cdivr(cscale(e, dbH * macro * c.coef_U), gam);
      D.coef[(size_t)h * tot + n] = make_double2(mc.re, mc.im);
    }
  }
  // Ez source (solveField.cpp:331-357): every particle, no grid test.
  const double phi = (F > 1) ? ((x == 0.0) ? 0.0 : fm::atan2(y, x)) : 0.0;
  const double r = sqrt(x * x + y * y);
  const int idxR = r / G.dr + 0.5;
  D.wr1[n] = (r * r / (G.dr * G.dr) - idxR * idxR) / (2.0 * idxR);
  int rk = -1;
  if (idxR > 0 && idxR < nr) {
    rk = idxR;
    if (idxR == nr - 1 && F > 1) set_flag(a.err, ERR_RADIAL);
    for (int l = 0; l < L; ++l)
      for (int f = 0; f < F; ++f) {
        const cd e = cexpi(-1.0 * ((l + 1) * theta + f * phi));
        const cd ic = C(0.0 * c.coef_Ez * (l + 1.0), 1.0 * c.coef_Ez * (l + 1.0));
        const cd cc = cdivr(cscale(cmul(ic, e), macro), 1.0 * idxR);
        D.ez[(size_t)(l * F + f) * tot + n] = make_double2(cc.re, cc.im);
      }
  } else if (idxR == 0) {
    rk = 0;
    for (int l = 0; l < L; ++l) {
      const cd e = cexpi(-1.0 * ((l + 1) * theta));
      const cd ic = C(0.0 * c.coef_Ez * (l + 1.0), 1.0 * c.coef_Ez * (l + 1.0));
      const cd cc = cscale(cmul(ic, e), macro);
      D.ez[(size_t)(l * F + 0) * tot + n] = make_double2(cc.re, cc.im);
    }
  }
  D.rkey[n] = rk;
}

// Deterministic block sum of `v` (fixed shuffle tree, then warps in order).
__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
  return t;
}

__global__ void __launch_bounds__(256) k_particles(ParticleLaunch a) {
  __shared__ double red[8];
  const DevGeom& G = a.G;
  const int4 tile = a.P.tiles[blockIdx.x];
  const int sp = tile.x, s = tile.y;
  const int64_t n = (int64_t)tile.z + threadIdx.x;
  const bool active = n < (int64_t)tile.w;
  const unsigned ops = a.ops;
  const int sliceI = s + 1;
  double wakeE = 0.0;
  if (G.wakeOn) wakeE = G.wakeE[sliceI - 1 + G.minI] / (K_MC2 * 1.0e6);
  const double macro = a.P.weight[(size_t)sp * G.S + s];
  double x = 0, y = 0, px = 0, py = 0, th = 0, ga = 1;
  if (active) {
    x = a.P.x[n]; y = a.P.y[n]; px = a.P.px[n]; py = a.P.py[n]; th = a.P.th[n]; ga = a.P.ga[n];
    if (ops & OP_T0) transverse_one(a.t0, x, y, px, py, ga);
    if (ops & OP_T1) transverse_one(a.t1, x, y, px, py, ga);
    if (ops & OP_PUSH) push_one(a, s, wakeE, x, y, px, py, th, ga);
    else if (ops & OP_DRIFT) drift_one(a, s, wakeE, x, y, px, py, th);
    if (ops & OP_PHASE) th += a.theta_shift;
    if (ops & OP_WRAP) wrap_one(G.numSlice * 2 * M_PI, th, a.err);
    if (ops & (OP_T0 | OP_T1)) {
      a.P.x[n] = x; a.P.y[n] = y; a.P.px[n] = px; a.P.py[n] = py;
    }
    if (ops & (OP_PUSH | OP_DRIFT | OP_PHASE | OP_WRAP)) a.P.th[n] = th;
    if (ops & OP_PUSH) a.P.ga[n] = ga;
    if (!(x - x == 0.0) || !(y - y == 0.0) || !(th - th == 0.0) || !(ga - ga == 0.0)) set_flag(a.err, ERR_NAN);
    if (ops & OP_PREP) prep_one(a, n, macro, x, y, px, py, th, ga);
  }
  if (ops & OP_DIAG) {
    // twiss.cpp:146-166 and saveFile.cpp:126-137 partial sums of this tile.
    double* out = a.diag + (size_t)blockIdx.x * a.diag_stride;
    const double invGam = 1.0 / ga;
    const double xP = px * invGam, yP = py * invGam;
    const double on = active ? 1.0 : 0.0;
    const double v[7] = {x * x * on, y * y * on, xP * xP * on, yP * yP * on, x * xP * on, y * yP * on, on};
    for (int k = 0; k < 7; ++k) {
      const double t = block_sum(v[k], red);
      if (threadIdx.x == 0) out[k] = t;
    }
    for (int h = 0; h < G.H; ++h) {
      double sv, cv;
      sincos((double)G.harmony[h] * th, &sv, &cv);
      const double tr = block_sum(cv * macro * on, red);
      const double ti = block_sum(sv * macro * on, red);
      if (threadIdx.x == 0) { out[7 + 2 * h] = tr; out[8 + 2 * h] = ti; }
    }
    const double tw = block_sum(macro * on, red);
    if (threadIdx.x == 0) out[7 + 2 * G.H] = tw;
  }
}

// Level 1: block b sums tiles [b*per, (b+1)*per) of every quantity in a
// fixed order: 7 twiss sums per species, then the 2H+1 bFactor sums.
__global__ void __launch_bounds__(256) k_diag_level1(const double* part, int ntiles, int stride, int nspecies,
                                                     int H, const int4* tiles, int per, double* out) {
  __shared__ double red[8];
  const int t0 = blockIdx.x * per, t1 = min(ntiles, t0 + per);
  const int nq = 7 * nspecies + 2 * H + 1;
  double* o = out + (size_t)blockIdx.x * nq;
  for (int sp = 0; sp < nspecies; ++sp)
    for (int k = 0; k < 7; ++k) {
      double v = 0.0;
      for (int t = t0 + threadIdx.x; t < t1; t += blockDim.x)
        if (tiles[t].x == sp) v += part[(size_t)t * stride + k];
      const double r = block_sum(v, red);
      if (threadIdx.x == 0) o[7 * sp + k] = r;
    }
  for (int k = 0; k < 2 * H + 1; ++k) {
    double v = 0.0;
    for (int t = t0 + threadIdx.x; t < t1; t += blockDim.x) v += part[(size_t)t * stride + 7 + k];
    const double r = block_sum(v, red);
    if (threadIdx.x == 0) o[7 * nspecies + k] = r;
  }
}

// Level 2: one block adds the level-1 rows in order and finishes
// twiss.cpp:177-192 and saveFile.cpp:166 (b / totalN).
__global__ void __launch_bounds__(256) k_diag_level2(const double* l1, int nblocks, int nspecies, int H,
                                                     double* twiss, double* bf) {
  __shared__ double red[8];
  const int nq = 7 * nspecies + 2 * H + 1;
  __shared__ double tot[7 * FELIS_MAX_SPECIES + 2 * FELIS_MAX_HARMONY + 1];
  for (int k = 0; k < nq; ++k) {
    double v = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v += l1[(size_t)b * nq + k];
    const double r = block_sum(v, red);
    if (threadIdx.x == 0) tot[k] = r;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int sp = 0; sp < nspecies; ++sp) {
      const double* acc = tot + 7 * sp;
      double* o = twiss + 6 * sp;
      for (int k = 0; k < 6; ++k) o[k] = 0.0;
      const double cnt = acc[6];
      if (cnt > 0.0) {
        const double avgX2 = acc[0] / cnt, avgY2 = acc[1] / cnt;
        const double avgXP = acc[2] / cnt, avgYP = acc[3] / cnt;
        const double avgCX = acc[4] / cnt, avgCY = acc[5] / cnt;
        const double ex = sqrt(avgX2 * avgXP - avgCX * avgCX), ey = sqrt(avgY2 * avgYP - avgCY * avgCY);
        o[0] = ex; o[1] = avgX2 / ex; o[2] = -avgCX / ex;
        o[3] = ey; o[4] = avgY2 / ey; o[5] = -avgCY / ey;
      }
    }
    const double wsum = tot[7 * nspecies + 2 * H];
    for (int k = 0; k < 2 * H; ++k) bf[k] = tot[7 * nspecies + k] / wsum;
  }
}

}  // namespace

void launch_particles(const ParticleLaunch& a, cudaStream_t st) {
  if (a.P.ntiles <= 0) return;
  k_particles<<<a.P.ntiles, 256, 0, st>>>(a);
}

void launch_diag_finalize(const double* partials, int ntiles, int stride, int nspecies, int H, const int4* tiles,
                          double* l1, int l1_blocks, double* out_twiss, double* out_bf, cudaStream_t st) {
  const int per = (ntiles + l1_blocks - 1) / l1_blocks;
  k_diag_level1<<<l1_blocks, 256, 0, st>>>(partials, ntiles, stride, nspecies, H, tiles, per, l1);
  k_diag_level2<<<1, 256, 0, st>>>(l1, l1_blocks, nspecies, H, out_twiss, out_bf);
}

}  // namespace felis
