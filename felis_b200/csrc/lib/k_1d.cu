// 1D model kernels of the FP64 path (see oned.cuh).  Built without FMA
// contraction and with the deterministic sin/cos, so that every expression
// takes the operation order of the CPU restatement and the results are
// bit-identical to it.
#include "oned.cuh"

namespace felis {

namespace {

// Source and space-charge modes of one slice, the slice's particles in
// order (species by species), as the restatement's solve_sc_1d sums them;
// then U += source.
__global__ void __launch_bounds__(128) k_field_1d(OneDLaunch a, int current) {
  const DevGeom& G = a.G;
  const int S = G.S, H_n = G.H, L = G.L;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= S) return;
  cd sx[FELIS_MAX_HARMONY], sy[FELIS_MAX_HARMONY], ez[4];
  for (int h = 0; h < H_n; ++h) { sx[h] = C(0, 0); sy[h] = C(0, 0); }
  for (int l = 0; l < L; ++l) ez[l] = C(0, 0);
  if (current) {
    for (int sp = 0; sp < a.ns; ++sp) {
      const double macro = a.weight[(size_t)sp * S + s], coef = a.coefU[sp];
      for (int64_t n = a.soff[(size_t)sp * (S + 1) + s]; n < a.soff[(size_t)sp * (S + 1) + s + 1]; ++n) {
        const double th = a.th[n], gam = a.ga[n];
        for (int h = 0; h < H_n; ++h) {
          const double H = (double)G.harmony[h];
          const cd m = cdivr(cscale(cexpi((-1.0 * H) * (th + a.Phi * 0.5)), macro * coef), gam);
          sx[h] = csub(sx[h], cmul(cmul(a.etaX, a.fsrc[h][0]), m));
          sy[h] = csub(sy[h], cmul(cmul(a.etaY, a.fsrc[h][1]), m));
        }
      }
    }
    for (int sp = 0; sp < a.ns; ++sp) {
      const double macro = a.weight[(size_t)sp * S + s], coef = a.coefE[sp];
      for (int64_t n = a.soff[(size_t)sp * (S + 1) + s]; n < a.soff[(size_t)sp * (S + 1) + s + 1]; ++n) {
        const double th = a.th[n];
        for (int l = 0; l < L; ++l) {
          cd t = C(-0.0, -1.0);  // -1.0*I*coef/(1.0+l)*macro*exp(-I*(l+1.0)*th), left to right
          t = cscale(t, coef);
          t = cdivr(t, 1.0 + l);
          t = cscale(t, macro);
          t = cmul(t, cexpi(-((l + 1.0) * th)));
          ez[l] = cadd(ez[l], t);
        }
      }
    }
    for (int l = 0; l < L; ++l) {
      double2* E = a.Ez + (size_t)l * (S + 2);
      E[s + 1] = make_double2(ez[l].re, ez[l].im);
      if (s == 0) E[0] = make_double2(0.0, 0.0);
      if (s == S - 1) E[S + 1] = make_double2(0.0, 0.0);
    }
  }
  for (int h = 0; h < H_n; ++h)
    for (int pol = 0; pol < 2; ++pol) {
      const cd sc = pol ? sy[h] : sx[h];
      a.Sc[((size_t)h * 2 + pol) * S + s] = make_double2(sc.re, sc.im);
      double2* u = a.U + field_plane(S, h, pol, s, a.ring_base);
      const cd v = cadd(C(u->x, u->y), sc);
      *u = make_double2(v.re, v.im);
    }
}

__global__ void __launch_bounds__(256) k_push_1d(OneDLaunch a) {
  const DevGeom& G = a.G;
  const int S = G.S, H_n = G.H, L = G.L;
  const int s = blockIdx.x;
  const double coefList[5] = {0, 0, 0.5, 0.5, 1};
  const double wakeE = G.wakeOn ? G.wakeE[s + G.minI] / (K_MC2 * 1.0e6) : 0.0;
  cd Em[4], Ux[FELIS_MAX_HARMONY], Uy[FELIS_MAX_HARMONY];
  for (int ll = 0; ll < L; ++ll) {
    const double2 e = a.Ez[(size_t)ll * (S + 2) + s + 1];
    Em[ll] = C(e.x, e.y);
  }
  double sumU2 = 0.0;
  for (int h = 0; h < H_n; ++h) {
    const double2 ux = a.U[field_plane(S, h, 0, s, a.ring_base)], uy = a.U[field_plane(S, h, 1, s, a.ring_base)];
    Ux[h] = C(ux.x, ux.y);
    Uy[h] = C(uy.x, uy.y);
    const int H = G.harmony[h];
    sumU2 += (cnorm(Ux[h]) + cnorm(Uy[h])) / (2.0 * H * H);
  }
  int overflow = 0;
  for (int sp = 0; sp < a.ns; ++sp) {
    const int64_t n0 = a.soff[(size_t)sp * (S + 1) + s], n1 = a.soff[(size_t)sp * (S + 1) + s + 1];
    for (int64_t n = n0 + threadIdx.x; n < n1; n += blockDim.x) {
      const double th0 = a.th[n], gam0 = a.ga[n];
      double k_th[5] = {0, 0, 0, 0, 0}, k_gam[5] = {0, 0, 0, 0, 0};
      for (int m = 1; m < 5; ++m) {
        const double th = th0 + a.dz * k_th[m - 1] * coefList[m];
        const double gam = gam0 + a.dz * k_gam[m - 1] * coefList[m];
        double sumTh = 0.0, sumG = 0.0, sumEzPart = 0.0;
        for (int ll = 0; ll < L; ++ll) {
          const cd e = cexpi((ll + 1.0) * th);
          sumEzPart += 2.0 * (Em[ll].re * e.re - Em[ll].im * e.im);
        }
        for (int h = 0; h < H_n; ++h) {
          const double H = (double)G.harmony[h];
          const cd e = cexpi((1.0 * H) * (th + a.Phi * 0.5));
          const cd tmpComp = cmul(e, csub(cmul(cmul(a.etaX, a.fpush[h][0]), Ux[h]), cmul(cmul(a.etaY, a.fpush[h][1]), Uy[h])));
          sumTh += (0.0 * tmpComp.re - 1.0 * tmpComp.im) / (1.0 * H);
          sumG += tmpComp.re / (2.0 * gam);
        }
        k_th[m] = a.ku - G.ks / (2.0 * gam * gam) * (a.K2 + sumU2 + a.K0 * a.sq * sumTh);
        k_gam[m] = G.ks * a.K0 * a.sq * sumG + a.e_mc2 * sumEzPart;
      }
      const double tmpTh = a.dz / 6.0 * (k_th[1] + 2.0 * k_th[2] + 2.0 * k_th[3] + k_th[4]);
      if (tmpTh > a.dPhi || tmpTh <= -a.dPhi) overflow = 1;
      a.th[n] = th0 + tmpTh;
      const double tmpGam = a.dz / 6.0 * (k_gam[1] + 2 * k_gam[2] + 2 * k_gam[3] + k_gam[4]) - a.dz * wakeE;
      a.ga[n] = gam0 + tmpGam;
    }
  }
  if (overflow) set_flag(a.err, ERR_THETA_OVERFLOW);
}

}  // namespace

cudaError_t launch_1d_field(const OneDLaunch& a, int current, cudaStream_t st) {
  const int S = a.G.S;
  k_field_1d<<<(S + 127) / 128, 128, 0, st>>>(a, current);
  return cudaGetLastError();
}

cudaError_t launch_1d_push(const OneDLaunch& a, cudaStream_t st) {
  k_push_1d<<<a.G.S, 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace felis
