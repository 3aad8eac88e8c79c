// Beam loader kernel (loadBeam.cpp:28-269, 3D): one thread per beamlet.
//
// The host loader draws the Halton points in beamlet order; point n of the
// sequence only depends on n (radical inverses in the bases 2..17), so every
// beamlet computes its own with the same operations.  The Gaussian noise
// amplitudes come from the host's sequential random stream.  Built without
// FMA contraction so that the Halton sums and the per-particle arithmetic
// take the host's operation order; log, sqrt, sin and cos are CUDA's (within
// an ulp or two of the host C library).
#include "load.cuh"

namespace felis {

namespace {

__device__ void halton7(uint64_t count, double v[7]) {
  const int primes[7] = {2, 3, 5, 7, 11, 13, 17};
  for (int d = 0; d < 7; ++d) {
    const int p = primes[d];
    double f = 1.0 / p, x = 0.0;
    uint64_t c = count;
    while (c > 0) {
      x += f * (double)(c % p);
      c /= p;
      f /= p;
    }
    v[d] = x;
  }
}

__global__ void __launch_bounds__(256) k_load_beam(LoadArgs a) {
  for (int s = blockIdx.x; s < a.S; s += gridDim.x) {
    const LoadSlice L = a.slices[s];
    for (int b = threadIdx.x; b < L.beamlets; b += blockDim.x) {
      const int64_t g = L.first + b;
      double v1[7];
      halton7(a.halton0 + (uint64_t)g + 1, v1);
      const double theta0 = v1[4] * a.dPhi;
      double r1 = v1[0];
      if (r1 == 0.0) r1 = 1e-10;
      const double r2 = v1[1];
      double pr1 = v1[2];
      if (pr1 == 0.0) pr1 = 1e-10;
      const double pr2 = v1[3];
      double gam = v1[5];
      if (gam == 0.0) gam = 1e-10;
      double x, y, xPrime, yPrime;
      double coef = a.trans_flat ? sqrt(r1) : sqrt(-2.0 * log(r1));
      x = coef * cos(2.0 * M_PI * r2) * L.sigX;
      y = coef * sin(2.0 * M_PI * r2) * L.sigY;
      coef = sqrt(-2.0 * log(pr1));
      xPrime = coef * cos(2.0 * M_PI * pr2) * L.sigXPrime;
      yPrime = coef * sin(2.0 * M_PI * pr2) * L.sigYPrime;
      const double tmp = sqrt(-2.0 * log(gam)) * cos(v1[6] * 2.0 * M_PI);
      gam = L.gamma0 + L.dGam * tmp * L.ESn0;
      const double pz = sqrt((gam * gam - 1.0) / (1.0 + xPrime * xPrime + yPrime * yPrime));
      const double px = xPrime * pz, py = yPrime * pz;
      x -= L.delTX * px / gam;
      y -= L.delTY * py / gam;
      const double* nz = a.noise + (size_t)g * 2 * a.maxH;
      for (int n = 0; n < a.num_in_beamlet; ++n) {
        const size_t k = (size_t)g * a.num_in_beamlet + n;
        a.x[k] = x; a.y[k] = y; a.px[k] = px; a.py[k] = py; a.gamma[k] = gam;
        const double theta = theta0 + n * a.div;
        double noise = 0.0;
        for (int m = 1; m <= a.maxH; ++m) noise += nz[2 * (m - 1)] * cos(m * theta) + nz[2 * (m - 1) + 1] * sin(m * theta);
        a.theta[k] = theta + noise * a.noise_on;
      }
    }
  }
}

}  // namespace

cudaError_t launch_load_beam(const LoadArgs& a, cudaStream_t st) {
  if (a.S <= 0) return cudaSuccess;
  const int grid = a.S < 4096 ? a.S : 4096;
  k_load_beam<<<grid, 256, 0, st>>>(a);
  return cudaGetLastError();
}

}  // namespace felis
