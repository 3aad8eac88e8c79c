// Wake function and wake field on the device (see wake.cuh).  Built without
// FMA contraction, so that the per-slice sums take the operation order of
// wakeField.cpp term by term.  The impedance integral is a block reduction
// (a fixed tree, so deterministic, but not the serial order of the
// reference), and CUDA's cos, cosh and sinh round differently from the host
// library's by an ulp or so: the wake function agrees with the host's to
// about 1e-13 relative, not bit for bit.  The wake field (the convolution with
// the slice density) sums in the reference's order and is bit-identical to
// the host's given the same wake function.
#include "wake.cuh"

namespace felis {

namespace {

struct zc {
  double re, im;
};
__device__ __forceinline__ zc zmul(zc a, zc b) { return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; }
__device__ __forceinline__ zc zdiv(zc a, zc b) {
  // Smith's algorithm (scaled by the larger component of b)
  if (fabs(b.re) >= fabs(b.im)) {
    const double r = b.im / b.re, d = b.re + b.im * r;
    return {(a.re + a.im * r) / d, (a.im - a.re * r) / d};
  }
  const double r = b.re / b.im, d = b.re * r + b.im;
  return {(a.re * r + a.im) / d, (a.im * r - a.re) / d};
}
// principal square root: t = sqrt((|z| + |re|) / 2) on the larger part
__device__ __forceinline__ zc zsqrt(zc z) {
  if (z.re == 0.0 && z.im == 0.0) return {0.0, z.im};
  const double t = sqrt((hypot(z.re, z.im) + fabs(z.re)) * 0.5);
  if (z.re >= 0.0) return {t, z.im / (2.0 * t)};
  return {fabs(z.im) / (2.0 * t), copysign(t, z.im)};
}

// Flat shape (wakeField.cpp:80-103): impZ[i] = Re sum_j ccal(k_i, x_j) dX,
// one block per wavenumber i = 1..numK; the terms beyond x = 320 are zero.
__global__ void __launch_bounds__(256) k_wake_imp_flat(WakeArgs a) {
  __shared__ double red[256];
  const int i = blockIdx.x + 1;
  const double dK = kWakeMaxK / (kWakeNumK * 1.0), dX = kWakeMaxX / (kWakeNumX * 1.0);
  const double k = 0.0 + i * dK;
  const double sk = sqrt(k);
  // 2 / (1 - i) / sqrt(k - i k^2 ctau / s0), constant along x
  const zc A = zdiv(zdiv({2.0, 0.0}, {1.0, -1.0}), zsqrt({k, -(k * k * a.ctau / a.s0)}));
  double sum = 0.0;
  for (int j = threadIdx.x; j <= kWakeNumX; j += blockDim.x) {
    const double x = 0.0 + j * dX;
    double re;
    if (x == 0.0) {
      re = sk / (2.0 + k * k * k - 2.0 * sk * k);
    } else if (x > 320) {
      break;  // x grows with j: every later term of this thread is zero too
    } else {
      const double ch = cosh(x), sh = sinh(x);
      const zc cd = {A.re * ch, A.im * ch - k * sh / x};
      re = zdiv({1.0 / ch, 0.0}, cd).re;
    }
    sum += re * dX;
  }
  red[threadIdx.x] = sum;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) a.impZ[i] = red[0];
  if (i == 1 && threadIdx.x == 0) a.impZ[0] = 0.0;
}

// Circular shape (wakeField.cpp:104-116), one thread per wavenumber.
__global__ void k_wake_imp_circ(WakeArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i > kWakeNumK) return;
  if (i == 0) { a.impZ[0] = 0.0; return; }
  const double dK = kWakeMaxK / (kWakeNumK * 1.0);
  const double k = 0.0 + i * dK;
  if (a.acdc == 1) {
    // sqrt(2 s0 / ctau) / k (i + s0 0.5 / k / ctau) - i 0.5 k
    const double m = sqrt(2.0 * a.s0 / a.ctau) / k;
    const zc cd = {m * (a.s0 * 0.5 / k / a.ctau), m * 1.0 - 0.5 * k};
    a.impZ[i] = zdiv({1.0, 0.0}, cd).re;
  } else {
    const double dino = 2.0 / k + 0.25 * k * k - sqrt(k);
    a.impZ[i] = 1.0 / sqrt(k) / dino;
  }
}

// wakeField.cpp:128-140: wakeF[i] = coef sum_j impZ[j] cos(k_j z_i) dK, j in order.
__global__ void k_wake_fn(WakeArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.S) return;
  const double dK = kWakeMaxK / (kWakeNumK * 1.0);
  const double z = (i * a.dZ) / a.s0;
  double sum = 0.0;
  for (int j = 0; j <= kWakeNumK; ++j) {
    const double k = 0.0 + (double)j * dK;
    sum += a.impZ[j] * cos(k * z) * dK;
  }
  a.wakeF[i] = 0.0 + sum * a.coef;
}

// wakeField.cpp:30-35: for a fixed ii the reference adds the terms of
// i = S-1, S-2, ..., ii in that order.
__global__ void k_wake_field(const double* __restrict__ den, const double* __restrict__ wakeF, int S, double dZ,
                             double coef, double* __restrict__ wakeE) {
  const int ii = blockIdx.x * blockDim.x + threadIdx.x;
  if (ii >= S) return;
  double w = 0.0;
  for (int i = S - 1; i >= ii; --i) w += den[i] * wakeF[i - ii] * dZ * coef;
  wakeE[ii] = w;
}

}  // namespace

cudaError_t launch_wake_function(const WakeArgs& a, cudaStream_t st) {
  if (a.shape == 1) {
    k_wake_imp_flat<<<kWakeNumK, 256, 0, st>>>(a);
  } else if (a.shape == 2) {
    k_wake_imp_circ<<<(kWakeNumK + 1 + 127) / 128, 128, 0, st>>>(a);
  } else {
    cudaError_t e = cudaMemsetAsync(a.impZ, 0, (kWakeNumK + 1) * sizeof(double), st);
    if (e != cudaSuccess) return e;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (a.S > 0) k_wake_fn<<<(a.S + 127) / 128, 128, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_wake_field(const double* den, const double* wakeF, int S, double dZ, double coef, double* wakeE,
                              cudaStream_t st) {
  if (S > 0) k_wake_field<<<(S + 127) / 128, 128, 0, st>>>(den, wakeF, S, dZ, coef, wakeE);
  return cudaGetLastError();
}

}  // namespace felis
