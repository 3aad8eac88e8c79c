// Wake function and wake field on the device (wakeField.cpp:9-50, 53-159):
// the kernel side of felis_config_wake_device (host side in host/config.cpp).
#pragma once

#include <cuda_runtime.h>

namespace felis {

// Impedance samples of wakeField.cpp:63-75: numK + 1 wavenumbers, and for the
// flat (parallel-plate) shape the x integral on numX + 1 points.
constexpr int kWakeNumK = 1000;
constexpr int kWakeNumX = 50000;
constexpr double kWakeMaxK = 20.0;
constexpr double kWakeMaxX = 2000.0;

struct WakeArgs {
  int shape;     // 1: flat, 2: circular
  int acdc;      // circular shape: 1 AC, else DC
  int S;         // global slices
  double dZ;     // slice length numSlice * lambda0
  double s0;     // (2 r^2 / (Z0 sigma))^(1/3)
  double ctau;   // conductor relaxation length
  double coef;   // Z0 c / (pi r^2 pi)
  double* impZ;  // [kWakeNumK + 1], device
  double* wakeF; // [S], device
};

// impZ, then wakeF (the wake function per slice distance).
cudaError_t launch_wake_function(const WakeArgs& a, cudaStream_t st);
// wakeE[ii] = sum over i >= ii (from the last slice down) of den[i] wakeF[i - ii] dZ coef.
cudaError_t launch_wake_field(const double* den, const double* wakeF, int S, double dZ, double coef, double* wakeE,
                              cudaStream_t st);

}  // namespace felis
