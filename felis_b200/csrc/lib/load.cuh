// Initial-state loader on the device (loadBeam.cpp:28-269, 3D): the kernel
// side of felis_config_load_beam_device (host side in host/config.cpp).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace felis {

// Per-slice quantities the host computes (SliceLoad in config.cpp) and the
// slice's first beamlet in the global beamlet order.
struct LoadSlice {
  double gamma0, dGam, sigX, sigY, sigXPrime, sigYPrime, delTX, delTY, ESn0;
  int64_t first;
  int beamlets, pad;
};

struct LoadArgs {
  const LoadSlice* slices;  // [S]
  const double* noise;      // [beamlets][maxH][2]: a_m, b_m of each beamlet (host random stream)
  int S, maxH, num_in_beamlet, trans_flat;
  double noise_on, dPhi, div;
  uint64_t halton0;         // Halton points consumed before the first beamlet (the rank's skip)
  double *x, *y, *px, *py, *theta, *gamma;  // device, beamlet-major
};

cudaError_t launch_load_beam(const LoadArgs& a, cudaStream_t st);

}  // namespace felis
