// Stable integer key sort of particles by slice.
//
// The reference never moves particles between slices in its live loop
// (rearrangeParticles.cpp:7-75 is commented out); slice order matters when
// particles are binned on restart (restoreParticleHDF.cpp:166-214 keeps file
// order inside a slice) and when they are written slice-major
// (saveParticleHDF.cpp:95-109).  This sort reproduces that binning: the
// output permutation equals a stable CPU sort of the slice keys.
//
// LSD radix sort, 8-bit digits, 4096-element tiles:
//   1. per-tile digit histogram (shared-memory int atomics; counts only)
//   2. exclusive scan of the histogram in digit-major order (one block)
//   3. per tile: bitonic sort of (digit << 12 | local index) in shared
//      memory, which orders the tile stably by digit; each element's
//      destination is its digit's scanned offset for this tile plus its rank
//      inside the tile's run of that digit.
// Memory traffic per pass: read key + value, write key + value (16 B per
// element) plus the histograms; the tile sort stays in shared memory.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>

#include <cuda.h>
#include <mutex>
#include <vector>

#include "../../../include/felis_b200.h"

namespace {

constexpr int kTile = 4096;
constexpr int kThreads = 512;

__global__ void __launch_bounds__(kThreads) k_hist(const int32_t* keys, int64_t n, int shift, int ntiles,
                                                   uint32_t* hist) {
  __shared__ uint32_t h[256];
  for (int d = threadIdx.x; d < 256; d += blockDim.x) h[d] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kTile;
  for (int i = threadIdx.x; i < kTile; i += blockDim.x) {
    const int64_t e = base + i;
    if (e < n) atomicAdd(&h[((uint32_t)keys[e] >> shift) & 255u], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += blockDim.x) hist[(size_t)d * ntiles + blockIdx.x] = h[d];
}

// Exclusive scan of m entries in place, one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_scan(uint32_t* a, int64_t m) {
  __shared__ uint64_t part[1024];
  const int64_t per = (m + blockDim.x - 1) / blockDim.x;
  const int64_t b = per * threadIdx.x, e = b + per < m ? b + per : m;
  uint64_t s = 0;
  for (int64_t i = b; i < e; ++i) s += a[i];
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint64_t run = 0;
    for (int t = 0; t < (int)blockDim.x; ++t) {
      const uint64_t v = part[t];
      part[t] = run;
      run += v;
    }
  }
  __syncthreads();
  uint64_t run = part[threadIdx.x];
  for (int64_t i = b; i < e; ++i) {
    const uint32_t v = a[i];
    a[i] = (uint32_t)run;
    run += v;
  }
}

__global__ void __launch_bounds__(kThreads) k_scatter(const int32_t* kin, const int64_t* vin, int64_t n, int shift,
                                                      int ntiles, const uint32_t* offs, int32_t* kout, int64_t* vout) {
  __shared__ uint32_t s[kTile];
  const int64_t base = (int64_t)blockIdx.x * kTile;
  for (int i = threadIdx.x; i < kTile; i += blockDim.x) {
    const int64_t e = base + i;
    s[i] = e < n ? ((((uint32_t)kin[e] >> shift) & 255u) << 12) | (uint32_t)i : 0xFFFFFFFFu;
  }
  __syncthreads();
  for (int k = 2; k <= kTile; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < kTile; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const uint32_t a = s[i], b = s[ixj];
          const bool up = (i & k) == 0;
          if ((a > b) == up) { s[i] = b; s[ixj] = a; }
        }
      }
      __syncthreads();
    }
  for (int q = threadIdx.x; q < kTile; q += blockDim.x) {
    const uint32_t c = s[q];
    if (c == 0xFFFFFFFFu) continue;
    const uint32_t d = c >> 12;
    // first position of digit d in the sorted tile
    int lo = 0, hi = q;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if ((s[mid] >> 12) < d) lo = mid + 1;
      else hi = mid;
    }
    const int64_t e = base + (c & 4095u);
    const uint64_t dst = (uint64_t)offs[(size_t)d * ntiles + blockIdx.x] + (uint64_t)(q - lo);
    kout[dst] = kin[e];
    vout[dst] = vin[e];
  }
}

__global__ void k_iota(int64_t* v, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) v[i] = i;
}

}  // namespace

extern "C" felis_status felis_sort_by_slice(const int32_t* keys, int64_t n, int64_t* perm) {
  if (n < 0 || (n > 0 && (!keys || !perm))) return FELIS_BAD_ARG;
  if (n == 0) return FELIS_OK;
  if (n > ((int64_t)1 << 32)) return FELIS_UNSUPPORTED;
  int32_t kmax = 0;
  for (int64_t i = 0; i < n; ++i) {
    if (keys[i] < 0 || keys[i] >= (1 << 30)) return FELIS_BAD_ARG;
    if (keys[i] > kmax) kmax = keys[i];
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FELIS_NO_DEVICE;
  int bits = 0;
  while (bits < 31 && (kmax >> bits) != 0) ++bits;
  const int passes = bits == 0 ? 1 : (bits + 7) / 8;
  const int ntiles = (int)((n + kTile - 1) / kTile);
  int32_t *k0 = nullptr, *k1 = nullptr;
  int64_t *v0 = nullptr, *v1 = nullptr;
  uint32_t* hist = nullptr;
  cudaStream_t st = nullptr;
  felis_status rc = FELIS_OK;
  cudaError_t e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&k0, n * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc(&k1, n * sizeof(int32_t));
  if (e == cudaSuccess) e = cudaMalloc(&v0, n * sizeof(int64_t));
  if (e == cudaSuccess) e = cudaMalloc(&v1, n * sizeof(int64_t));
  if (e == cudaSuccess) e = cudaMalloc(&hist, (size_t)256 * ntiles * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemcpyAsync(k0, keys, n * sizeof(int32_t), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    k_iota<<<1184, 256, 0, st>>>(v0, n);
    for (int p = 0; p < passes; ++p) {
      k_hist<<<ntiles, kThreads, 0, st>>>(k0, n, 8 * p, ntiles, hist);
      k_scan<<<1, 1024, 0, st>>>(hist, (int64_t)256 * ntiles);
      k_scatter<<<ntiles, kThreads, 0, st>>>(k0, v0, n, 8 * p, ntiles, hist, k1, v1);
      int32_t* tk = k0; k0 = k1; k1 = tk;
      int64_t* tv = v0; v0 = v1; v1 = tv;
    }
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpyAsync(perm, v0, n * sizeof(int64_t), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) rc = FELIS_CUDA_ERROR;
  if (k0) cudaFree(k0);
  if (k1) cudaFree(k1);
  if (v0) cudaFree(v0);
  if (v1) cudaFree(v1);
  if (hist) cudaFree(hist);
  if (st) cudaStreamDestroy(st);
  return rc;
}

// ---------------------------------------------------------------------------
// Allocation-free variant.  Its scratch lives in one file-scope device array:
// two 32-bit key buffers, two 32-bit index buffers and the per-tile digit
// histogram, sized for FELIS_SORT_NOALLOC_MAX_KEYS keys.  Every GPU that
// loads this library holds the array until the process exits.  Each pass
// writes every scratch word it later reads, so nothing has to be cleared
// between calls; calls that overlap on the GPU share the array and race.
namespace {

constexpr int64_t kNaMax = FELIS_SORT_NOALLOC_MAX_KEYS;
constexpr int64_t kNaTiles = (kNaMax + kTile - 1) / kTile;
constexpr size_t kNaBytes = (size_t)4 * kNaMax * 4 + (size_t)256 * kNaTiles * 4;

static __device__ __align__(256) unsigned char g_sort_scratch[kNaBytes];

// Device address of g_sort_scratch per CUDA context.  The address belongs to
// the context that loaded the module: it is resolved again on every call made
// outside stream capture (so a context recreated after cudaDeviceReset, or
// another context made current on the device, gets its own), and a call made
// during capture uses the address last resolved in the current context.
std::mutex g_na_mu;
struct NaEntry {
  CUcontext ctx;
  void* ptr;
};
NaEntry g_na_cache[64];
int g_na_count = 0;
typedef CUresult (*CtxGetCurrentFn)(CUcontext*);
CtxGetCurrentFn g_ctx_get_current = nullptr;

CUcontext current_context() {
  if (!g_ctx_get_current) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return nullptr;
    g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(fn);
  }
  CUcontext c = nullptr;
  return g_ctx_get_current(&c) == CUDA_SUCCESS ? c : nullptr;
}

// Caller-owned buffers must be device (or managed) memory of device `dev`.
bool on_device(const void* p, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
}

__global__ void k_iota32(int32_t* v, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    v[i] = (int32_t)i;
}

__global__ void __launch_bounds__(kThreads) k_scatter32(const int32_t* kin, const int32_t* vin, int64_t n, int shift,
                                                        int ntiles, const uint32_t* offs, int32_t* kout,
                                                        int32_t* vout) {
  __shared__ uint32_t s[kTile];
  const int64_t base = (int64_t)blockIdx.x * kTile;
  for (int i = threadIdx.x; i < kTile; i += blockDim.x) {
    const int64_t e = base + i;
    s[i] = e < n ? ((((uint32_t)kin[e] >> shift) & 255u) << 12) | (uint32_t)i : 0xFFFFFFFFu;
  }
  __syncthreads();
  for (int k = 2; k <= kTile; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < kTile; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const uint32_t a = s[i], b = s[ixj];
          const bool up = (i & k) == 0;
          if ((a > b) == up) { s[i] = b; s[ixj] = a; }
        }
      }
      __syncthreads();
    }
  for (int q = threadIdx.x; q < kTile; q += blockDim.x) {
    const uint32_t c = s[q];
    if (c == 0xFFFFFFFFu) continue;
    const uint32_t d = c >> 12;
    int lo = 0, hi = q;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      if ((s[mid] >> 12) < d) lo = mid + 1;
      else hi = mid;
    }
    const int64_t e = base + (c & 4095u);
    const uint64_t dst = (uint64_t)offs[(size_t)d * ntiles + blockIdx.x] + (uint64_t)(q - lo);
    kout[dst] = kin[e];
    vout[dst] = vin[e];
  }
}

__global__ void k_widen(const int32_t* v, int64_t n, int64_t* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = v[i];
}

}  // namespace

extern "C" felis_status felis_sort_by_slice_noalloc(const int32_t* keys_dev, int64_t n, int64_t* perm_dev,
                                                    void* stream) {
  if (n < 0 || (n > 0 && (!keys_dev || !perm_dev))) return FELIS_BAD_ARG;
  if (n > kNaMax) {
    fprintf(stderr, "felis_sort_by_slice_noalloc: %lld keys exceed the fixed scratch of %lld keys\n",
            (long long)n, (long long)kNaMax);
    return FELIS_BAD_ARG;
  }
  if (n == 0) return FELIS_OK;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return FELIS_NO_DEVICE;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) return FELIS_CUDA_ERROR;
  const bool capturing = cap != cudaStreamCaptureStatusNone;
  if (!capturing && (!on_device(keys_dev, dev) || !on_device(perm_dev, dev))) {
    fprintf(stderr, "felis_sort_by_slice_noalloc: keys_dev and perm_dev must be device memory of the current "
                    "device (%d)\n", dev);
    return FELIS_BAD_ARG;
  }
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_na_mu);
    const CUcontext ctx = current_context();
    if (!ctx) return FELIS_CUDA_ERROR;
    int slot = -1;
    for (int i = 0; i < g_na_count; ++i)
      if (g_na_cache[i].ctx == ctx) slot = i;
    if (!capturing) {
      // resolve the array's device address in this context (the host-side
      // symbol is only a stand-in, not a device address)
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_sort_scratch) != cudaSuccess || !p) return FELIS_CUDA_ERROR;
      if (slot < 0) {
        if (g_na_count == 64) return FELIS_UNSUPPORTED;
        slot = g_na_count++;
        g_na_cache[slot].ctx = ctx;
      }
      g_na_cache[slot].ptr = p;
    } else if (slot < 0) {
      fprintf(stderr, "felis_sort_by_slice_noalloc: the first call in a context must come before stream capture\n");
      return FELIS_BAD_ARG;
    }
    base = g_na_cache[slot].ptr;
  }
  int32_t* K0 = reinterpret_cast<int32_t*>(base);
  int32_t* K1 = K0 + kNaMax;
  int32_t* V0 = K1 + kNaMax;
  int32_t* V1 = V0 + kNaMax;
  uint32_t* hist = reinterpret_cast<uint32_t*>(V1 + kNaMax);
  const int ntiles = (int)((n + kTile - 1) / kTile);
  // four 8-bit passes: keys ordered as unsigned 32-bit values, stable
  k_iota32<<<256, 256, 0, st>>>(V0, n);
  const int32_t* kin = keys_dev;
  const int32_t* vin = V0;
  int32_t* kouts[2] = {K1, K0};
  int32_t* vouts[2] = {V1, V0};
  for (int p = 0; p < 4; ++p) {
    k_hist<<<ntiles, kThreads, 0, st>>>(kin, n, 8 * p, ntiles, hist);
    k_scan<<<1, 1024, 0, st>>>(hist, (int64_t)256 * ntiles);
    k_scatter32<<<ntiles, kThreads, 0, st>>>(kin, vin, n, 8 * p, ntiles, hist, kouts[p & 1], vouts[p & 1]);
    kin = kouts[p & 1];
    vin = vouts[p & 1];
  }
  k_widen<<<256, 256, 0, st>>>(vin, n, perm_dev);
  return cudaGetLastError() == cudaSuccess ? FELIS_OK : FELIS_CUDA_ERROR;
}
