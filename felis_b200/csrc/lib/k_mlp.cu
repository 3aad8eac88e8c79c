// Elementwise kernels of the taper-surrogate MLP (its GEMMs are in
// k_gemm.cu) and the self-test of the library's bounded mbarrier wait.
#include <math.h>

#include "mlp.cuh"
#include "tc.cuh"

namespace felis {

namespace {

constexpr int kWaitLimit = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Bounded wait for the phase `parity` of an mbarrier; false when it ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, int limit = kWaitLimit) {
  for (int it = 0; it < limit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// The bounded wait on an mbarrier that nothing arrives on: phase 0 never
// completes, so every thread's wait runs out after `limit` tries and the
// kernel records that, then returns with nothing in flight.
__global__ void __launch_bounds__(128) k_wait_selftest(int limit, int* timed_out) {
  __shared__ __align__(8) uint64_t bar;
  const uint32_t b = smem_u32(&bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(b) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  const bool done = mbar_wait(b, 0u, limit);
  const int all_ran_out = __syncthreads_and(done ? 0 : 1);
  if (threadIdx.x == 0) *timed_out = all_ran_out;
}

// Derivative of the tanh-form GELU of tc.cuh: with t = tanh(u),
// u = c (z + a z^3): 0.5 (1 + t) + 0.5 z (1 - t^2) c (1 + 3 a z^2).
__device__ __forceinline__ float gelu_grad(float z) {
  const float c = 0.79788456080286536f, a = 0.044715f;
  const float t = tc::tanh_hw(c * fmaf(a * z, z * z, z));
  return 0.5f * (1.f + t) + 0.5f * z * (1.f - t * t) * c * fmaf(3.f * a * z, z, 1.f);
}

__global__ void k_f32_to_bf16(const float* in, bf16* out, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn(in[i]);
}

__global__ void k_transpose_bf16(const bf16* in, int rows, int cols, int ld_in, bf16* out, int rows_pad,
                                 int cols_pad) {
  const int64_t n = (int64_t)rows_pad * cols_pad;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i / rows_pad), r = (int)(i % rows_pad);
    out[i] = (r < rows && c < cols) ? in[(size_t)r * ld_in + c] : __float2bfloat16_rn(0.f);
  }
}

__global__ void k_gelu_backward(const float* z, const float* g, bf16* dz, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dz[i] = __float2bfloat16_rn(g[i] * gelu_grad(z[i]));
}

constexpr int kMseRows = 32;  // rows per block of the loss kernel

__global__ void __launch_bounds__(256) k_mse_grad(const float* y, const float* t, int rows, int rows_real,
                                                  int cols_pad, int cols_real, float scale, bf16* dy,
                                                  double* part) {
  __shared__ double red[8];
  double acc = 0.0;
  const int r0 = blockIdx.x * kMseRows;
  for (int k = threadIdx.x; k < kMseRows * cols_pad; k += blockDim.x) {
    const int r = r0 + k / cols_pad, c = k % cols_pad;
    if (r >= rows) continue;
    const size_t i = (size_t)r * cols_pad + c;
    float d = 0.f;
    if (r < rows_real && c < cols_real) {
      d = y[i] - t[i];
      acc += (double)d * d;
    }
    dy[i] = __float2bfloat16_rn(scale * d);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    part[blockIdx.x] = s;
  }
}

__global__ void k_col_sum(const bf16* in, int rows, int cols, float* out) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= cols) return;
  float s = 0.f;
  for (int r = 0; r < rows; ++r) s += __bfloat162float(in[(size_t)r * cols + c]);
  out[c] = s;
}

__global__ void k_adamw(float* w, const float* g, float* m, float* v, bf16* wb, int64_t n, float lr, float b1,
                        float b2, float eps, float wd, float bc1, float bc2) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float upd = (mi / bc1) / (sqrtf(vi / bc2) + eps) + wd * w[i];
    const float wi = w[i] - lr * upd;
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
  }
}

int grid_for(int64_t n) { return (int)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096); }

}  // namespace

void launch_f32_to_bf16(const float* in, bf16* out, int64_t n, cudaStream_t st) {
  if (n > 0) k_f32_to_bf16<<<grid_for(n), 256, 0, st>>>(in, out, n);
}

void launch_transpose_bf16(const bf16* in, int rows, int cols, int ld_in, bf16* out, int rows_pad, int cols_pad,
                           cudaStream_t st) {
  const int64_t n = (int64_t)rows_pad * cols_pad;
  if (n > 0) k_transpose_bf16<<<grid_for(n), 256, 0, st>>>(in, rows, cols, ld_in, out, rows_pad, cols_pad);
}

void launch_gelu_backward(const float* z, const float* g, bf16* dz, int64_t n, cudaStream_t st) {
  if (n > 0) k_gelu_backward<<<grid_for(n), 256, 0, st>>>(z, g, dz, n);
}

int mse_blocks(int rows) { return (rows + kMseRows - 1) / kMseRows; }

void launch_mse_grad(const float* y, const float* t, int rows, int rows_real, int cols_pad, int cols_real,
                     float scale, bf16* dy, double* loss_part, cudaStream_t st) {
  k_mse_grad<<<mse_blocks(rows), 256, 0, st>>>(y, t, rows, rows_real, cols_pad, cols_real, scale, dy, loss_part);
}

void launch_col_sum(const bf16* in, int rows, int cols, float* out, cudaStream_t st) {
  k_col_sum<<<(cols + 127) / 128, 128, 0, st>>>(in, rows, cols, out);
}

void launch_adamw(float* w, const float* g, float* m, float* v, bf16* w_bf16, int64_t n, float lr, float b1,
                  float b2, float eps, float wd, float bc1, float bc2, cudaStream_t st) {
  if (n > 0) k_adamw<<<grid_for(n), 256, 0, st>>>(w, g, m, v, w_bf16, n, lr, b1, b2, eps, wd, bc1, bc2);
}

void launch_wait_selftest(int limit, int* timed_out, cudaStream_t st) {
  k_wait_selftest<<<1, 128, 0, st>>>(limit, timed_out);
}

}  // namespace felis
