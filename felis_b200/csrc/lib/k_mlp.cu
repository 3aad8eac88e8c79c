// Kernels of the taper-surrogate MLP.
//
// k_gemm_tc: C = A . B^T on the tcgen05 tensor cores.  One CTA of four warps
// owns a 128 x N tile (N <= 256) of C, held as FP32 in tensor memory (256
// columns, allocated by warp 0).  K is staged 64 columns at a time into shared
// memory with 16-byte cp.async copies, in the canonical K-major layout without
// swizzle: 8-row x 16-byte core matrices, the two core matrices of one
// 16-element K step 128 B apart (leading byte offset), consecutive 8-row groups
// 1024 B apart (stride byte offset).  One thread issues the MMAs (M = 128,
// N = tile width, K = 16 each) and commits them to an mbarrier; every wait on
// it is bounded.  The epilogue reads the accumulator back with tcgen05.ld
// (warp w owns rows 32w..32w+31, one row per thread) and applies bias and
// GELU.
#include <math.h>

#include "mlp.cuh"

namespace felis {

namespace {

constexpr int kBM = 128;        // rows of the C tile (the MMA M)
constexpr int kBN = 256;        // widest C tile (the MMA N limit)
constexpr int kKC = 64;         // K columns staged per chunk
constexpr int kTmemCols = 256;  // FP32 accumulator columns
constexpr int kGroupBytes = 1024;  // one 8-row group of a 64-column chunk
constexpr int kWaitLimit = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: canonical K-major layout, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         (1ull << 46);  // descriptor version of this architecture
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, dense, shape M x N.
__device__ __forceinline__ uint32_t instr_desc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}

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

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

#define TMEM_LD32(taddr, r)                                                                                      \
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "                                                        \
               "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"                                         \
               "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"                       \
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),  \
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),         \
                 "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),       \
                 "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),       \
                 "=r"(r[29]), "=r"(r[30]), "=r"(r[31])                                                            \
               : "r"(taddr))

__global__ void __launch_bounds__(128) k_gemm_tc(GemmArgs g) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * kBM, n0 = blockIdx.y * kBN;
  const int NT = min(kBN, g.N - n0);  // a multiple of 16
  const uint32_t a_s = smem_u32(sm), b_s = a_s + kBM / 8 * kGroupBytes;
  const uint32_t bar_s = smem_u32(&bar);
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar_s) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t idesc = instr_desc_bf16(kBM, NT);
  uint32_t parity = 0;
  bool ok = true;
  for (int k0 = 0; k0 < g.K && ok; k0 += kKC) {
    const int kc = min(kKC, g.K - k0);  // a multiple of 16
    const int cpr = kc / 8;             // 16-byte pieces per row
    for (int p = tid; p < kBM * cpr; p += blockDim.x) {
      const int r = p / cpr, c = p % cpr;
      cp_async16(a_s + (r >> 3) * kGroupBytes + c * 128 + (r & 7) * 16, g.A + (size_t)(m0 + r) * g.lda + k0 + 8 * c);
    }
    for (int p = tid; p < NT * cpr; p += blockDim.x) {
      const int r = p / cpr, c = p % cpr;
      cp_async16(b_s + (r >> 3) * kGroupBytes + c * 128 + (r & 7) * 16, g.B + (size_t)(n0 + r) * g.ldb + k0 + 8 * c);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      for (int ks = 0; ks < kc / 16; ++ks) {
        const uint64_t da = smem_desc(a_s + ks * 256, 128, kGroupBytes);
        const uint64_t db = smem_desc(b_s + ks * 256, 128, kGroupBytes);
        const uint32_t accumulate = (k0 > 0 || ks > 0) ? 1u : 0u;
        const uint32_t mask = 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(accumulate), "r"(mask)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar_s)
                   : "memory");
    }
    // the MMAs read the staged tiles: wait before the next chunk overwrites them
    ok = mbar_wait(bar_s, parity);
    parity ^= 1u;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    ok = __syncthreads_and(ok) != 0;
  }
  if (!ok) {
    // give MMAs still in flight a second bounded wait before the memory goes
    mbar_wait(bar_s, parity ^ 1u);
    if (tid == 0 && g.err) atomicOr(g.err, 1);
  } else {
    const int row = m0 + warp * 32 + lane;
    const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
    for (int c0 = 0; c0 < NT; c0 += 32) {
      uint32_t r[32];
      TMEM_LD32(trow + (uint32_t)c0, r);
      asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
      const bool full = c0 + 32 <= NT;
#pragma unroll
      for (int j = 0; j < 32; ++j) {
        const int cl = c0 + j;
        if (!full && cl >= NT) break;
        const int col = n0 + cl;
        float v = __uint_as_float(r[j]);
        if (col < g.n_valid) {
          if (g.bias) v += g.bias[col];
        } else {
          v = 0.f;
        }
        if (g.out_f32) g.out_f32[(size_t)row * g.ldc + col] = v;
        if (g.out_bf16) g.out_bf16[(size_t)row * g.ldc + col] = __float2bfloat16_rn(g.gelu && col < g.n_valid ? gelu(v) : v);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols) : "memory");
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

cudaError_t gemm_tc_prepare() {
  return cudaFuncSetAttribute(k_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (kBM + kBN) / 8 * kGroupBytes);
}

void launch_gemm_tc(const GemmArgs& g, cudaStream_t st) {
  const dim3 grid(g.M / kBM, (g.N + kBN - 1) / kBN);
  const int smem = (kBM + kBN) / 8 * kGroupBytes;  // 48 KB
  k_gemm_tc<<<grid, 128, smem, st>>>(g);
}

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
