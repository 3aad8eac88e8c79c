// BF16 GEMM of the taper surrogate on the 5th-generation tensor cores:
// C[M][N] = A[M][K] . B[N][K]^T, FP32 accumulation in tensor memory, with the
// epilogue of mlp.cuh (bias, GELU, FP32 and/or BF16 outputs).
//
// One persistent CTA per SM walks the 128-row tiles of C (N <= 256 columns,
// one tile wide).  Warp roles:
//   warp 0     one lane issues the TMA loads: the A tile (128 x 64) and the
//              B tile (N x 64) of every 64-column K chunk, 128-byte swizzle,
//              into a ring of kStages shared-memory stages (full / empty
//              mbarriers per stage)
//   warp 1     allocates tensor memory (two accumulators of N columns, 32-column
//              aligned); one lane issues tcgen05.mma (M = 128, N, K = 16; four
//              per chunk) and commits each stage back to the producer and each
//              finished accumulator to the epilogue
//   warps 2-9  the epilogue: warp w reads lanes 32 (w % 4) .. + 31 of the
//              accumulator (tcgen05.ld, one row per thread), two warps per
//              lane quarter taking alternate 32-column chunks; each thread
//              applies bias / GELU to its 32 values and writes them with
//              16-byte stores, then the warps free the accumulator
// The two accumulators alternate, so a tile's epilogue overlaps the next
// tile's loads and MMAs.  Every mbarrier wait is bounded: one that runs out
// sets the error word and the flag that stops the other roles; the MMA lane
// then waits (bounded) for its MMAs in flight before the tensor memory is
// freed.  The TMA loads read this GPU's own memory, without multicast.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "mlp.cuh"

namespace felis {

namespace {

constexpr int kBM = 128;          // rows of a C tile (the MMA M)
constexpr int kBK = 64;           // K columns per stage: 128 bytes of BF16, the swizzle span
constexpr int kStages = 4;
constexpr int kEpiWarps = 8;
constexpr int kThreads = 32 * (2 + kEpiWarps);
constexpr int kWaitTries = 1 << 20;
constexpr uint32_t kABytes = kBM * kBK * 2;  // 16 KB

__device__ __forceinline__ uint32_t sa(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait; false when it ran out or another role gave up.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag) {
  for (int it = 0; it < kWaitTries; ++it) {
    if (mbar_try(bar, parity)) return true;
    if ((it & 255) == 255 && *abort_flag) return false;
  }
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}

// 2-D tiled TMA load from this GPU's memory (no multicast); x is the element
// column (a multiple of 64 here: 128 bytes), y the row.
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}

// Shared-memory descriptor of a K-major operand tile in the 128-byte swizzled
// layout the TMA writes: 8-row groups 1024 bytes apart (stride byte offset),
// layout type SWIZZLE_128B (2), descriptor version 1.
__device__ __forceinline__ uint64_t desc_sw128(uint32_t addr) {
  return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) |
         ((uint64_t)1 << 46) | ((uint64_t)2 << 61);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, dense, M x N.
__device__ __forceinline__ uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(bar) : "memory");
}

#define TMEM_LD32X32(taddr, r)                                                                                  \
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "                                                        \
               "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"                                         \
               "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"                       \
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),  \
                 "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),         \
                 "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),       \
                 "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),       \
                 "=r"(r[29]), "=r"(r[30]), "=r"(r[31])                                                            \
               : "r"(taddr))

__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }

struct TmaGemm {
  int M, N, K;     // M a multiple of 128, N a multiple of 16 (<= 256), K a multiple of 16
  int tmem_cols;   // allocated tensor-memory columns
  int acc_stride;  // column offset of the second accumulator (N rounded up to 32)
  const float* bias;
  float* out_f32;
  bf16* out_bf16;
  int ldc, n_valid, gelu;
  int* err;
};

__global__ void __launch_bounds__(kThreads, 1) k_gemm_tma(const __grid_constant__ CUtensorMap tmA,
                                                           const __grid_constant__ CUtensorMap tmB, TmaGemm g) {
  extern __shared__ unsigned char smraw[];
  __shared__ __align__(8) uint64_t full[kStages], empty[kStages], tfull[2], tempty[2];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  // the swizzled operand tiles start on 1024-byte boundaries of the shared window
  unsigned char* sm = smraw + ((1024u - (sa(smraw) & 1023u)) & 1023u);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int N = g.N;
  const uint32_t stage_bytes = kABytes + (uint32_t)N * kBK * 2;
  const int ntiles = g.M / kBM;
  const int nk = (g.K + kBK - 1) / kBK;
  volatile int* abort_v = &abort_flag;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(sa(&full[s]), 1);
      mbar_init(sa(&empty[s]), 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(sa(&tfull[b]), 1);
      mbar_init(sa(&tempty[b]), kEpiWarps * 32);
    }
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sa(&tmem_slot)),
                 "r"(g.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_slot;

  auto give_up = [&]() {
    *abort_v = 1;
    if (g.err) atomicOr(g.err, 1);
  };

  if (warp == 0) {
    if (lane == 0) {
      asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&tmA)) : "memory");
      asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(&tmB)) : "memory");
      int s = 0;
      uint32_t ph = 0;
      bool ok = true;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x)
        for (int k = 0; k < nk && ok; ++k) {
          // a fresh stage passes at once (the phase before the first counts as complete)
          if (!mbar_wait(sa(&empty[s]), ph ^ 1u, abort_v)) { give_up(); ok = false; break; }
          const uint32_t a_s = sa(sm + (size_t)s * stage_bytes);
          mbar_expect_tx(sa(&full[s]), stage_bytes);
          tma_load_2d(a_s, &tmA, k * kBK, t * kBM, sa(&full[s]));
          tma_load_2d(a_s + kABytes, &tmB, k * kBK, 0, sa(&full[s]));
          if (++s == kStages) { s = 0; ph ^= 1u; }
        }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = idesc_bf16(kBM, N);
      int s = 0, it = 0;
      uint32_t ph = 0;
      uint32_t last_bar = 0, last_par = 0;  // last commit, waited for on the way out
      bool ok = true;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++it) {
        const int b = it & 1;
        const uint32_t bph = (uint32_t)(it >> 1) & 1u;
        if (!mbar_wait(sa(&tempty[b]), bph ^ 1u, abort_v)) { give_up(); ok = false; break; }
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const uint32_t d = tmem + (uint32_t)(b * g.acc_stride);
        for (int k = 0; k < nk; ++k) {
          if (!mbar_wait(sa(&full[s]), ph, abort_v)) { give_up(); ok = false; break; }
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          const uint32_t a_s = sa(sm + (size_t)s * stage_bytes), b_s = a_s + kABytes;
#pragma unroll
          for (int kk = 0; kk < kBK / 16; ++kk)
            mma_bf16(d, desc_sw128(a_s + 32u * kk), desc_sw128(b_s + 32u * kk), idesc, (k | kk) ? 1u : 0u);
          mma_commit(sa(&empty[s]));
          last_bar = sa(&empty[s]);
          last_par = ph;
          if (++s == kStages) { s = 0; ph ^= 1u; }
        }
        if (!ok) break;
        mma_commit(sa(&tfull[b]));
        last_bar = sa(&tfull[b]);
        last_par = bph;
      }
      // the tensor memory is freed below: wait for the last MMAs issued
      if (last_bar) {
        for (int i = 0; i < kWaitTries && !mbar_try(last_bar, last_par); ++i) {
        }
      }
    }
    __syncwarp();
  } else {
    const int q = warp & 3;            // tensor-memory lane quarter this warp may read
    const int half = (warp - 2) >> 2;  // which of the two warps of that quarter
    int it = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
      const int b = it & 1;
      const uint32_t bph = (uint32_t)(it >> 1) & 1u;
      if (!mbar_wait(sa(&tfull[b]), bph, abort_v)) { give_up(); break; }
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * g.acc_stride);
      const size_t row = (size_t)t * kBM + (size_t)q * 32 + lane;
      for (int c0 = 32 * half; c0 < N; c0 += 64) {
        uint32_t r[32];
        TMEM_LD32X32(tbase + (uint32_t)c0, r);
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
        const int ncol = N - c0 < 32 ? N - c0 : 32;  // 16 or 32 (N is a multiple of 16)
        float v[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) {
          const int col = c0 + j;
          const bool valid = col < g.n_valid;
          v[j] = valid ? __uint_as_float(r[j]) + (g.bias ? __ldg(g.bias + col) : 0.f) : 0.f;
        }
        const size_t o = row * (size_t)g.ldc + c0;
        if (g.out_f32) {
          float4* dst = reinterpret_cast<float4*>(g.out_f32 + o);
#pragma unroll
          for (int j = 0; j < 8; ++j)
            if (4 * j < ncol) dst[j] = make_float4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
        }
        if (g.out_bf16) {
          uint4* dst = reinterpret_cast<uint4*>(g.out_bf16 + o);
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            if (8 * j >= ncol) break;
            uint32_t w[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
              float x0 = v[8 * j + 2 * k], x1 = v[8 * j + 2 * k + 1];
              if (g.gelu) {
                if (c0 + 8 * j + 2 * k < g.n_valid) x0 = gelu_f(x0);
                if (c0 + 8 * j + 2 * k + 1 < g.n_valid) x1 = gelu_f(x1);
              }
              const __nv_bfloat162 p2 = __floats2bfloat162_rn(x0, x1);
              w[k] = *reinterpret_cast<const uint32_t*>(&p2);
            }
            dst[j] = make_uint4(w[0], w[1], w[2], w[3]);
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
      mbar_arrive(sa(&tempty[b]));
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(g.tmem_cols) : "memory");
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn g_encode = nullptr;
int g_sms = 0;

size_t tma_smem(int N) { return 1024 + (size_t)kStages * (kABytes + (size_t)N * kBK * 2); }

// Row-major BF16 matrix [rows][ld] read in (64 x box_rows) tiles of its
// first `cols` columns; out-of-range elements read as zero.
bool encode(CUtensorMap* map, const bf16* base, int rows, int cols, int ld, int box_rows) {
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return g_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

cudaError_t gemm_tma_prepare() {
  if (!g_encode) {
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess) return e;
    if (q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
    g_encode = reinterpret_cast<EncodeTiledFn>(fn);
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_gemm_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tma_smem(256));
  return e;
}

cudaError_t launch_gemm_tma(const GemmArgs& a, cudaStream_t st) {
  if (!g_encode || g_sms <= 0) return cudaErrorNotReady;
  if (a.M % kBM || a.N % 16 || a.N < 16 || a.N > 256 || a.K % 16 || a.K < 16 || a.lda % 8 || a.ldb % 8 ||
      (reinterpret_cast<uintptr_t>(a.A) & 15) || (reinterpret_cast<uintptr_t>(a.B) & 15))
    return cudaErrorInvalidValue;
  CUtensorMap ta, tb;
  if (!encode(&ta, a.A, a.M, a.K, a.lda, kBM) || !encode(&tb, a.B, a.N, a.K, a.ldb, a.N)) return cudaErrorInvalidValue;
  TmaGemm g;
  g.M = a.M; g.N = a.N; g.K = a.K;
  // two accumulators 32-column aligned (the epilogue reads 32 columns at a
  // time), in a power-of-two allocation of at least 32 columns
  g.acc_stride = (a.N + 31) & ~31;
  int cols = 32;
  while (cols < 2 * g.acc_stride) cols <<= 1;
  g.tmem_cols = cols;
  g.bias = a.bias; g.out_f32 = a.out_f32; g.out_bf16 = a.out_bf16;
  g.ldc = a.ldc; g.n_valid = a.n_valid; g.gelu = a.gelu; g.err = a.err;
  const int tiles = a.M / kBM;
  const int grid = tiles < g_sms ? tiles : g_sms;
  k_gemm_tma<<<grid, kThreads, tma_smem(a.N), st>>>(ta, tb, g);
  return cudaGetLastError();
}

}  // namespace felis
