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
#include "tc.cuh"

namespace felis {

namespace {

using namespace tc;

constexpr int kBM = 128;          // rows of a C tile (the MMA M)
constexpr int kBK = 64;           // K columns per stage: 128 bytes of BF16, the swizzle span
constexpr int kStages = 4;
constexpr int kEpiWarps = 8;
constexpr int kThreads = 32 * (2 + kEpiWarps);
constexpr uint32_t kABytes = kBM * kBK * 2;  // 16 KB

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

}  // namespace

bool tma_encode_bf16(CUtensorMap* map, const bf16* base, int rows, int cols, int ld, int box_rows) {
  if (!g_encode) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
  const cuuint32_t box[2] = {(cuuint32_t)kBK, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return g_encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<bf16*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

int gemm_sm_count() { return g_sms; }

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
  if (!tma_encode_bf16(&ta, a.A, a.M, a.K, a.lda, kBM) || !tma_encode_bf16(&tb, a.B, a.N, a.K, a.ldb, a.N)) return cudaErrorInvalidValue;
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
