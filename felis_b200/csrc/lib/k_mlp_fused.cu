// Inference pass of the taper surrogate with the four layers fused: one
// persistent CTA per SM takes 128-row tiles of the input and carries each
// tile through 48 -> 256 -> 256 -> 256 -> 48 on the tensor cores; the hidden
// activations never leave the SM.
//
// Per CTA: two tile slots.  A slot owns a 64 KB activation buffer in shared
// memory (128 rows x 256 BF16 columns as four K-major, 128-byte swizzled
// chunks: the A operand of the next layer) and a 256-column FP32 accumulator
// in tensor memory (512 columns in all).  The weights stream through a ring
// of three 32 KB stages (one 64-column K chunk of a weight matrix each),
// loaded by TMA from L2.  Work goes in a fixed order known to every role:
// for each pair of tiles, layer by layer, slot 0 then slot 1, so that one
// slot's epilogue runs while the other slot's MMAs do.
//   warp 0     one lane: TMA loads of the input tile (into its slot's buffer,
//              once the slot's last-layer MMAs have finished with it) and of
//              the weight chunks, in job order
//   warp 1     allocates the tensor memory; one lane issues tcgen05.mma
//              (M = 128, K = 16) per job once its operand is in place and
//              the slot's accumulator has been read, commits each weight
//              stage back to the producer and each finished accumulator to
//              the epilogue
//   warps 2-9  the epilogue: warp w reads lanes 32 (w % 4) .. + 31 of the
//              accumulator (one row per thread), two warps per lane quarter
//              splitting the columns; bias and GELU, BF16 into the slot's
//              activation buffer in the swizzled layout (hidden layers), or
//              bias and FP32 rows to global memory (last layer)
// Every mbarrier wait is bounded (tc::mbar_wait); one that runs out sets the
// error word and the flag that stops the other roles, and the MMA lane waits
// (bounded) for its MMAs in flight before the tensor memory is freed.  The
// TMA loads read this GPU's own memory, without multicast.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "mlp.cuh"
#include "tc.cuh"

namespace felis {

namespace {

using namespace tc;

constexpr int kBM = 128;                          // rows of a tile (the MMA M)
constexpr int kWidth = 256;                       // hidden width
constexpr uint32_t kActChunk = kBM * 128;         // one 64-column K chunk of a tile: 16 KB
constexpr uint32_t kAct = 4 * kActChunk;          // a slot's activation buffer: 64 KB
constexpr uint32_t kWStage = kWidth * 128;        // one K chunk of a 256-row weight: 32 KB
constexpr int kWStages = 3;
constexpr int kEpiWarps = 8;
constexpr int kThreads = 32 * (2 + kEpiWarps);
constexpr int kTmemCols = 2 * kWidth;
constexpr size_t kSmem = 1024 + 2 * (size_t)kAct + (size_t)kWStages * kWStage;

struct FusedParams {
  int M, in_k, out_n;
  const float* bias[4];
  float* y;
  int* err;
};

__global__ void __launch_bounds__(kThreads, 1)
    k_mlp_fused(const __grid_constant__ CUtensorMap tmX, const __grid_constant__ CUtensorMap tmW1,
                const __grid_constant__ CUtensorMap tmW2, const __grid_constant__ CUtensorMap tmW3,
                const __grid_constant__ CUtensorMap tmW4, FusedParams f) {
  extern __shared__ unsigned char smraw[];
  __shared__ __align__(8) uint64_t wfull[kWStages], wempty[kWStages];
  __shared__ __align__(8) uint64_t xfull[2], afree[2], accfull[2], epidone[2];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  unsigned char* sm = smraw + ((1024u - (sa(smraw) & 1023u)) & 1023u);
  unsigned char* act = sm;                  // [2][kAct]
  unsigned char* wring = sm + 2 * kAct;     // [kWStages][kWStage]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ntiles = f.M / kBM;
  // tiles of this CTA: blockIdx.x + k gridDim.x, k < nt; tile k sits in slot
  // k & 1 as that slot's (k >> 1)-th tile
  const int nt = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  volatile int* abort_v = &abort_flag;

  if (threadIdx.x == 0) {
    for (int s = 0; s < kWStages; ++s) {
      mbar_init(sa(&wfull[s]), 1);
      mbar_init(sa(&wempty[s]), 1);
    }
    for (int s = 0; s < 2; ++s) {
      mbar_init(sa(&xfull[s]), 1);
      mbar_init(sa(&afree[s]), 1);
      mbar_init(sa(&accfull[s]), 1);
      mbar_init(sa(&epidone[s]), kEpiWarps * 32);
    }
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sa(&tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = tmem_slot;

  auto give_up = [&]() {
    *abort_v = 1;
    if (f.err) atomicOr(f.err, 1);
  };

  if (warp == 0) {
    if (lane == 0) {
      const CUtensorMap* maps[5] = {&tmX, &tmW1, &tmW2, &tmW3, &tmW4};
      for (int i = 0; i < 5; ++i)
        asm volatile("prefetch.tensormap [%0];\n" ::"l"(reinterpret_cast<uint64_t>(maps[i])) : "memory");
      int ws = 0;
      uint32_t wph = 0;
      bool ok = true;
      // one weight chunk into the next ring stage
      auto load_w = [&](const CUtensorMap* map, int kc, uint32_t bytes) {
        // a fresh stage passes at once (the phase before the first counts as complete)
        if (!mbar_wait(sa(&wempty[ws]), wph ^ 1u, abort_v)) { give_up(); ok = false; return; }
        mbar_expect_tx(sa(&wfull[ws]), bytes);
        tma_load_2d(sa(wring + (size_t)ws * kWStage), map, kc * 64, 0, sa(&wfull[ws]));
        if (++ws == kWStages) { ws = 0; wph ^= 1u; }
      };
      for (int p = 0; 2 * p < nt && ok; ++p)
        for (int l = 0; l < 4 && ok; ++l)
          for (int s = 0; s < 2 && ok; ++s) {
            const int k = 2 * p + s;
            if (k >= nt) continue;
            if (l == 0) {
              // the slot's buffer is free once its previous tile's last-layer MMAs finished
              if (p > 0 && !mbar_wait(sa(&afree[s]), (uint32_t)(p - 1) & 1u, abort_v)) { give_up(); ok = false; break; }
              const int tile = blockIdx.x + k * gridDim.x;
              mbar_expect_tx(sa(&xfull[s]), kActChunk);
              tma_load_2d(sa(act + (size_t)s * kAct), &tmX, 0, tile * kBM, sa(&xfull[s]));
              load_w(&tmW1, 0, kWStage);
            } else {
              for (int kc = 0; kc < 4 && ok; ++kc)
                load_w(l == 1 ? &tmW2 : (l == 2 ? &tmW3 : &tmW4), kc, l == 3 ? (uint32_t)f.out_n * 128u : kWStage);
            }
          }
    }
    __syncwarp();
  } else if (warp == 1) {
    if (lane == 0) {
      int ws = 0;
      uint32_t wph = 0;
      uint32_t last_bar = 0, last_par = 0;  // last commit, waited for on the way out
      bool ok = true;
      const uint32_t id_hidden = idesc_bf16(kBM, kWidth), id_out = idesc_bf16(kBM, f.out_n);
      for (int p = 0; 2 * p < nt && ok; ++p)
        for (int l = 0; l < 4 && ok; ++l)
          for (int s = 0; s < 2 && ok; ++s) {
            if (2 * p + s >= nt) continue;
            // operand A in place, and the accumulator read by the epilogue
            if (l == 0) {
              if (!mbar_wait(sa(&xfull[s]), (uint32_t)p & 1u, abort_v)) { give_up(); ok = false; break; }
              if (p > 0 && !mbar_wait(sa(&epidone[s]), 1u, abort_v)) { give_up(); ok = false; break; }
            } else if (!mbar_wait(sa(&epidone[s]), (uint32_t)(l - 1) & 1u, abort_v)) {
              give_up(); ok = false; break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
            const uint32_t d = tmem + (uint32_t)(s * kWidth);
            const uint32_t a_s = sa(act + (size_t)s * kAct);
            const int nkc = l == 0 ? 1 : 4;
            const int ksteps = l == 0 ? f.in_k / 16 : 4;
            for (int kc = 0; kc < nkc; ++kc) {
              if (!mbar_wait(sa(&wfull[ws]), wph, abort_v)) { give_up(); ok = false; break; }
              asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
              const uint32_t w_s = sa(wring + (size_t)ws * kWStage);
              const uint32_t ak = a_s + (uint32_t)kc * kActChunk;
              for (int kk = 0; kk < ksteps; ++kk)
                mma_bf16(d, desc_sw128(ak + 32u * kk), desc_sw128(w_s + 32u * kk), l == 3 ? id_out : id_hidden,
                         (kc | kk) ? 1u : 0u);
              mma_commit(sa(&wempty[ws]));
              last_bar = sa(&wempty[ws]);
              last_par = wph;
              if (++ws == kWStages) { ws = 0; wph ^= 1u; }
            }
            if (!ok) break;
            mma_commit(sa(&accfull[s]));
            last_bar = sa(&accfull[s]);
            last_par = (uint32_t)l & 1u;  // the (4p + l + 1)-th completion of accfull[s]
            if (l == 3) mma_commit(sa(&afree[s]));
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
    const int r = q * 32 + lane;       // this thread's row of the tile
    bool ok = true;
    for (int p = 0; 2 * p < nt && ok; ++p)
      for (int l = 0; l < 4 && ok; ++l)
        for (int s = 0; s < 2 && ok; ++s) {
          const int k = 2 * p + s;
          if (k >= nt) continue;
          // the (4p + l + 1)-th completion of the slot's accumulator barrier
          if (!mbar_wait(sa(&accfull[s]), (uint32_t)l & 1u, abort_v)) { give_up(); ok = false; break; }
          asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
          const uint32_t tbase = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(s * kWidth);
          const float* __restrict__ bias = f.bias[l];
          if (l < 3) {
            unsigned char* a_s = act + (size_t)s * kAct;
#pragma unroll 1
            for (int i = 0; i < 4; ++i) {
              const int c0 = half * 128 + i * 32;
              uint32_t v[32];
              TMEM_LD32X32(tbase + (uint32_t)c0, v);
              asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
              uint32_t w[16];
#pragma unroll
              for (int j = 0; j < 16; ++j) {
                const float2 b2 = __ldg(reinterpret_cast<const float2*>(bias + c0) + j);
                const float x0 = gelu_f(__uint_as_float(v[2 * j]) + b2.x);
                const float x1 = gelu_f(__uint_as_float(v[2 * j + 1]) + b2.y);
                const __nv_bfloat162 h2 = __floats2bfloat162_rn(x0, x1);
                w[j] = *reinterpret_cast<const uint32_t*>(&h2);
              }
              // 128-byte swizzle: 16-byte granule g of row r sits at granule g ^ (r % 8)
              unsigned char* rowp = a_s + (size_t)(c0 >> 6) * kActChunk + (size_t)r * 128;
              const int g0 = (c0 & 63) >> 3;
#pragma unroll
              for (int j = 0; j < 4; ++j)
                *reinterpret_cast<uint4*>(rowp + (((g0 + j) ^ (r & 7)) << 4)) =
                    make_uint4(w[4 * j], w[4 * j + 1], w[4 * j + 2], w[4 * j + 3]);
            }
            // the next layer's MMAs read these through the async proxy
            asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
          } else {
            const int tile = blockIdx.x + k * gridDim.x;
            float* yrow = f.y + ((size_t)tile * kBM + r) * (size_t)f.out_n;
            for (int c0 = half * 32; c0 < f.out_n; c0 += 64) {
              uint32_t v[32];
              TMEM_LD32X32(tbase + (uint32_t)c0, v);
              asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
              const int ncol = f.out_n - c0 < 32 ? f.out_n - c0 : 32;  // 16 or 32
#pragma unroll
              for (int j = 0; j < 8; ++j) {
                if (4 * j >= ncol) break;
                const float4 b4 = __ldg(reinterpret_cast<const float4*>(bias + c0) + j);
                *reinterpret_cast<float4*>(yrow + c0 + 4 * j) =
                    make_float4(__uint_as_float(v[4 * j]) + b4.x, __uint_as_float(v[4 * j + 1]) + b4.y,
                                __uint_as_float(v[4 * j + 2]) + b4.z, __uint_as_float(v[4 * j + 3]) + b4.w);
              }
            }
          }
          asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
          mbar_arrive(sa(&epidone[s]));
        }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 1)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kTmemCols) : "memory");
}

}  // namespace

cudaError_t mlp_fused_prepare() {
  return cudaFuncSetAttribute(k_mlp_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
}

bool mlp_fused_supported(int width, int in_k, int out_n) {
  return width == kWidth && in_k % 16 == 0 && in_k >= 16 && in_k <= 64 && out_n % 16 == 0 && out_n >= 16 &&
         out_n <= kWidth;
}

cudaError_t launch_mlp_fused(const MlpFusedArgs& a, cudaStream_t st) {
  const int sms = gemm_sm_count();
  if (sms <= 0) return cudaErrorNotReady;
  if (a.M % kBM || !mlp_fused_supported(a.width, a.in_k, a.out_n) || (reinterpret_cast<uintptr_t>(a.x) & 15) ||
      (reinterpret_cast<uintptr_t>(a.y) & 15))
    return cudaErrorInvalidValue;
  for (int l = 0; l < 4; ++l)
    if (!a.w[l] || !a.bias[l] || (reinterpret_cast<uintptr_t>(a.w[l]) & 15) ||
        (reinterpret_cast<uintptr_t>(a.bias[l]) & 15))
      return cudaErrorInvalidValue;
  CUtensorMap mx, m1, m2, m3, m4;
  // input [M][in_k] and W1 [256][in_k]: 64-column boxes, the columns past in_k read as zero
  if (!tma_encode_bf16(&mx, a.x, a.M, a.in_k, a.in_k, kBM) || !tma_encode_bf16(&m1, a.w[0], kWidth, a.in_k, a.in_k, kWidth) ||
      !tma_encode_bf16(&m2, a.w[1], kWidth, kWidth, kWidth, kWidth) ||
      !tma_encode_bf16(&m3, a.w[2], kWidth, kWidth, kWidth, kWidth) ||
      !tma_encode_bf16(&m4, a.w[3], a.out_n, kWidth, kWidth, a.out_n))
    return cudaErrorInvalidValue;
  FusedParams f;
  f.M = a.M; f.in_k = a.in_k; f.out_n = a.out_n;
  for (int l = 0; l < 4; ++l) f.bias[l] = a.bias[l];
  f.y = a.y; f.err = a.err;
  const int tiles = a.M / kBM;
  const int grid = tiles < sms ? tiles : sms;
  if (grid == 0) return cudaSuccess;
  k_mlp_fused<<<grid, kThreads, kSmem, st>>>(mx, m1, m2, m3, m4, f);
  return cudaGetLastError();
}

}  // namespace felis
