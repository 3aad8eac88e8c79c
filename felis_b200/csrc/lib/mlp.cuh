// Taper-surrogate MLP: tensor-core GEMM and the elementwise kernels of its
// forward pass, backward pass and AdamW update.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace felis {

typedef __nv_bfloat16 bf16;

// C[M][N] = A[M][K] . B[N][K]^T on the 5th-generation tensor cores (BF16
// operands, FP32 accumulation in tensor memory), with an optional epilogue:
//   z = C + bias[n]                (bias may be null)
//   out_f32[m][n] = z              (may be null)
//   out_bf16[m][n] = gelu ? GELU(z) : z   (may be null)
// A and B are row-major with leading dimensions lda, ldb (elements, multiples
// of 8); M is a multiple of 128, N a multiple of 16, K a multiple of 16.
// Columns n >= n_valid of the outputs are written as 0.  err (may be null)
// receives 1 when a tensor-core wait ran out.
struct GemmArgs {
  const bf16* A;
  const bf16* B;
  int M, N, K, lda, ldb;
  const float* bias;
  float* out_f32;
  bf16* out_bf16;
  int ldc;       // leading dimension of both outputs
  int n_valid;
  int gelu;
  int* err;
};
// Computed by the TMA-fed, warp-specialised persistent kernel of k_gemm.cu
// (N <= 256; 16-byte aligned A and B); cudaErrorInvalidValue for shapes
// outside that.  gemm_tma_prepare() once per device before use.
cudaError_t launch_gemm_tma(const GemmArgs& g, cudaStream_t st);
cudaError_t gemm_tma_prepare();
// 2-D tensor map of a row-major BF16 matrix [rows][ld] read in (64 x
// box_rows) tiles of its first `cols` columns, 128-byte swizzle; elements
// outside the matrix read as zero.  Valid after gemm_tma_prepare().
bool tma_encode_bf16(CUtensorMap* map, const bf16* base, int rows, int cols, int ld, int box_rows);
int gemm_sm_count();

// The whole inference pass x -> W1 -> GELU -> W2 -> GELU -> W3 -> GELU -> W4
// in one kernel (k_mlp_fused.cu): y[m][n] = (network)(x[m]) in FP32 for M rows
// (a multiple of 128), hidden width 256; x [M][in_k] BF16; W_l row-major
// [rows][cols] BF16 (W1 [256][in_k], W2 and W3 [256][256], W4 [out_n][256]);
// bias_l FP32; in_k and out_n multiples of 16, in_k <= 64, out_n <= 256;
// 16-byte aligned pointers.  Same rounding points as the layer-by-layer
// chain (BF16 hidden activations, FP32 accumulation).
struct MlpFusedArgs {
  const bf16* x;
  int M, width, in_k, out_n;
  const bf16* w[4];
  const float* bias[4];
  float* y;
  int* err;
};
bool mlp_fused_supported(int width, int in_k, int out_n);
cudaError_t mlp_fused_prepare();
cudaError_t launch_mlp_fused(const MlpFusedArgs& a, cudaStream_t st);

// Elementwise and reduction helpers (row-major [rows][cols] unless stated).
void launch_f32_to_bf16(const float* in, bf16* out, int64_t n, cudaStream_t st);
// out[c][r] = in[r][c] for r < rows, c < cols; rows_pad / cols_pad zero padding
// of the destination ([cols_pad][rows_pad])
void launch_transpose_bf16(const bf16* in, int rows, int cols, int ld_in, bf16* out, int rows_pad, int cols_pad,
                           cudaStream_t st);
// dz = g * GELU'(z), written as BF16
void launch_gelu_backward(const float* z, const float* g, bf16* dz, int64_t n, cudaStream_t st);
// dy = scale * (y - t) on real rows / columns, 0 elsewhere (y, t, dy all
// [rows][cols_pad]); loss_part[b] = sum of (y - t)^2 of block b, blocks =
// mse_blocks(rows)
int mse_blocks(int rows);
void launch_mse_grad(const float* y, const float* t, int rows, int rows_real, int cols_pad, int cols_real,
                     float scale, bf16* dy, double* loss_part, cudaStream_t st);
// column sums of a BF16 [rows][cols] matrix into FP32 out[cols] (fixed order)
void launch_col_sum(const bf16* in, int rows, int cols, float* out, cudaStream_t st);
// AdamW on n FP32 parameters; writes the BF16 copy
void launch_adamw(float* w, const float* g, float* m, float* v, bf16* w_bf16, int64_t n, float lr, float b1,
                  float b2, float eps, float wd, float bc1, float bc2, cudaStream_t st);

// The library's bounded mbarrier wait (the one the GEMM uses) on a barrier
// phase that nothing completes: *timed_out = 1 when every thread's wait gave
// up after `limit` tries.
void launch_wait_selftest(int limit, int* timed_out, cudaStream_t st);

}  // namespace felis
