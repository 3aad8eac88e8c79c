// Host side of the taper-surrogate MLP (felis_mlp_*).
//
// Four linear layers n_in -> W -> W -> W -> n_out with GELU after the first
// three.  FP32 master parameters and AdamW state; BF16 weights and
// activations feed the tensor-core GEMMs (FP32 accumulation).  Shapes are
// padded to the GEMM's granules: inputs and outputs to multiples of 16,
// batches to multiples of 128 (padding rows and columns are zero and carry
// no loss).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <random>
#include <string>
#include <vector>

#include "../../../include/felis_b200.h"
#include "mlp.cuh"

using namespace felis;

namespace {

constexpr int kLayers = 4;
constexpr int kChunk = 65536;  // rows per device pass (a multiple of 128)
constexpr int kFwdChunk = 1 << 20;  // rows per inference pass (felis_mlp_forward)

int round_up(int v, int m) { return (v + m - 1) / m * m; }

}  // namespace

struct felis_mlp {
  int n_in = 0, width = 0, n_out = 0;
  int in_p = 0, out_p = 0, out_rows = 0;  // padded sizes; out_rows: out_p rounded to 128
  cudaStream_t st = nullptr;
  std::string err;
  int* d_err = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;  // around the inference kernels of the last forward chunk
  bool fused = false;                        // inference by the fused kernel (k_mlp_fused.cu)
  double fwd_ms = 0.0, fwd_flops = 0.0;
  // per layer: rows (outputs) x cols (inputs), padded
  int rows[kLayers], cols[kLayers], rows_real[kLayers], cols_real[kLayers];
  size_t w_off[kLayers], b_off[kLayers], n_param = 0;
  float* p = nullptr;        // FP32 master parameters (padded layout)
  float* grad = nullptr;     // gradients, same layout (W4 block has out_rows rows)
  float* m = nullptr;        // AdamW moments
  float* v = nullptr;
  bf16* wb[kLayers] = {};    // BF16 weights [rows][cols]
  bf16* wt[kLayers] = {};    // BF16 transposed weights [cols][rows] (layers 2..4)
  int64_t steps = 0;
  // activations of one chunk
  int cap = 0;
  bf16* xb = nullptr;        // [cap][in_p]
  float* xf = nullptr;       // staging for uploads [cap][max(in_p, out_p)]
  float* z[kLayers] = {};    // pre-activations [cap][rows]
  bf16* a[kLayers] = {};     // activations / outputs [cap][rows]
  float* tgt = nullptr;      // targets [cap][out_p]
  bf16* dz = nullptr;        // [cap][width]
  bf16* dzt = nullptr;       // transposed [max(width, out_rows)][cap]
  bf16* at = nullptr;        // transposed activation [max(width, in_p)][cap]
  float* da = nullptr;       // [cap][width]
  double* loss_part = nullptr;
  std::vector<double> h_part;
  // training set
  bf16* dx = nullptr;
  float* dt = nullptr;
  int64_t n_data = 0;
  int* d_idx = nullptr;
};

namespace {

#define MCK(call)                                                                    \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      m->err = std::string(#call) + ": " + cudaGetErrorString(e_);                   \
      return FELIS_CUDA_ERROR;                                                       \
    }                                                                                \
  } while (0)

felis_status mfail(felis_mlp* m, felis_status s, const std::string& e) {
  if (m) m->err = e;
  return s;
}

__global__ void k_gather_rows(const bf16* x, const float* t, const int* idx, int n, int in_p, int out_p, bf16* xb,
                              float* tb) {
  const int r = blockIdx.x;
  if (r >= n) return;
  const int64_t s = idx[r];
  for (int c = threadIdx.x; c < in_p; c += blockDim.x) xb[(size_t)r * in_p + c] = x[s * in_p + c];
  for (int c = threadIdx.x; c < out_p; c += blockDim.x) tb[(size_t)r * out_p + c] = t[s * out_p + c];
}

__global__ void k_zero_rows_bf16(bf16* x, int64_t from, int64_t to) {
  for (int64_t i = from + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < to; i += (int64_t)gridDim.x * blockDim.x)
    x[i] = __float2bfloat16_rn(0.f);
}

// Host rows [n][c_real] (FP32) -> device padded rows [n][c_pad].
felis_status upload_rows(felis_mlp* m, const float* h, int64_t n, int c_real, int c_pad, float* d) {
  std::vector<float> buf((size_t)n * c_pad, 0.f);
  for (int64_t r = 0; r < n; ++r) memcpy(&buf[(size_t)r * c_pad], h + (size_t)r * c_real, c_real * sizeof(float));
  MCK(cudaMemcpyAsync(d, buf.data(), buf.size() * sizeof(float), cudaMemcpyHostToDevice, m->st));
  MCK(cudaStreamSynchronize(m->st));
  return FELIS_OK;
}

felis_status ensure_cap(felis_mlp* m, int rows) {
  if (rows <= m->cap) return FELIS_OK;
  void** bufs[] = {(void**)&m->xb, (void**)&m->xf, (void**)&m->tgt, (void**)&m->dz, (void**)&m->dzt,
                   (void**)&m->at, (void**)&m->da, (void**)&m->loss_part};
  for (auto b : bufs) { if (*b) cudaFree(*b); *b = nullptr; }
  for (int l = 0; l < kLayers; ++l) {
    if (m->z[l]) cudaFree(m->z[l]);
    if (m->a[l]) cudaFree(m->a[l]);
    m->z[l] = nullptr;
    m->a[l] = nullptr;
  }
  m->cap = rows;
  const int wide = std::max(m->width, std::max(m->in_p, m->out_rows));
  MCK(cudaMalloc(&m->xb, (size_t)rows * m->in_p * sizeof(bf16)));
  MCK(cudaMalloc(&m->xf, (size_t)rows * std::max(m->in_p, m->out_p) * sizeof(float)));
  MCK(cudaMalloc(&m->tgt, (size_t)rows * m->out_p * sizeof(float)));
  MCK(cudaMalloc(&m->dz, (size_t)rows * m->width * sizeof(bf16)));
  MCK(cudaMalloc(&m->dzt, (size_t)wide * rows * sizeof(bf16)));
  MCK(cudaMalloc(&m->at, (size_t)wide * rows * sizeof(bf16)));
  MCK(cudaMalloc(&m->da, (size_t)rows * m->width * sizeof(float)));
  MCK(cudaMalloc(&m->loss_part, (size_t)mse_blocks(rows) * sizeof(double)));
  for (int l = 0; l < kLayers; ++l) {
    MCK(cudaMalloc(&m->z[l], (size_t)rows * m->rows[l] * sizeof(float)));
    MCK(cudaMalloc(&m->a[l], (size_t)rows * m->rows[l] * sizeof(bf16)));
  }
  m->h_part.assign(mse_blocks(rows), 0.0);
  return FELIS_OK;
}

void gemm(felis_mlp* m, const bf16* A, const bf16* B, int M, int N, int K, int lda, int ldb, const float* bias,
          float* out_f32, bf16* out_bf16, int ldc, int n_valid, int gelu) {
  GemmArgs g{A, B, M, N, K, lda, ldb, bias, out_f32, out_bf16, ldc, n_valid, gelu, m->d_err};
  if (launch_gemm_tma(g, m->st) != cudaSuccess) {
    // shapes the network never produces (M % 128, N > 256, unaligned rows):
    // reported through the error word like a device failure
    cudaMemsetAsync(m->d_err, 0xff, sizeof(int), m->st);
  }
}

// Forward pass of rows [0, M) of xb (M a multiple of 128).  Training keeps
// every layer's FP32 pre-activation z (the backward pass needs it);
// inference writes the hidden layers' BF16 activations and the last layer's
// FP32 output only.
void forward(felis_mlp* m, int M, bool keep_z = true) {
  const bf16* in = m->xb;
  int ld_in = m->in_p;
  for (int l = 0; l < kLayers; ++l) {
    const bool last = l == kLayers - 1;
    gemm(m, in, m->wb[l], M, m->rows[l], m->cols[l], ld_in, m->cols[l], m->p + m->b_off[l],
         (keep_z || last) ? m->z[l] : nullptr, (keep_z || !last) ? m->a[l] : nullptr,
         m->rows[l], m->rows_real[l], last ? 0 : 1);
    in = m->a[l];
    ld_in = m->rows[l];
  }
}

// The inference pass of rows [0, M) of xb as one fused kernel; the output
// goes where forward() leaves it (z of the last layer).
void forward_fused(felis_mlp* m, int M) {
  MlpFusedArgs a;
  a.x = m->xb;
  a.M = M; a.width = m->width; a.in_k = m->in_p; a.out_n = m->out_p;
  for (int l = 0; l < kLayers; ++l) {
    a.w[l] = m->wb[l];
    a.bias[l] = m->p + m->b_off[l];
  }
  a.y = m->z[kLayers - 1];
  a.err = m->d_err;
  if (launch_mlp_fused(a, m->st) != cudaSuccess) cudaMemsetAsync(m->d_err, 0xff, sizeof(int), m->st);
}

// Gradients of the mean squared error over the first n_real rows of the
// chunk (targets in tgt) into m->grad; returns the summed squared error.
felis_status backward(felis_mlp* m, int M, int n_real, double* sse) {
  const int L = kLayers;
  const float scale = 2.f / ((float)n_real * (float)m->n_out);
  launch_mse_grad(m->z[L - 1], m->tgt, M, n_real, m->out_p, m->n_out, scale, m->dz, m->loss_part, m->st);
  int dz_cols = m->out_p;  // current dz is [M][dz_cols]
  for (int l = L - 1; l >= 0; --l) {
    const int R = m->rows[l], Cc = m->cols[l];
    const int Rt = l == L - 1 ? m->out_rows : R;  // transposed dz rows (A operand: a multiple of 128)
    // dW = dz^T . a_{l-1}: A = dz^T [Rt][M], B = a_{l-1}^T [Cc][M]
    launch_transpose_bf16(m->dz, M, dz_cols, dz_cols, m->dzt, M, Rt, m->st);
    const bf16* prev = l == 0 ? m->xb : m->a[l - 1];
    launch_transpose_bf16(prev, M, Cc, Cc, m->at, M, Cc, m->st);
    gemm(m, m->dzt, m->at, Rt, Cc, M, M, M, nullptr, m->grad + m->w_off[l], nullptr, Cc, Cc, 0);
    launch_col_sum(m->dz, M, dz_cols, m->grad + m->b_off[l], m->st);
    if (l == 0) break;
    // da_{l-1} = dz . W_l: A = dz [M][R], B = W_l^T [Cc][R]
    gemm(m, m->dz, m->wt[l], M, Cc, R, dz_cols, R, nullptr, m->da, nullptr, Cc, Cc, 0);
    launch_gelu_backward(m->z[l - 1], m->da, m->dz, (int64_t)M * Cc, m->st);
    dz_cols = Cc;
  }
  MCK(cudaMemcpyAsync(m->h_part.data(), m->loss_part, mse_blocks(M) * sizeof(double), cudaMemcpyDeviceToHost, m->st));
  MCK(cudaStreamSynchronize(m->st));
  double s = 0.0;
  for (int b = 0; b < mse_blocks(M); ++b) s += m->h_part[b];
  *sse = s;
  return FELIS_OK;
}

felis_status refresh_bf16(felis_mlp* m) {
  for (int l = 0; l < kLayers; ++l) {
    const int64_t n = (int64_t)m->rows[l] * m->cols[l];
    launch_f32_to_bf16(m->p + m->w_off[l], m->wb[l], n, m->st);
    if (l > 0) launch_transpose_bf16(m->wb[l], m->rows[l], m->cols[l], m->cols[l], m->wt[l], m->rows[l], m->cols[l], m->st);
  }
  MCK(cudaGetLastError());
  return FELIS_OK;
}

felis_status adamw_step(felis_mlp* m, float lr, float wd) {
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  m->steps += 1;
  const float bc1 = 1.f - powf(b1, (float)m->steps), bc2 = 1.f - powf(b2, (float)m->steps);
  for (int l = 0; l < kLayers; ++l) {
    const int64_t nw = (int64_t)m->rows[l] * m->cols[l];
    launch_adamw(m->p + m->w_off[l], m->grad + m->w_off[l], m->m + m->w_off[l], m->v + m->w_off[l], m->wb[l], nw,
                 lr, b1, b2, eps, wd, bc1, bc2, m->st);
    launch_adamw(m->p + m->b_off[l], m->grad + m->b_off[l], m->m + m->b_off[l], m->v + m->b_off[l], nullptr,
                 m->rows[l], lr, b1, b2, eps, 0.f, bc1, bc2, m->st);
    if (l > 0) launch_transpose_bf16(m->wb[l], m->rows[l], m->cols[l], m->cols[l], m->wt[l], m->rows[l], m->cols[l], m->st);
  }
  MCK(cudaGetLastError());
  return FELIS_OK;
}

felis_status check_err(felis_mlp* m) {
  int e = 0;
  MCK(cudaMemcpyAsync(&e, m->d_err, sizeof(int), cudaMemcpyDeviceToHost, m->st));
  MCK(cudaStreamSynchronize(m->st));
  if (e) {
    MCK(cudaMemsetAsync(m->d_err, 0, sizeof(int), m->st));
    return mfail(m, FELIS_TIMEOUT, "tensor-core wait ran out");
  }
  return FELIS_OK;
}

// Padded parameter layout <-> flat unpadded layout W1, b1, ..., W4, b4.
int64_t flat_count(const felis_mlp* m) {
  int64_t n = 0;
  for (int l = 0; l < kLayers; ++l) n += (int64_t)m->rows_real[l] * m->cols_real[l] + m->rows_real[l];
  return n;
}

}  // namespace

extern "C" {

felis_status felis_mlp_create(int32_t n_in, int32_t width, int32_t n_out, uint64_t seed, felis_mlp** out) {
  if (!out || n_in < 1 || n_out < 1 || (width != 128 && width != 256) || n_in > 256 || n_out > width)
    return FELIS_BAD_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return FELIS_NO_DEVICE;
  felis_mlp* m = new felis_mlp();
  m->n_in = n_in; m->width = width; m->n_out = n_out;
  m->in_p = round_up(n_in, 16);
  m->out_p = round_up(n_out, 16);
  m->out_rows = round_up(m->out_p, 128);
  m->fused = mlp_fused_supported(width, m->in_p, m->out_p);
  const int r[kLayers] = {width, width, width, m->out_p};
  const int c[kLayers] = {m->in_p, width, width, width};
  const int rr[kLayers] = {width, width, width, n_out};
  const int cr[kLayers] = {n_in, width, width, width};
  size_t off = 0;
  for (int l = 0; l < kLayers; ++l) {
    m->rows[l] = r[l]; m->cols[l] = c[l]; m->rows_real[l] = rr[l]; m->cols_real[l] = cr[l];
    m->w_off[l] = off;
    // the last layer's gradient block is written as out_rows rows by the GEMM
    off += (size_t)(l == kLayers - 1 ? m->out_rows : r[l]) * c[l];
    m->b_off[l] = off;
    off += round_up(r[l], 4);
  }
  m->n_param = off;
  auto bad = [&](felis_status s, const char* msg) {
    fprintf(stderr, "felis_mlp_create: %s\n", msg);
    felis_mlp_destroy(m);
    return s;
  };
  cudaError_t e = cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaMalloc(&m->d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(m->d_err, 0, sizeof(int));
  float** fb[] = {&m->p, &m->grad, &m->m, &m->v};
  for (auto f : fb) {
    if (e == cudaSuccess) e = cudaMalloc(f, m->n_param * sizeof(float));
    if (e == cudaSuccess) e = cudaMemset(*f, 0, m->n_param * sizeof(float));
  }
  for (int l = 0; l < kLayers && e == cudaSuccess; ++l) {
    e = cudaMalloc(&m->wb[l], (size_t)r[l] * c[l] * sizeof(bf16));
    if (e == cudaSuccess) e = cudaMalloc(&m->wt[l], (size_t)r[l] * c[l] * sizeof(bf16));
  }
  if (e == cudaSuccess) e = gemm_tma_prepare();
  if (e == cudaSuccess) e = mlp_fused_prepare();
  if (e == cudaSuccess) e = cudaEventCreate(&m->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&m->ev1);
  if (e != cudaSuccess) return bad(FELIS_CUDA_ERROR, cudaGetErrorString(e));
  // He-style initialisation for GELU layers (std sqrt(2 / fan_in)), zero biases
  std::mt19937_64 rng(seed ? seed : 1);
  std::vector<float> h(m->n_param, 0.f);
  for (int l = 0; l < kLayers; ++l) {
    std::normal_distribution<float> nd(0.f, sqrtf((l == kLayers - 1 ? 1.f : 2.f) / (float)m->cols_real[l]));
    for (int i = 0; i < m->rows_real[l]; ++i)
      for (int j = 0; j < m->cols_real[l]; ++j) h[m->w_off[l] + (size_t)i * c[l] + j] = nd(rng);
  }
  e = cudaMemcpy(m->p, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return bad(FELIS_CUDA_ERROR, cudaGetErrorString(e));
  if (refresh_bf16(m) != FELIS_OK) return bad(FELIS_CUDA_ERROR, m->err.c_str());
  *out = m;
  return FELIS_OK;
}

void felis_mlp_destroy(felis_mlp* m) {
  if (!m) return;
  if (m->st) cudaStreamSynchronize(m->st);
  void* ptrs[] = {m->d_err, m->p, m->grad, m->m, m->v, m->xb, m->xf, m->tgt, m->dz, m->dzt, m->at, m->da,
                  m->loss_part, m->dx, m->dt, m->d_idx};
  for (void* q : ptrs) if (q) cudaFree(q);
  for (int l = 0; l < kLayers; ++l) {
    void* q[] = {m->wb[l], m->wt[l], m->z[l], m->a[l]};
    for (void* x : q) if (x) cudaFree(x);
  }
  if (m->ev0) cudaEventDestroy(m->ev0);
  if (m->ev1) cudaEventDestroy(m->ev1);
  if (m->st) cudaStreamDestroy(m->st);
  delete m;
}

const char* felis_mlp_last_error(const felis_mlp* m) { return m ? m->err.c_str() : "null network"; }

felis_status felis_mlp_param_count(const felis_mlp* m, int64_t* count) {
  if (!m || !count) return FELIS_BAD_ARG;
  *count = flat_count(m);
  return FELIS_OK;
}

felis_status felis_mlp_get_params(felis_mlp* m, float* out) {
  if (!m || !out) return FELIS_BAD_ARG;
  std::vector<float> h(m->n_param);
  MCK(cudaStreamSynchronize(m->st));
  MCK(cudaMemcpy(h.data(), m->p, h.size() * sizeof(float), cudaMemcpyDeviceToHost));
  int64_t k = 0;
  for (int l = 0; l < kLayers; ++l) {
    for (int i = 0; i < m->rows_real[l]; ++i)
      for (int j = 0; j < m->cols_real[l]; ++j) out[k++] = h[m->w_off[l] + (size_t)i * m->cols[l] + j];
    for (int i = 0; i < m->rows_real[l]; ++i) out[k++] = h[m->b_off[l] + i];
  }
  return FELIS_OK;
}

felis_status felis_mlp_set_params(felis_mlp* m, const float* in) {
  if (!m || !in) return FELIS_BAD_ARG;
  std::vector<float> h(m->n_param, 0.f);
  int64_t k = 0;
  for (int l = 0; l < kLayers; ++l) {
    for (int i = 0; i < m->rows_real[l]; ++i)
      for (int j = 0; j < m->cols_real[l]; ++j) h[m->w_off[l] + (size_t)i * m->cols[l] + j] = in[k++];
    for (int i = 0; i < m->rows_real[l]; ++i) h[m->b_off[l] + i] = in[k++];
  }
  MCK(cudaStreamSynchronize(m->st));
  MCK(cudaMemcpy(m->p, h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice));
  MCK(cudaMemset(m->m, 0, m->n_param * sizeof(float)));
  MCK(cudaMemset(m->v, 0, m->n_param * sizeof(float)));
  m->steps = 0;
  return refresh_bf16(m);
}

felis_status felis_mlp_forward(felis_mlp* m, const float* x, int64_t n, float* y) {
  if (!m || n < 0 || (n > 0 && (!x || !y))) return mfail(m, FELIS_BAD_ARG, "bad argument");
  felis_status s =
      ensure_cap(m, (int)std::min<int64_t>(round_up((int)std::min<int64_t>(n, kFwdChunk), 128), kFwdChunk));
  if (s != FELIS_OK) return s;
  std::vector<float> hy;
  for (int64_t r0 = 0; r0 < n; r0 += kFwdChunk) {
    const int nr = (int)std::min<int64_t>(kFwdChunk, n - r0);
    const int M = round_up(nr, 128);
    MCK(cudaMemsetAsync(m->xf, 0, (size_t)M * m->in_p * sizeof(float), m->st));
    s = upload_rows(m, x + (size_t)r0 * m->n_in, nr, m->n_in, m->in_p, m->xf);
    if (s != FELIS_OK) return s;
    launch_f32_to_bf16(m->xf, m->xb, (int64_t)M * m->in_p, m->st);
    MCK(cudaEventRecord(m->ev0, m->st));
    if (m->fused) forward_fused(m, M);
    else forward(m, M, false);
    MCK(cudaEventRecord(m->ev1, m->st));
    hy.resize((size_t)nr * m->out_p);
    MCK(cudaMemcpyAsync(hy.data(), m->z[kLayers - 1], hy.size() * sizeof(float), cudaMemcpyDeviceToHost, m->st));
    MCK(cudaStreamSynchronize(m->st));
    for (int r = 0; r < nr; ++r) memcpy(y + (size_t)(r0 + r) * m->n_out, &hy[(size_t)r * m->out_p], m->n_out * sizeof(float));
    float ms = 0.f;
    MCK(cudaEventElapsedTime(&ms, m->ev0, m->ev1));
    m->fwd_ms = ms;
    double fl = 0.0;
    for (int l = 0; l < kLayers; ++l) fl += 2.0 * M * m->rows[l] * m->cols[l];
    m->fwd_flops = fl;
  }
  return check_err(m);
}

felis_status felis_mlp_set_fused(felis_mlp* m, int32_t enable) {
  if (!m) return FELIS_BAD_ARG;
  if (enable && !mlp_fused_supported(m->width, m->in_p, m->out_p))
    return mfail(m, FELIS_UNSUPPORTED, "the fused inference kernel needs width 256, n_in <= 64, n_out <= 256");
  m->fused = enable != 0;
  return FELIS_OK;
}

felis_status felis_mlp_gradients(felis_mlp* m, const float* x, const float* t, int64_t n, float* grads,
                                 double* loss) {
  if (!m || !x || !t || n < 1 || n > kChunk) return mfail(m, FELIS_BAD_ARG, "bad argument (1 <= n <= 65536)");
  const int M = round_up((int)n, 128);
  felis_status s = ensure_cap(m, M);
  if (s != FELIS_OK) return s;
  MCK(cudaMemsetAsync(m->xf, 0, (size_t)M * m->in_p * sizeof(float), m->st));
  if ((s = upload_rows(m, x, n, m->n_in, m->in_p, m->xf)) != FELIS_OK) return s;
  launch_f32_to_bf16(m->xf, m->xb, (int64_t)M * m->in_p, m->st);
  MCK(cudaMemsetAsync(m->tgt, 0, (size_t)M * m->out_p * sizeof(float), m->st));
  if ((s = upload_rows(m, t, n, m->n_out, m->out_p, m->tgt)) != FELIS_OK) return s;
  forward(m, M);
  double sse = 0.0;
  if ((s = backward(m, M, (int)n, &sse)) != FELIS_OK) return s;
  if ((s = check_err(m)) != FELIS_OK) return s;
  std::vector<float> h(m->n_param);
  MCK(cudaMemcpy(h.data(), m->grad, h.size() * sizeof(float), cudaMemcpyDeviceToHost));
  int64_t k = 0;
  for (int l = 0; l < kLayers; ++l) {
    for (int i = 0; i < m->rows_real[l]; ++i)
      for (int j = 0; j < m->cols_real[l]; ++j) grads[k++] = h[m->w_off[l] + (size_t)i * m->cols[l] + j];
    for (int i = 0; i < m->rows_real[l]; ++i) grads[k++] = h[m->b_off[l] + i];
  }
  if (loss) *loss = sse / ((double)n * m->n_out);
  return FELIS_OK;
}

felis_status felis_mlp_set_data(felis_mlp* m, const float* x, const float* t, int64_t n) {
  if (!m || !x || !t || n < 1) return mfail(m, FELIS_BAD_ARG, "bad argument");
  if (m->dx) cudaFree(m->dx);
  if (m->dt) cudaFree(m->dt);
  if (m->d_idx) cudaFree(m->d_idx);
  m->dx = nullptr; m->dt = nullptr; m->d_idx = nullptr;
  float* tmp = nullptr;
  MCK(cudaMalloc(&m->dx, (size_t)n * m->in_p * sizeof(bf16)));
  MCK(cudaMalloc(&m->dt, (size_t)n * m->out_p * sizeof(float)));
  MCK(cudaMalloc(&m->d_idx, (size_t)n * sizeof(int)));
  MCK(cudaMalloc(&tmp, (size_t)n * m->in_p * sizeof(float)));
  felis_status s = upload_rows(m, x, n, m->n_in, m->in_p, tmp);
  if (s == FELIS_OK) {
    launch_f32_to_bf16(tmp, m->dx, n * m->in_p, m->st);
    s = upload_rows(m, t, n, m->n_out, m->out_p, m->dt);
  }
  cudaStreamSynchronize(m->st);
  cudaFree(tmp);
  m->n_data = n;
  return s;
}

felis_status felis_mlp_train(felis_mlp* m, int32_t epochs, int32_t batch, float lr, float weight_decay,
                             uint64_t seed, double* loss_per_epoch) {
  if (!m || epochs < 1 || batch < 128 || batch % 128 || batch > kChunk || m->n_data < 1)
    return mfail(m, FELIS_BAD_ARG, "bad argument (batch a multiple of 128, data set first)");
  felis_status s = ensure_cap(m, batch);
  if (s != FELIS_OK) return s;
  std::mt19937_64 rng(seed ? seed : 1);
  std::vector<int> perm(m->n_data);
  for (int64_t i = 0; i < m->n_data; ++i) perm[i] = (int)i;
  for (int ep = 0; ep < epochs; ++ep) {
    std::shuffle(perm.begin(), perm.end(), rng);
    MCK(cudaMemcpyAsync(m->d_idx, perm.data(), perm.size() * sizeof(int), cudaMemcpyHostToDevice, m->st));
    double sse = 0.0;
    for (int64_t b0 = 0; b0 < m->n_data; b0 += batch) {
      const int nr = (int)std::min<int64_t>(batch, m->n_data - b0);
      const int M = round_up(nr, 128);
      k_gather_rows<<<nr, 64, 0, m->st>>>(m->dx, m->dt, m->d_idx + b0, nr, m->in_p, m->out_p, m->xb, m->tgt);
      if (M > nr) {
        k_zero_rows_bf16<<<64, 256, 0, m->st>>>(m->xb, (int64_t)nr * m->in_p, (int64_t)M * m->in_p);
        MCK(cudaMemsetAsync(m->tgt + (size_t)nr * m->out_p, 0, (size_t)(M - nr) * m->out_p * sizeof(float), m->st));
      }
      forward(m, M);
      double part = 0.0;
      if ((s = backward(m, M, nr, &part)) != FELIS_OK) return s;
      sse += part;
      if ((s = adamw_step(m, lr, weight_decay)) != FELIS_OK) return s;
    }
    if (loss_per_epoch) loss_per_epoch[ep] = sse / ((double)m->n_data * m->n_out);
  }
  return check_err(m);
}

felis_status felis_mlp_last_forward(const felis_mlp* m, double* ms, double* flops) {
  if (!m || !ms || !flops) return FELIS_BAD_ARG;
  *ms = m->fwd_ms;
  *flops = m->fwd_flops;
  return FELIS_OK;
}

felis_status felis_wait_selftest(int32_t limit, int32_t* timed_out) {
  if (limit < 1 || !timed_out) return FELIS_BAD_ARG;
  int* d = nullptr;
  cudaError_t e = cudaMalloc(&d, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(d, 0, sizeof(int));
  if (e == cudaSuccess) {
    launch_wait_selftest(limit, d, 0);
    e = cudaGetLastError();
  }
  int h = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost);
  if (d) cudaFree(d);
  if (e != cudaSuccess) return FELIS_CUDA_ERROR;
  *timed_out = h;
  return h ? FELIS_TIMEOUT : FELIS_OK;
}

}  // extern "C"
