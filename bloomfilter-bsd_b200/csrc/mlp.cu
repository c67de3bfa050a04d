// mlp.cu -- the cost model's multilayer perceptron: forward pass, backward
// pass and Adam as hand-written FP32 kernels behind the dtlg_mlp_* C ABI.
//
// No counterpart in the reference, whose configuration choice is the
// exhaustive calibrated search (model/optimizer.hpp:25-140,
// tool/calibration/src/skyline_matrix_builder.cpp:19-276).  The network maps a
// query (log2 n, target FPR, hit ratio, downstream work, L2-residency flag) to
// per-candidate outputs: `hidden_layers` ReLU layers of `width` units and a
// linear output layer.
//
// Layout: activations are row-major [rows x units].  Layer l owns W_l
// [in x out] (W[i*out + j] connects input i to output j) followed by b_l
// [out]; all layers lie back to back in one float buffer.
// Loss: L = (1/N) sum_ij w_ij (y_ij - t_ij)^2 over a batch of N rows.
// Every reduction runs in a fixed order, so all results are deterministic.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "../../include/dtlg.h"
#include "status.hpp"

namespace {

constexpr int kTile = 64;        // GEMM tile: 64 x 64 outputs per CTA
constexpr int kTileK = 16;       // K step staged in shared memory
constexpr int kLossBlocks = 256; // fixed grid of the loss kernel (fixed reduction order)

enum Epilogue { kPlain = 0, kBiasRelu = 1, kBias = 2, kReluMask = 3 };

// C[M x N] = op(A)[M x K] * op(B)[K x N] with an epilogue.
//   op(A)[m][k] = TA ? A[k*lda + m] : A[m*lda + k]
//   op(B)[k][n] = TB ? B[n*ldb + k] : B[k*ldb + n]
//   kBiasRelu: max(C + bias[n], 0); kBias: C + bias[n];
//   kReluMask: C where mask[m*ldm + n] > 0, else 0 (ReLU derivative).
// 256 threads as 16 x 16, each owning rows ty + 16i and columns tx + 16j
// (i, j < 4); the K sum runs in order, k = 0 .. K-1.
template <bool TA, bool TB, int EPI>
__global__ void __launch_bounds__(256) mlp_gemm(int M, int N, int K, const float* __restrict__ A, int lda,
                                                const float* __restrict__ B, int ldb, float* __restrict__ C,
                                                int ldc, const float* __restrict__ bias,
                                                const float* __restrict__ mask, int ldm) {
  __shared__ float As[kTileK][kTile + 4];
  __shared__ float Bs[kTileK][kTile + 4];
  const int tid = threadIdx.x, tx = tid % 16, ty = tid / 16;
  const int m0 = blockIdx.y * kTile, n0 = blockIdx.x * kTile;
  float acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
  for (int k0 = 0; k0 < K; k0 += kTileK) {
    for (int e = tid; e < kTile * kTileK; e += 256) {
      int mm, kk;
      if (TA) {
        kk = e / kTile;
        mm = e % kTile;
      } else {
        mm = e / kTileK;
        kk = e % kTileK;
      }
      const int gm = m0 + mm, gk = k0 + kk;
      float v = 0.f;
      if (gm < M && gk < K) v = TA ? A[static_cast<size_t>(gk) * lda + gm] : A[static_cast<size_t>(gm) * lda + gk];
      As[kk][mm] = v;
    }
    for (int e = tid; e < kTile * kTileK; e += 256) {
      int nn, kk;
      if (TB) {
        nn = e / kTileK;
        kk = e % kTileK;
      } else {
        kk = e / kTile;
        nn = e % kTile;
      }
      const int gn = n0 + nn, gk = k0 + kk;
      float v = 0.f;
      if (gn < N && gk < K) v = TB ? B[static_cast<size_t>(gn) * ldb + gk] : B[static_cast<size_t>(gk) * ldb + gn];
      Bs[kk][nn] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kTileK; kk++) {
      float a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int gm = m0 + ty + 16 * i;
    if (gm >= M) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int gn = n0 + tx + 16 * j;
      if (gn >= N) continue;
      float v = acc[i][j];
      if (EPI == kBiasRelu) v = fmaxf(v + bias[gn], 0.f);
      if (EPI == kBias) v += bias[gn];
      if (EPI == kReluMask) v = mask[static_cast<size_t>(gm) * ldm + gn] > 0.f ? v : 0.f;
      C[static_cast<size_t>(gm) * ldc + gn] = v;
    }
  }
}

// dY = scale * w * (y - t); partial[block] = sum of w (y - t)^2 over the
// block's elements (grid-stride order, then a fixed tree).
__global__ void __launch_bounds__(256) mlp_loss_grad(uint32_t rows, uint32_t cols, const float* __restrict__ Y,
                                                     const float* __restrict__ T, const float* __restrict__ W,
                                                     float* __restrict__ dY, float* __restrict__ partial,
                                                     float scale) {
  __shared__ float s[256];
  float acc = 0.f;
  const size_t total = static_cast<size_t>(rows) * cols;
  for (size_t i = blockIdx.x * 256ull + threadIdx.x; i < total; i += static_cast<size_t>(gridDim.x) * 256) {
    const float d = Y[i] - T[i];
    const float w = W[i];
    acc = fmaf(w * d, d, acc);
    dY[i] = scale * w * d;
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

__global__ void mlp_loss_sum(const float* __restrict__ partial, int n, float inv_rows, float* __restrict__ out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    float s = 0.f;
    for (int i = 0; i < n; i++) s += partial[i];
    *out = s * inv_rows;
  }
}

// out[j] = sum_i A[i][j], i in order.
__global__ void __launch_bounds__(128) mlp_colsum(uint32_t rows, uint32_t cols, const float* __restrict__ A,
                                                  float* __restrict__ out) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= cols) return;
  float s = 0.f;
  for (uint32_t i = 0; i < rows; i++) s += A[static_cast<size_t>(i) * cols + j];
  out[j] = s;
}

// Adam (Kingma & Ba, 2015) with bias corrections bc1 = 1 - b1^t, bc2 = 1 - b2^t.
__global__ void __launch_bounds__(256) mlp_adam(uint32_t n, float* __restrict__ p, const float* __restrict__ g,
                                                float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                                                float b2, float eps, float bc1, float bc2) {
  const uint32_t i = blockIdx.x * 256 + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
}

// dst[r][c] = src[idx[r]][c]; rows whose index is out of range read zeros.
__global__ void __launch_bounds__(256) mlp_gather(uint32_t rows, const uint32_t* __restrict__ idx, uint32_t n_src,
                                                  const float* __restrict__ src, uint32_t width,
                                                  float* __restrict__ dst) {
  const size_t total = static_cast<size_t>(rows) * width;
  for (size_t e = blockIdx.x * 256ull + threadIdx.x; e < total; e += static_cast<size_t>(gridDim.x) * 256) {
    const uint32_t r = static_cast<uint32_t>(e / width), c = static_cast<uint32_t>(e % width);
    const uint32_t s = idx[r];
    dst[e] = s < n_src ? src[static_cast<size_t>(s) * width + c] : 0.f;
  }
}

// One warp per row: the smallest of the first n_cand outputs (NaN counts as
// +inf; ties go to the lower index).  aux = output n_cand + choice, if present.
__global__ void __launch_bounds__(256) mlp_argmin(uint32_t rows, uint32_t cols, uint32_t n_cand,
                                                  const float* __restrict__ Y, int32_t* __restrict__ choice,
                                                  float* __restrict__ aux) {
  const uint32_t row = (blockIdx.x * 256 + threadIdx.x) / 32, lane = threadIdx.x % 32;
  if (row >= rows) return;
  const float* y = Y + static_cast<size_t>(row) * cols;
  float best = INFINITY;
  int bi = 0x7fffffff;
  for (uint32_t j = lane; j < n_cand; j += 32) {
    float v = y[j];
    if (v != v) v = INFINITY;
    if (v < best || (v == best && static_cast<int>(j) < bi)) {
      best = v;
      bi = static_cast<int>(j);
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ov < best || (ov == best && oi < bi)) {
      best = ov;
      bi = oi;
    }
  }
  if (lane == 0) {
    if (bi == 0x7fffffff) bi = 0;
    choice[row] = bi;
    if (aux) aux[row] = (n_cand + bi < cols) ? y[n_cand + bi] : 0.f;
  }
}

struct DeviceGuard {
  int prev = -1;
  cudaError_t err = cudaSuccess;
  explicit DeviceGuard(int dev) {
    err = cudaGetDevice(&prev);
    if (err == cudaSuccess && prev != dev) err = cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

struct dtlg_mlp {
  int device = 0;
  std::vector<uint32_t> dims;   // n_in, width x hidden_layers, n_out
  std::vector<size_t> w_off, b_off;
  size_t n_params = 0;
  uint32_t max_batch = 0;
  float* params = nullptr;
  float* grads = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  std::vector<float*> act;      // act[l]: output of layer l (max_batch x dims[l+1])
  std::vector<float*> dact;     // dact[l]: loss gradient w.r.t. act[l]
  float* xb = nullptr;          // gathered training batch
  float* tb = nullptr;
  float* wb = nullptr;
  float* partial = nullptr;     // kLossBlocks loss partials
  float* loss = nullptr;        // scratch loss value
  uint64_t adam_t = 0;

  int layers() const { return static_cast<int>(dims.size()) - 1; }
  uint32_t n_in() const { return dims.front(); }
  uint32_t n_out() const { return dims.back(); }

  ~dtlg_mlp() {
    DeviceGuard g(device);
    for (float* p : {params, grads, adam_m, adam_v, xb, tb, wb, partial, loss}) cudaFree(p);
    for (float* p : act) cudaFree(p);
    for (float* p : dact) cudaFree(p);
  }
};

namespace {

dim3 gemm_grid(int M, int N) { return dim3((N + kTile - 1) / kTile, (M + kTile - 1) / kTile); }

// Forward over n <= max_batch rows; the last layer writes to y (or act.back()).
void forward(dtlg_mlp* m, const float* x, uint32_t n, float* y, cudaStream_t s) {
  const float* in = x;
  const int L = m->layers();
  for (int l = 0; l < L; l++) {
    const int K = m->dims[l], N = m->dims[l + 1];
    const float* W = m->params + m->w_off[l];
    const float* b = m->params + m->b_off[l];
    float* out = (l == L - 1 && y) ? y : m->act[l];
    if (l < L - 1) {
      mlp_gemm<false, false, kBiasRelu><<<gemm_grid(n, N), 256, 0, s>>>(n, N, K, in, K, W, N, out, N, b, nullptr, 0);
    } else {
      mlp_gemm<false, false, kBias><<<gemm_grid(n, N), 256, 0, s>>>(n, N, K, in, K, W, N, out, N, b, nullptr, 0);
    }
    in = out;
  }
}

// Loss and gradients of one batch (x, t, w of n <= max_batch rows).
void loss_and_grads(dtlg_mlp* m, const float* x, const float* t, const float* w, uint32_t n, float* loss_out,
                    cudaStream_t s) {
  const int L = m->layers();
  forward(m, x, n, nullptr, s);
  mlp_loss_grad<<<kLossBlocks, 256, 0, s>>>(n, m->n_out(), m->act[L - 1], t, w, m->dact[L - 1], m->partial,
                                            2.f / static_cast<float>(n));
  mlp_loss_sum<<<1, 32, 0, s>>>(m->partial, kLossBlocks, 1.f / static_cast<float>(n), loss_out);
  for (int l = L - 1; l >= 0; l--) {
    const int in_w = m->dims[l], out_w = m->dims[l + 1];
    const float* in = l == 0 ? x : m->act[l - 1];
    float* gW = m->grads + m->w_off[l];
    float* gb = m->grads + m->b_off[l];
    // dW_l = in^T dact[l]     [in_w x out_w], K = n
    mlp_gemm<true, false, kPlain><<<gemm_grid(in_w, out_w), 256, 0, s>>>(in_w, out_w, n, in, in_w, m->dact[l],
                                                                         out_w, gW, out_w, nullptr, nullptr, 0);
    mlp_colsum<<<(out_w + 127) / 128, 128, 0, s>>>(n, out_w, m->dact[l], gb);
    if (l > 0) {
      // dact[l-1] = (dact[l] W_l^T) * [act[l-1] > 0]
      const float* W = m->params + m->w_off[l];
      mlp_gemm<false, true, kReluMask><<<gemm_grid(n, in_w), 256, 0, s>>>(n, in_w, out_w, m->dact[l], out_w, W,
                                                                          out_w, m->dact[l - 1], in_w, nullptr,
                                                                          m->act[l - 1], in_w);
    }
  }
}

void adam_step(dtlg_mlp* m, float lr, float b1, float b2, float eps, cudaStream_t s) {
  m->adam_t++;
  const double t = static_cast<double>(m->adam_t);
  const float bc1 = static_cast<float>(1.0 - std::pow(static_cast<double>(b1), t));
  const float bc2 = static_cast<float>(1.0 - std::pow(static_cast<double>(b2), t));
  const uint32_t n = static_cast<uint32_t>(m->n_params);
  mlp_adam<<<(n + 255) / 256, 256, 0, s>>>(n, m->params, m->grads, m->adam_m, m->adam_v, lr, b1, b2, eps, bc1,
                                           bc2);
}

dtlg_status alloc(float** p, size_t count) {
  DTLG_TRY_CUDA(cudaMalloc(p, sizeof(float) * (count ? count : 1)));
  DTLG_TRY_CUDA(cudaMemset(*p, 0, sizeof(float) * (count ? count : 1)));
  return DTLG_OK;
}

}  // namespace

extern "C" {

dtlg_status dtlg_mlp_create(uint32_t n_in, uint32_t width, uint32_t hidden_layers, uint32_t n_out,
                            uint32_t max_batch, dtlg_mlp** out) {
  if (!out) return DTLG_ERR_NULL;
  *out = nullptr;
  if (!n_in || !width || !hidden_layers || !n_out || !max_batch || n_in > 4096 || width > 4096 || n_out > 65536 ||
      hidden_layers > 16 || max_batch > (1u << 20))
    return DTLG_ERR_INVALID_CONFIG;
  int device = 0;
  DTLG_TRY_CUDA(cudaGetDevice(&device));
  auto* m = new dtlg_mlp();
  m->device = device;
  m->dims.push_back(n_in);
  for (uint32_t i = 0; i < hidden_layers; i++) m->dims.push_back(width);
  m->dims.push_back(n_out);
  m->max_batch = max_batch;
  size_t off = 0;
  for (int l = 0; l < m->layers(); l++) {
    m->w_off.push_back(off);
    off += static_cast<size_t>(m->dims[l]) * m->dims[l + 1];
    m->b_off.push_back(off);
    off += m->dims[l + 1];
  }
  m->n_params = off;
  dtlg_status st = DTLG_OK;
  for (float** p : {&m->params, &m->grads, &m->adam_m, &m->adam_v})
    if (st == DTLG_OK) st = alloc(p, m->n_params);
  m->act.assign(m->layers(), nullptr);
  m->dact.assign(m->layers(), nullptr);
  for (int l = 0; l < m->layers() && st == DTLG_OK; l++) {
    st = alloc(&m->act[l], static_cast<size_t>(max_batch) * m->dims[l + 1]);
    if (st == DTLG_OK) st = alloc(&m->dact[l], static_cast<size_t>(max_batch) * m->dims[l + 1]);
  }
  if (st == DTLG_OK) st = alloc(&m->xb, static_cast<size_t>(max_batch) * n_in);
  if (st == DTLG_OK) st = alloc(&m->tb, static_cast<size_t>(max_batch) * n_out);
  if (st == DTLG_OK) st = alloc(&m->wb, static_cast<size_t>(max_batch) * n_out);
  if (st == DTLG_OK) st = alloc(&m->partial, kLossBlocks);
  if (st == DTLG_OK) st = alloc(&m->loss, 1);
  if (st != DTLG_OK) {
    delete m;
    return st;
  }
  *out = m;
  return DTLG_OK;
}

void dtlg_mlp_destroy(dtlg_mlp* m) { delete m; }

uint64_t dtlg_mlp_param_count(const dtlg_mlp* m) { return m ? m->n_params : 0; }

dtlg_status dtlg_mlp_set_params(dtlg_mlp* m, const float* params_host) {
  if (!m || !params_host) return DTLG_ERR_NULL;
  DeviceGuard g(m->device);
  DTLG_TRY_CUDA(g.err);
  DTLG_TRY_CUDA(cudaMemcpy(m->params, params_host, sizeof(float) * m->n_params, cudaMemcpyHostToDevice));
  DTLG_TRY_CUDA(cudaMemset(m->adam_m, 0, sizeof(float) * m->n_params));
  DTLG_TRY_CUDA(cudaMemset(m->adam_v, 0, sizeof(float) * m->n_params));
  m->adam_t = 0;
  return DTLG_OK;
}

dtlg_status dtlg_mlp_get_params(const dtlg_mlp* m, float* params_host) {
  if (!m || !params_host) return DTLG_ERR_NULL;
  DeviceGuard g(m->device);
  DTLG_TRY_CUDA(g.err);
  DTLG_TRY_CUDA(cudaMemcpy(params_host, m->params, sizeof(float) * m->n_params, cudaMemcpyDeviceToHost));
  return DTLG_OK;
}

dtlg_status dtlg_mlp_get_grads(const dtlg_mlp* m, float* grads_host) {
  if (!m || !grads_host) return DTLG_ERR_NULL;
  DeviceGuard g(m->device);
  DTLG_TRY_CUDA(g.err);
  DTLG_TRY_CUDA(cudaMemcpy(grads_host, m->grads, sizeof(float) * m->n_params, cudaMemcpyDeviceToHost));
  return DTLG_OK;
}

dtlg_status dtlg_mlp_forward(dtlg_mlp* m, const float* x, uint32_t n, float* y, dtlg_stream_t stream) {
  if (!m || (n && (!x || !y))) return DTLG_ERR_NULL;
  DeviceGuard g(m->device);
  DTLG_TRY_CUDA(g.err);
  auto s = reinterpret_cast<cudaStream_t>(stream);
  for (uint32_t r = 0; r < n; r += m->max_batch) {
    const uint32_t c = n - r < m->max_batch ? n - r : m->max_batch;
    forward(m, x + static_cast<size_t>(r) * m->n_in(), c, y + static_cast<size_t>(r) * m->n_out(), s);
  }
  DTLG_TRY_CUDA(cudaGetLastError());
  return DTLG_OK;
}

dtlg_status dtlg_mlp_loss_grad(dtlg_mlp* m, const float* x, const float* t, const float* w, uint32_t n,
                               float* loss, dtlg_stream_t stream) {
  if (!m || !x || !t || !w || !loss) return DTLG_ERR_NULL;
  if (n == 0 || n > m->max_batch) return DTLG_ERR_WORKSPACE;
  DeviceGuard g(m->device);
  DTLG_TRY_CUDA(g.err);
  loss_and_grads(m, x, t, w, n, loss, reinterpret_cast<cudaStream_t>(stream));
  DTLG_TRY_CUDA(cudaGetLastError());
  return DTLG_OK;
}

dtlg_status dtlg_mlp_adam_step(dtlg_mlp* m, float lr, float beta1, float beta2, float eps, dtlg_stream_t stream) {
  if (!m) return DTLG_ERR_NULL;
  DeviceGuard g(m->device);
  DTLG_TRY_CUDA(g.err);
  adam_step(m, lr, beta1, beta2, eps, reinterpret_cast<cudaStream_t>(stream));
  DTLG_TRY_CUDA(cudaGetLastError());
  return DTLG_OK;
}

dtlg_status dtlg_mlp_train(dtlg_mlp* m, const float* x, const float* t, const float* w, uint32_t n_rows,
                           const uint32_t* batch_rows, uint32_t batch, uint32_t steps, float lr_start,
                           float lr_end, float* loss_curve, dtlg_stream_t stream) {
  if (!m || !x || !t || !w || !batch_rows || !loss_curve) return DTLG_ERR_NULL;
  if (batch == 0 || batch > m->max_batch || n_rows == 0) return DTLG_ERR_WORKSPACE;
  DeviceGuard g(m->device);
  DTLG_TRY_CUDA(g.err);
  auto s = reinterpret_cast<cudaStream_t>(stream);
  const unsigned gblocks = 296;
  for (uint32_t step = 0; step < steps; step++) {
    const uint32_t* rows = batch_rows + static_cast<size_t>(step) * batch;
    mlp_gather<<<gblocks, 256, 0, s>>>(batch, rows, n_rows, x, m->n_in(), m->xb);
    mlp_gather<<<gblocks, 256, 0, s>>>(batch, rows, n_rows, t, m->n_out(), m->tb);
    mlp_gather<<<gblocks, 256, 0, s>>>(batch, rows, n_rows, w, m->n_out(), m->wb);
    loss_and_grads(m, m->xb, m->tb, m->wb, batch, loss_curve + step, s);
    // cosine decay from lr_start to lr_end
    const double frac = steps > 1 ? static_cast<double>(step) / (steps - 1) : 0.0;
    const float lr = static_cast<float>(lr_end + 0.5 * (lr_start - lr_end) * (1.0 + std::cos(M_PI * frac)));
    adam_step(m, lr, 0.9f, 0.999f, 1e-8f, s);
  }
  DTLG_TRY_CUDA(cudaGetLastError());
  return DTLG_OK;
}

dtlg_status dtlg_mlp_choose(dtlg_mlp* m, const float* x, uint32_t n, uint32_t n_cand, float* y_scratch,
                            int32_t* choice, float* aux, dtlg_stream_t stream) {
  if (!m || (n && (!x || !y_scratch || !choice))) return DTLG_ERR_NULL;
  if (n_cand == 0 || n_cand > m->n_out()) return DTLG_ERR_INVALID_CONFIG;
  dtlg_status st = dtlg_mlp_forward(m, x, n, y_scratch, stream);
  if (st != DTLG_OK || n == 0) return st;
  DeviceGuard g(m->device);
  DTLG_TRY_CUDA(g.err);
  mlp_argmin<<<(n * 32 + 255) / 256, 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(n, m->n_out(), n_cand,
                                                                                       y_scratch, choice, aux);
  DTLG_TRY_CUDA(cudaGetLastError());
  return DTLG_OK;
}

}  // extern "C"
