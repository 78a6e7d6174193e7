// Surrogate network for VCA: a multilayer perceptron n_in -> W -> W -> W -> 1
// with GELU activations, trained by Adam on data this solver generates
// (Potthoff functional values at points of the variational parameters).
//
// Arithmetic: weights and activations enter the matrix products in BF16 on
// the tensor cores with FP32 accumulation; biases, pre-activations, gradients,
// the loss and Adam's master weights and moments are FP32. Every matrix
// product is one kernel of 16 x 16 x 16 BF16 tensor-core tiles (one warp per
// 32 x 32 output tile); sizes are padded to multiples of 16 (the input width
// to 16 with zero columns).
//
// One training step (forward, backward, Adam) is a fixed sequence of kernels
// on the network's stream; the steps of an epoch are captured once into a
// CUDA graph and replayed, the epoch's shuffled data being gathered into the
// same device buffers before each replay.
#include <cuda_bf16.h>
#include <mma.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <type_traits>
#include <vector>

#include "common.hpp"
#include "qed_b200.h"

using namespace nvcuda;
typedef __nv_bfloat16 bf16;

namespace qed {
namespace {

constexpr int kTile = 16;
constexpr int kGemmWarps = 4;  // a CTA: 2 x 2 warps, 64 x 64 outputs

inline int pad16(int x) { return (x + 15) / 16 * 16; }

// C[M x N] (fp32, row-major, ldc) (+)= op(A) op(B), op(A) M x K, op(B) K x N.
// TA: A stored K x M (A^T row-major), else M x K row-major. TB: B stored N x K,
// else K x N row-major. M, N, K multiples of 16; leading dimensions multiples of 16.
template <bool TA, bool TB>
__global__ void __launch_bounds__(kGemmWarps * 32) k_mlp_gemm(int M, int N, int K, const bf16 *__restrict__ A,
                                                               int lda, const bf16 *__restrict__ B, int ldb,
                                                               float *__restrict__ C, int ldc, int accumulate) {
  using LA = typename std::conditional<TA, wmma::col_major, wmma::row_major>::type;
  using LB = typename std::conditional<TB, wmma::col_major, wmma::row_major>::type;
  const int warp = threadIdx.x / 32;
  const int m0 = (blockIdx.y * 2 + warp / 2) * 32, n0 = (blockIdx.x * 2 + warp % 2) * 32;
  if (m0 >= M || n0 >= N) return;
  wmma::fragment<wmma::accumulator, 16, 16, 16, float> acc[2][2];
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) {
      const int mi = m0 + 16 * i, nj = n0 + 16 * j;
      if (accumulate && mi < M && nj < N)
        wmma::load_matrix_sync(acc[i][j], C + (size_t)mi * ldc + nj, ldc, wmma::mem_row_major);
      else
        wmma::fill_fragment(acc[i][j], 0.0f);
    }
  for (int k0 = 0; k0 < K; k0 += kTile) {
    wmma::fragment<wmma::matrix_a, 16, 16, 16, bf16, LA> a[2];
    wmma::fragment<wmma::matrix_b, 16, 16, 16, bf16, LB> b[2];
    for (int i = 0; i < 2; ++i) {
      const int mi = m0 + 16 * i;
      if (mi < M) wmma::load_matrix_sync(a[i], TA ? A + (size_t)k0 * lda + mi : A + (size_t)mi * lda + k0, lda);
    }
    for (int j = 0; j < 2; ++j) {
      const int nj = n0 + 16 * j;
      if (nj < N) wmma::load_matrix_sync(b[j], TB ? B + (size_t)nj * ldb + k0 : B + (size_t)k0 * ldb + nj, ldb);
    }
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j)
        if (m0 + 16 * i < M && n0 + 16 * j < N) wmma::mma_sync(acc[i][j], a[i], b[j], acc[i][j]);
  }
  for (int i = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j) {
      const int mi = m0 + 16 * i, nj = n0 + 16 * j;
      if (mi < M && nj < N) wmma::store_matrix_sync(C + (size_t)mi * ldc + nj, acc[i][j], ldc, wmma::mem_row_major);
    }
}

template <bool TA, bool TB>
void gemm(int M, int N, int K, const bf16 *A, int lda, const bf16 *B, int ldb, float *C, int ldc, bool acc,
          cudaStream_t s) {
  dim3 grid((N + 63) / 64, (M + 63) / 64);
  k_mlp_gemm<TA, TB><<<grid, kGemmWarps * 32, 0, s>>>(M, N, K, A, lda, B, ldb, C, ldc, acc ? 1 : 0);
  QED_LAUNCH();
}

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// Z[b][f] += bias[f]; H = bf16(GELU(Z))
__global__ void k_bias_gelu(int rows, int F, float *Z, const float *bias, bf16 *H) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)rows * F; t += (size_t)gridDim.x * blockDim.x) {
    const float z = Z[t] + bias[t % F];
    Z[t] = z;
    H[t] = __float2bfloat16_rn(gelu(z));
  }
}

// y[b] = sum_k H[b][k] w[k] + b0 (fp32 accumulation), one warp per row
__global__ void k_head(int rows, int F, const bf16 *H, const bf16 *w, const float *b0, float *y) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32, lane = threadIdx.x % 32;
  if (warp >= rows) return;
  float s = 0.0f;
  for (int k = lane; k < F; k += 32) s += __bfloat162float(H[(size_t)warp * F + k]) * __bfloat162float(w[k]);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) y[warp] = s + b0[0];
}

// dy = 2 (y - t) / n and the loss terms (y - t)^2 / n per row
__global__ void k_mse(int rows, const float *y, const float *t, float *dy, float *loss_terms) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= rows) return;
  const float d = y[i] - t[i];
  dy[i] = 2.0f * d / rows;
  loss_terms[i] = d * d / rows;
}

// head backward: dZ[b][k] = dy[b] w[k] GELU'(Z[b][k]) (fp32 and bf16 copies)
__global__ void k_head_back(int rows, int F, const float *dy, const bf16 *w, const float *Z, float *dZ, bf16 *dZh) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)rows * F; t += (size_t)gridDim.x * blockDim.x) {
    const float g = dy[t / F] * __bfloat162float(w[t % F]) * gelu_grad(Z[t]);
    dZ[t] = g;
    dZh[t] = __float2bfloat16_rn(g);
  }
}

// dZ = dH GELU'(Z) in place (fp32) plus a bf16 copy
__global__ void k_gelu_back(int rows, int F, float *dH, const float *Z, bf16 *dZh) {
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < (size_t)rows * F; t += (size_t)gridDim.x * blockDim.x) {
    const float g = dH[t] * gelu_grad(Z[t]);
    dH[t] = g;
    dZh[t] = __float2bfloat16_rn(g);
  }
}

// out[f] = sum_b X[b][f] * (wrow ? wrow[b] : 1), fixed order, one thread per column
__global__ void k_colsum(int rows, int F, const float *X, const float *wrow, float *out) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= F) return;
  float s = 0.0f;
  for (int b = 0; b < rows; ++b) s += X[(size_t)b * F + f] * (wrow ? wrow[b] : 1.0f);
  out[f] = s;
}

// head weight gradient: g[k] = sum_b dy[b] H[b][k]
__global__ void k_head_wgrad(int rows, int F, const float *dy, const bf16 *H, float *g) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= F) return;
  float s = 0.0f;
  for (int b = 0; b < rows; ++b) s += dy[b] * __bfloat162float(H[(size_t)b * F + k]);
  g[k] = s;
}

// Adam (Kingma & Ba 2015, Algorithm 1) on fp32 master weights; the step count
// lives on the device so that a captured step can be replayed.
__global__ void k_adam(int n, float *w, const float *g, float *m, float *v, bf16 *wh, const int *step, float lr,
                       float b1, float b2, float eps, const unsigned char *mask) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (mask && !mask[i]) return;  // padding stays zero
  const int t = *step;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.0f - b1) * gi;
  const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float mh = mi / (1.0f - powf(b1, (float)t)), vh = vi / (1.0f - powf(b2, (float)t));
  const float wi = w[i] - lr * mh / (sqrtf(vh) + eps);
  w[i] = wi;
  if (wh) wh[i] = __float2bfloat16_rn(wi);
}

__global__ void k_incr(int *step) { *step += 1; }

__global__ void k_to_bf16(int n, const float *x, bf16 *y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16_rn(x[i]);
}

// gather rows (and pad the input width with zeros): X[b][0..n_in) -> Xp[b][0..ld)
__global__ void k_gather(int rows, int n_in, int ld, const float *X, const float *T, const int *perm, bf16 *Xp,
                         float *Tp) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= rows) return;
  const int src = perm ? perm[b] : b;
  for (int j = 0; j < ld; ++j) Xp[(size_t)b * ld + j] = __float2bfloat16_rn(j < n_in ? X[(size_t)src * n_in + j] : 0.0f);
  if (T) Tp[b] = T[src];
}

inline int blocks_for(size_t n, int threads = 256) {
  size_t g = (n + threads - 1) / threads;
  return (int)std::min<size_t>(std::max<size_t>(g, 1), 148 * 16);
}

}  // namespace

// ------------------------------------------------------------------ network --

struct MLP {
  int n_in = 0, k_in = 0, W = 0, L = 3;  // L hidden layers of width W
  cudaStream_t s = nullptr;
  // parameters (fp32 master) in one buffer: W1 [W][k_in], b1 [W], W2 [W][W], b2, W3 [W][W], b3, w4 [W], b4 [1]
  std::vector<size_t> off;  // offsets of the 8 parameter blocks
  size_t n_par = 0;
  DevBuf<float> p, g, m, v;
  DevBuf<bf16> ph;              // bf16 copy for the products
  DevBuf<unsigned char> mask;   // 0 on the input-width padding of W1
  DevBuf<int> step;
  // activations for a batch of `cap` rows
  int cap = 0;
  DevBuf<bf16> X, H[3], dZh[3];
  DevBuf<float> T, Z[3], dZ[3], y, dy, lt;
  DevBuf<float> tmp;
  DevBuf<int> perm;
  DevBuf<float> data_x, data_t;
  int n_data = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int graph_batch = 0, graph_steps = 0;
  float graph_lr = 0.0f;

  ~MLP() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }

  float *P(int i) { return p.p + off[i]; }
  bf16 *Ph(int i) { return ph.p + off[i]; }
  float *Gr(int i) { return g.p + off[i]; }

  void init(int nin, int width, uint64_t seed) {
    if (nin < 1 || nin > 16) fail(QED_ERR_ARGUMENT, "mlp: input width must be in [1, 16]");
    if (width < 16 || width % 16) fail(QED_ERR_ARGUMENT, "mlp: hidden width must be a positive multiple of 16");
    n_in = nin;
    k_in = pad16(nin);
    W = width;
    QED_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    const size_t sizes[8] = {(size_t)W * k_in, (size_t)W, (size_t)W * W, (size_t)W, (size_t)W * W, (size_t)W,
                             (size_t)W, 16};
    off.resize(8);
    size_t o = 0;
    for (int i = 0; i < 8; ++i) {
      off[i] = o;
      o += (sizes[i] + 15) / 16 * 16;  // 32-byte aligned blocks for the bf16 tiles
    }
    n_par = o;
    // He-style uniform init for the weights, zero biases (seeded)
    std::vector<float> h(n_par, 0.0f);
    std::vector<unsigned char> mk(n_par, 1);
    std::mt19937_64 rng(seed);
    auto fill = [&](int blk, int rows, int cols, int fan_in, int ld) {
      std::uniform_real_distribution<float> U(-1.0f, 1.0f);
      const float a = std::sqrt(3.0f / (float)fan_in);
      for (int r = 0; r < rows; ++r)
        for (int c = 0; c < ld; ++c) {
          const size_t i = off[blk] + (size_t)r * ld + c;
          if (c < cols) h[i] = a * U(rng);
          else mk[i] = 0;
        }
    };
    fill(0, W, n_in, n_in, k_in);
    fill(2, W, W, W, W);
    fill(4, W, W, W, W);
    fill(6, 1, W, W, W);
    for (size_t i = off[7] + 1; i < n_par; ++i) mk[i] = 0;
    p.alloc(n_par);
    g.alloc(n_par);
    m.alloc(n_par);
    v.alloc(n_par);
    ph.alloc(n_par);
    mask.alloc(n_par);
    step.alloc(1);
    QED_CUDA(cudaMemcpyAsync(p.p, h.data(), n_par * sizeof(float), cudaMemcpyHostToDevice, s));
    QED_CUDA(cudaMemcpyAsync(mask.p, mk.data(), n_par, cudaMemcpyHostToDevice, s));
    QED_CUDA(cudaMemsetAsync(g.p, 0, n_par * sizeof(float), s));
    QED_CUDA(cudaMemsetAsync(m.p, 0, n_par * sizeof(float), s));
    QED_CUDA(cudaMemsetAsync(v.p, 0, n_par * sizeof(float), s));
    QED_CUDA(cudaMemsetAsync(step.p, 0, sizeof(int), s));
    sync_bf16();
  }

  void sync_bf16() {
    k_to_bf16<<<blocks_for(n_par), 256, 0, s>>>((int)n_par, p.p, ph.p);
    QED_LAUNCH();
    QED_CUDA(cudaStreamSynchronize(s));
  }

  void reserve(int rows) {
    rows = pad16(rows);
    if (rows <= cap) return;
    if (exec) {
      cudaGraphExecDestroy(exec);
      exec = nullptr;
    }
    if (graph) {
      cudaGraphDestroy(graph);
      graph = nullptr;
    }
    cap = rows;
    X.alloc((size_t)cap * k_in);
    T.alloc(cap);
    for (int l = 0; l < 3; ++l) {
      H[l].alloc((size_t)cap * W);
      dZh[l].alloc((size_t)cap * W);
      Z[l].alloc((size_t)cap * W);
      dZ[l].alloc((size_t)cap * W);
    }
    y.alloc(cap);
    dy.alloc(cap);
    lt.alloc(cap);
    tmp.alloc((size_t)cap * 16);
  }

  // forward on rows [0, rows) of X (bf16, padded); y = network output
  void forward(int rows) {
    const bf16 *in = X.p;
    int kin = k_in;
    for (int l = 0; l < 3; ++l) {
      gemm<false, true>(rows, W, kin, in, kin, Ph(2 * l), kin, Z[l].p, W, false, s);
      k_bias_gelu<<<blocks_for((size_t)rows * W), 256, 0, s>>>(rows, W, Z[l].p, P(2 * l + 1), H[l].p);
      QED_LAUNCH();
      in = H[l].p;
      kin = W;
    }
    k_head<<<(rows * 32 + 255) / 256, 256, 0, s>>>(rows, W, H[2].p, Ph(6), P(7), y.p);
    QED_LAUNCH();
  }

  // gradients of the mean squared error over rows [0, rows) into g
  void backward(int rows) {
    k_mse<<<(rows + 255) / 256, 256, 0, s>>>(rows, y.p, T.p, dy.p, lt.p);
    QED_LAUNCH();
    k_head_wgrad<<<(W + 255) / 256, 256, 0, s>>>(rows, W, dy.p, H[2].p, Gr(6));
    QED_LAUNCH();
    k_colsum<<<1, 32, 0, s>>>(rows, 1, dy.p, nullptr, Gr(7));
    QED_LAUNCH();
    k_head_back<<<blocks_for((size_t)rows * W), 256, 0, s>>>(rows, W, dy.p, Ph(6), Z[2].p, dZ[2].p, dZh[2].p);
    QED_LAUNCH();
    for (int l = 2; l >= 0; --l) {
      const bf16 *prev = l > 0 ? H[l - 1].p : X.p;
      const int kin = l > 0 ? W : k_in;
      // dW_l [W][kin] = dZ_l^T prev ; db_l = column sums of dZ_l
      gemm<true, false>(W, kin, rows, dZh[l].p, W, prev, kin, Gr(2 * l), kin, false, s);
      k_colsum<<<(W + 255) / 256, 256, 0, s>>>(rows, W, dZ[l].p, nullptr, Gr(2 * l + 1));
      QED_LAUNCH();
      if (l > 0) {  // dH_{l-1} = dZ_l W_l, then through GELU'
        gemm<false, false>(rows, W, W, dZh[l].p, W, Ph(2 * l), W, dZ[l - 1].p, W, false, s);
        k_gelu_back<<<blocks_for((size_t)rows * W), 256, 0, s>>>(rows, W, dZ[l - 1].p, Z[l - 1].p, dZh[l - 1].p);
        QED_LAUNCH();
      }
    }
  }

  void adam(float lr) {
    k_incr<<<1, 1, 0, s>>>(step.p);
    QED_LAUNCH();
    k_adam<<<blocks_for(n_par), 256, 0, s>>>((int)n_par, p.p, g.p, m.p, v.p, ph.p, step.p, lr, 0.9f, 0.999f,
                                              1e-8f, mask.p);
    QED_LAUNCH();
  }

  void load_rows(int rows, const float *hx, const float *ht) {
    reserve(rows);
    DevBuf<float> dx((size_t)rows * n_in), dt(ht ? rows : 1);
    dx.upload(hx, (size_t)rows * n_in, s);
    if (ht) dt.upload(ht, rows, s);
    k_gather<<<(rows + 255) / 256, 256, 0, s>>>(rows, n_in, k_in, dx.p, ht ? dt.p : nullptr, nullptr, X.p, T.p);
    QED_LAUNCH();
    QED_CUDA(cudaStreamSynchronize(s));
  }
};

}  // namespace qed

using qed::MLP;

namespace {
thread_local std::string t_mlp_err;

template <class F> int mlp_guarded(F &&f) {
  try {
    f();
    return QED_OK;
  } catch (const qed::Error &e) {
    t_mlp_err = e.what();
    return e.code;
  } catch (const std::exception &e) {
    t_mlp_err = e.what();
    return QED_ERR_INTERNAL;
  }
}
}  // namespace

extern "C" {

int qed_mlp_last_error(char *buf, int len) {
  if (buf && len > 0) {
    std::strncpy(buf, t_mlp_err.c_str(), (size_t)len - 1);
    buf[len - 1] = 0;
  }
  return (int)t_mlp_err.size();
}

int qed_mlp_create(int n_in, int width, unsigned long long seed, void **handle) {
  return mlp_guarded([&] {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) qed::fail(QED_ERR_NO_DEVICE, "mlp: no CUDA device available");
    auto h = std::make_unique<MLP>();
    h->init(n_in, width, seed);
    *handle = h.release();
  });
}

void qed_mlp_destroy(void *handle) { delete static_cast<MLP *>(handle); }

int qed_mlp_num_params(void *handle, long *n) {
  return mlp_guarded([&] { *n = (long)static_cast<MLP *>(handle)->n_par; });
}

int qed_mlp_get_params(void *handle, float *out) {
  return mlp_guarded([&] {
    MLP &h = *static_cast<MLP *>(handle);
    QED_CUDA(cudaMemcpyAsync(out, h.p.p, h.n_par * sizeof(float), cudaMemcpyDeviceToHost, h.s));
    QED_CUDA(cudaStreamSynchronize(h.s));
  });
}

int qed_mlp_set_params(void *handle, const float *in) {
  return mlp_guarded([&] {
    MLP &h = *static_cast<MLP *>(handle);
    QED_CUDA(cudaMemcpyAsync(h.p.p, in, h.n_par * sizeof(float), cudaMemcpyHostToDevice, h.s));
    h.sync_bf16();
  });
}

int qed_mlp_layout(void *handle, long *offsets) {
  return mlp_guarded([&] {
    MLP &h = *static_cast<MLP *>(handle);
    for (int i = 0; i < 8; ++i) offsets[i] = (long)h.off[i];
    offsets[8] = h.k_in;
  });
}

int qed_mlp_forward(void *handle, int rows, const float *x, float *y) {
  return mlp_guarded([&] {
    MLP &h = *static_cast<MLP *>(handle);
    if (rows <= 0) return;
    h.load_rows(rows, x, nullptr);
    h.forward(qed::pad16(rows));
    QED_CUDA(cudaMemcpyAsync(y, h.y.p, rows * sizeof(float), cudaMemcpyDeviceToHost, h.s));
    QED_CUDA(cudaStreamSynchronize(h.s));
  });
}

int qed_mlp_gradients(void *handle, int rows, const float *x, const float *t, float *grads, float *loss) {
  return mlp_guarded([&] {
    MLP &h = *static_cast<MLP *>(handle);
    if (rows <= 0 || rows % 16) qed::fail(QED_ERR_ARGUMENT, "mlp: gradient batches are a positive multiple of 16 rows");
    h.load_rows(rows, x, t);
    h.forward(rows);
    h.backward(rows);
    std::vector<float> lt(rows);
    QED_CUDA(cudaMemcpyAsync(grads, h.g.p, h.n_par * sizeof(float), cudaMemcpyDeviceToHost, h.s));
    QED_CUDA(cudaMemcpyAsync(lt.data(), h.lt.p, rows * sizeof(float), cudaMemcpyDeviceToHost, h.s));
    QED_CUDA(cudaStreamSynchronize(h.s));
    double L = 0.0;
    for (float v : lt) L += v;
    *loss = (float)L;
  });
}

int qed_mlp_train(void *handle, int rows, const float *x, const float *t, int epochs, int batch, float lr,
                  unsigned long long seed, float *epoch_loss) {
  return mlp_guarded([&] {
    MLP &h = *static_cast<MLP *>(handle);
    if (batch <= 0 || batch % 16) qed::fail(QED_ERR_ARGUMENT, "mlp: batch must be a positive multiple of 16");
    const int steps = rows / batch;
    if (steps < 1) qed::fail(QED_ERR_ARGUMENT, "mlp: fewer rows than one batch");
    const int used = steps * batch;
    h.reserve(used);
    h.data_x.alloc((size_t)rows * h.n_in);
    h.data_t.alloc(rows);
    h.perm.alloc(used);
    h.data_x.upload(x, (size_t)rows * h.n_in, h.s);
    h.data_t.upload(t, rows, h.s);
    // one epoch = `steps` optimiser steps on consecutive batches of the gathered rows
    if (!h.exec || h.graph_batch != batch || h.graph_steps != steps || h.graph_lr != lr) {
      if (h.exec) cudaGraphExecDestroy(h.exec);
      if (h.graph) cudaGraphDestroy(h.graph);
      h.exec = nullptr;
      h.graph = nullptr;
      QED_CUDA(cudaStreamSynchronize(h.s));
      QED_CUDA(cudaStreamBeginCapture(h.s, cudaStreamCaptureModeThreadLocal));
      bf16 *X0 = h.X.p;
      float *T0 = h.T.p;
      try {
        for (int st = 0; st < steps; ++st) {
          h.X.p = X0 + (size_t)st * batch * h.k_in;  // views into the gathered rows
          h.T.p = T0 + (size_t)st * batch;
          h.forward(batch);
          h.backward(batch);
          h.adam(lr);
        }
      } catch (...) {
        h.X.p = X0;
        h.T.p = T0;
        cudaGraph_t broken = nullptr;
        cudaStreamEndCapture(h.s, &broken);
        if (broken) cudaGraphDestroy(broken);
        throw;
      }
      h.X.p = X0;
      h.T.p = T0;
      cudaError_t e = cudaStreamEndCapture(h.s, &h.graph);
      if (e != cudaSuccess) qed::fail(QED_ERR_CUDA, std::string("mlp: graph capture failed: ") + cudaGetErrorString(e));
      QED_CUDA(cudaGraphInstantiate(&h.exec, h.graph, 0));
      h.graph_batch = batch;
      h.graph_steps = steps;
      h.graph_lr = lr;
    }
    std::mt19937_64 rng(seed);
    std::vector<int> perm(rows);
    std::vector<float> lt(used);
    for (int ep = 0; ep < epochs; ++ep) {
      for (int i = 0; i < rows; ++i) perm[i] = i;
      std::shuffle(perm.begin(), perm.end(), rng);
      h.perm.upload(perm.data(), used, h.s);
      qed::k_gather<<<(used + 255) / 256, 256, 0, h.s>>>(used, h.n_in, h.k_in, h.data_x.p, h.data_t.p, h.perm.p,
                                                         h.X.p, h.T.p);
      QED_LAUNCH();
      QED_CUDA(cudaGraphLaunch(h.exec, h.s));
      if (epoch_loss) {  // the loss terms of the last batch of the epoch
        QED_CUDA(cudaMemcpyAsync(lt.data(), h.lt.p, batch * sizeof(float), cudaMemcpyDeviceToHost, h.s));
        QED_CUDA(cudaStreamSynchronize(h.s));
        double L = 0.0;
        for (int i = 0; i < batch; ++i) L += lt[i];
        epoch_loss[ep] = (float)L;
      }
    }
    QED_CUDA(cudaStreamSynchronize(h.s));
  });
}

}  // extern "C"
