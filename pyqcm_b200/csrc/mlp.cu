// Surrogate network for VCA: a multilayer perceptron n_in -> W -> W -> W -> 1
// with GELU activations, trained by Adam on data this solver generates
// (Potthoff functional values at points of the variational parameters).
//
// Arithmetic: weights and activations enter the matrix products in BF16 on
// the tensor cores with FP32 accumulation; biases, pre-activations, gradients,
// the loss and Adam's master weights and moments are FP32. Every matrix
// product is one tcgen05 kernel (128 x BN tiles accumulated in tensor memory,
// operands staged in shared memory); sizes are padded to multiples of 16 (the
// input width to 16 with zero columns).
//
// One training step (forward, backward, Adam) is a fixed sequence of kernels
// on the network's stream; the steps of an epoch are captured once into a
// CUDA graph and replayed, the epoch's shuffled data being gathered into the
// same device buffers before each replay.
#include <cuda_bf16.h>

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

typedef __nv_bfloat16 bf16;

namespace qed {
namespace {

inline int pad16(int x) { return (x + 15) / 16 * 16; }

// ---- matrix products on the 5th-generation tensor cores (tcgen05) ----------
//
// One CTA of 128 threads computes a 128 x BN tile of C = A B^T (A: M x K, B: N x K,
// both bf16 with K contiguous) into a TMEM accumulator (fp32, 128 lanes x BN
// columns). Per round of 64 K-elements the CTA stages the A and B tiles in
// shared memory with cp.async in the canonical K-major layout without swizzle
// (8 x 8 core matrices of 128 contiguous bytes, core matrices adjacent in K 128
// bytes apart, 8-row groups 1024 bytes apart); one elected thread then issues
// the round's four 128 x BN x 16 tcgen05.mma (kind::f16, bf16 inputs, fp32
// accumulation) and commits them to an mbarrier, which every thread waits on
// (bounded) before the tiles are overwritten. The epilogue reads the
// accumulator back with tcgen05.ld (each warp its 32 lanes = 32 rows).

constexpr int kUmmaM = 128;       // rows of a tile = TMEM lanes (cta_group::1)
constexpr int kUmmaBK = 64;       // K elements staged per round
constexpr int kUmmaMaxBN = 128;   // columns of a tile
constexpr int kUmmaThreads = 128;
constexpr uint32_t kUmmaSbo = kUmmaBK / 8 * 128;  // bytes between 8-row groups
constexpr uint32_t kUmmaLbo = 128;                // bytes between K-adjacent core matrices
constexpr size_t kUmmaTileBytes = (size_t)kUmmaM * kUmmaBK * 2;
// Dynamic shared memory per CTA: both tiles, the barrier and the TMEM address,
// rounded up so that at most three CTAs share an SM (3 x 128 TMEM columns <= 512).
constexpr size_t kUmmaSmem = 72 * 1024;

// Set when a bounded wait for the tensor core gave up; read by the host.
__device__ int g_mlp_wait_timeout = 0;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (sm_100 format): start address, leading and
// stride byte offsets (all >> 4), descriptor version 1 at bit 46, no swizzle.
__device__ __forceinline__ uint64_t umma_smem_desc(uint32_t saddr) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((kUmmaLbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((kUmmaSbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: fp32 D (bits 4-5 = 1), bf16 A and B
// (bits 7-9 and 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(src_bytes) : "memory");
}

// Waits for phase `parity` of the mbarrier; gives up after about two seconds.
__device__ __forceinline__ bool umma_wait(uint64_t *bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  uint64_t t0 = 0;
  for (uint32_t it = 0;; ++it) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if ((it & 255u) == 0) {
      uint64_t t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      if (it == 0) t0 = t;
      else if (t - t0 > 2000000000ull) {
        atomicExch(&g_mlp_wait_timeout, 1);
        return false;
      }
    }
  }
}

// Stages rows [r0, r0 + rows_tile) x K-elements [k0, k0 + kc) of a row-major
// bf16 matrix (leading dimension ld) in the canonical layout; rows at or past
// `rows_total` are zero-filled.
__device__ __forceinline__ void umma_stage(uint32_t sdst, const bf16 *src, int ld, int r0, int rows_tile,
                                           int rows_total, int k0, int kc) {
  const int chunks = kc >> 3;  // 16-byte chunks per row
  for (int c = threadIdx.x; c < rows_tile * chunks; c += kUmmaThreads) {
    const int r = c / chunks, q = c - r * chunks;
    const bool in = r0 + r < rows_total;
    const bf16 *g = src + (size_t)(in ? r0 + r : 0) * ld + k0 + 8 * q;
    cp_async16(sdst + (uint32_t)(r >> 3) * kUmmaSbo + (uint32_t)q * kUmmaLbo + (uint32_t)(r & 7) * 16, g,
               in ? 16 : 0);
  }
}

// C[M x N] (fp32 row-major, ldc) (+)= A[M x K] B[N x K]^T. A and B are bf16
// row-major with K contiguous (lda, ldb multiples of 8, 16-byte aligned rows);
// K a multiple of 16; bn (columns per tile) a multiple of 16 in [16, 128].
__global__ void __launch_bounds__(kUmmaThreads) k_umma_gemm(int M, int N, int K, const bf16 *__restrict__ A, int lda,
                                                            const bf16 *__restrict__ B, int ldb, float *__restrict__ C,
                                                            int ldc, int accumulate, int bn) {
  extern __shared__ __align__(1024) unsigned char sm[];
  const uint32_t sa = smem_u32(sm), sb = sa + (uint32_t)kUmmaTileBytes;
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm + 2 * kUmmaTileBytes);
  uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
  const int m0 = blockIdx.x * kUmmaM, n0 = blockIdx.y * bn;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t ncols = bn <= 32 ? 32u : bn <= 64 ? 64u : 128u;  // a power of two >= 32
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (threadIdx.x == 32) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tslot;
  const uint32_t idesc = umma_idesc_bf16(kUmmaM, bn);
  uint32_t phase = 0;
  bool ok = true;
  for (int k0 = 0; k0 < K; k0 += kUmmaBK) {
    const int kc = min(kUmmaBK, K - k0);
    umma_stage(sa, A, lda, m0, kUmmaM, M, k0, kc);
    umma_stage(sb, B, ldb, n0, bn, N, k0, kc);
    asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the tensor core's reads
    __syncthreads();
    if (threadIdx.x == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int kk = 0; kk < kc / 16; ++kk) {
        const uint64_t ad = umma_smem_desc(sa + 2u * kUmmaLbo * (uint32_t)kk);
        const uint64_t bd = umma_smem_desc(sb + 2u * kUmmaLbo * (uint32_t)kk);
        const uint32_t acc = (k0 > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
            "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(bar))
                   : "memory");
    }
    ok = __syncthreads_and(umma_wait(bar, phase));  // the MMAs have read the tiles
    phase ^= 1u;
    if (!ok) break;
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) {
    const int row = m0 + warp * 32 + lane;
    for (int c0 = 0; c0 < bn; c0 += 16) {
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
          "%14, %15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
            "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (row < M) {
        float *crow = C + (size_t)row * ldc + n0 + c0;
#pragma unroll
        for (int j = 0; j < 16; ++j)
          if (n0 + c0 + j < N) crow[j] = (accumulate ? crow[j] : 0.0f) + __uint_as_float(v[j]);
      }
    }
  } else {
    umma_wait(bar, phase ^ 1u);  // a commit still in flight has had its bounded chance to land
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols) : "memory");
}

// out[c][r] = in[r][c] for an R x Cn bf16 matrix (leading dimensions ld_in, ld_out).
__global__ void k_transpose_bf16(int R, int Cn, const bf16 *__restrict__ in, int ld_in, bf16 *__restrict__ out,
                                 int ld_out) {
  __shared__ bf16 t[32][34];
  const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int r = r0 + i, c = c0 + threadIdx.x;
    t[i][threadIdx.x] = (r < R && c < Cn) ? in[(size_t)r * ld_in + c] : __float2bfloat16_rn(0.0f);
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const int c = c0 + i, r = r0 + threadIdx.x;
    if (c < Cn && r < R) out[(size_t)c * ld_out + r] = t[threadIdx.x][i];
  }
}

void transpose(int R, int Cn, const bf16 *in, int ld_in, bf16 *out, int ld_out, cudaStream_t s) {
  k_transpose_bf16<<<dim3((Cn + 31) / 32, (R + 31) / 32), dim3(32, 8), 0, s>>>(R, Cn, in, ld_in, out, ld_out);
  QED_LAUNCH();
}

void umma_setup() {
  static bool done = false;  // the attribute is per function, once per process is enough
  if (!done) {
    QED_CUDA(cudaFuncSetAttribute(k_umma_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kUmmaSmem));
    done = true;
  }
}

// Fails the call if a product's bounded wait for the tensor core gave up since
// the last check (the flag is cleared for the next call).
void check_umma_wait(cudaStream_t s) {
  int flag = 0;
  QED_CUDA(cudaStreamSynchronize(s));
  QED_CUDA(cudaMemcpyFromSymbol(&flag, g_mlp_wait_timeout, sizeof(int)));
  if (flag) {
    const int zero = 0;
    cudaMemcpyToSymbol(g_mlp_wait_timeout, &zero, sizeof(int));
    fail(QED_ERR_CUDA, "mlp: a tensor-core product timed out waiting for its MMAs");
  }
}

// C[M x N] (+)= A B^T on the tensor cores, A: M x K, B: N x K (K contiguous).
void gemm_tn(int M, int N, int K, const bf16 *A, int lda, const bf16 *B, int ldb, float *C, int ldc, bool acc,
             cudaStream_t s) {
  if (M <= 0 || N <= 0 || K <= 0 || K % 16 || N % 16 || lda % 8 || ldb % 8)
    fail(QED_ERR_ARGUMENT, "mlp: tensor-core product needs K and N multiples of 16 and 16-byte rows");
  const int bn = std::min(N, kUmmaMaxBN);
  dim3 grid((M + kUmmaM - 1) / kUmmaM, (N + bn - 1) / bn);
  k_umma_gemm<<<grid, kUmmaThreads, kUmmaSmem, s>>>(M, N, K, A, lda, B, ldb, C, ldc, acc ? 1 : 0, bn);
  QED_LAUNCH();
}

// C[M x N] (fp32, row-major, ldc) (+)= op(A) op(B), op(A) M x K, op(B) K x N.
// TA: A stored K x M, else M x K row-major. TB: B stored N x K, else K x N
// row-major. Operands not already K-contiguous are transposed into the
// scratch buffers ta / tb first (each at least M*K / N*K elements).
template <bool TA, bool TB>
void gemm(int M, int N, int K, const bf16 *A, int lda, const bf16 *B, int ldb, float *C, int ldc, bool acc,
          bf16 *ta, bf16 *tb, cudaStream_t s) {
  if (TA) {
    transpose(K, M, A, lda, ta, K, s);
    A = ta;
    lda = K;
  }
  if (!TB) {
    transpose(K, N, B, ldb, tb, K, s);
    B = tb;
    ldb = K;
  }
  gemm_tn(M, N, K, A, lda, B, ldb, C, ldc, acc, s);
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
  DevBuf<bf16> ta, tb;  // transposed operands of the backward products
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
    umma_setup();
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
    ta.alloc((size_t)W * std::max(cap, W));
    tb.alloc((size_t)W * std::max(cap, W));
  }

  // forward on rows [0, rows) of X (bf16, padded); y = network output
  void forward(int rows) {
    const bf16 *in = X.p;
    int kin = k_in;
    for (int l = 0; l < 3; ++l) {
      gemm_tn(rows, W, kin, in, kin, Ph(2 * l), kin, Z[l].p, W, false, s);
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
      gemm<true, false>(W, kin, rows, dZh[l].p, W, prev, kin, Gr(2 * l), kin, false, ta.p, tb.p, s);
      k_colsum<<<(W + 255) / 256, 256, 0, s>>>(rows, W, dZ[l].p, nullptr, Gr(2 * l + 1));
      QED_LAUNCH();
      if (l > 0) {  // dH_{l-1} = dZ_l W_l, then through GELU'
        gemm<false, false>(rows, W, W, dZh[l].p, W, Ph(2 * l), W, dZ[l - 1].p, W, false, ta.p, tb.p, s);
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
    qed::check_umma_wait(h.s);
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
    qed::check_umma_wait(h.s);
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
        qed::check_umma_wait(h.s);
        double L = 0.0;
        for (int i = 0; i < batch; ++i) L += lt[i];
        epoch_loss[ep] = (float)L;
      }
    }
    qed::check_umma_wait(h.s);
  });
}

int qed_mlp_tensor_product(int M, int N, int K, const uint16_t *A, const uint16_t *B, float *C) {
  return mlp_guarded([&] {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) qed::fail(QED_ERR_NO_DEVICE, "mlp: no CUDA device available");
    if (M <= 0 || N <= 0 || K <= 0 || K % 16 || N % 16)
      qed::fail(QED_ERR_ARGUMENT, "mlp: tensor product needs positive M and K, N multiples of 16");
    cudaStream_t s = nullptr;
    QED_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct Guard {
      cudaStream_t s;
      ~Guard() {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
      }
    } guard{s};
    qed::umma_setup();
    qed::DevBuf<bf16> a((size_t)M * K), b((size_t)N * K);
    qed::DevBuf<float> c((size_t)M * N);
    QED_CUDA(cudaStreamSynchronize(qed::alloc_stream()));  // the allocations are usable on s
    a.upload(reinterpret_cast<const bf16 *>(A), (size_t)M * K, s);
    b.upload(reinterpret_cast<const bf16 *>(B), (size_t)N * K, s);
    qed::gemm_tn(M, N, K, a.p, K, b.p, K, c.p, N, false, s);
    c.download(C, (size_t)M * N, s);
    qed::check_umma_wait(s);
  });
}

}  // extern "C"
