// Dense block kernels of the block form of the band-Lanczos recurrence
// (block_lanczos_qmatrix, solver.cpp). A block is p <= 16 separate FP64 vectors
// of D states (pointer arrays, so the start vectors form a block without a
// copy); the H.v of a block is p staged H.v launches on its vectors.
//
// k_bl_update: Y = a Y + s1 X1 M1 (M1 p x p, row-major), then optionally the
// per-CTA partials of L^T Y for L = the updated Y or another block. One thread
// per state: the thread loads its state's p values of each block (coalesced
// across the warp), forms the update with M1 broadcast from shared memory and
// stores the result. The Gram matrix runs on the FP64 tensor cores: each warp
// copies its 32 states of L and Y into shared memory (rows padded to 20
// doubles, so the fragment reads are free of bank conflicts) and accumulates
// L^T Y with mma.sync m8n8k4 (A = L^T: row = vector, column = state; B = Y:
// row = state, column = vector), 2 x 2 tiles of 8 x 8 for p > 8.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "common.hpp"
#include "kernels.cuh"

namespace qed {

namespace {

constexpr int kBlThreads = 256;
constexpr int kBlWarps = kBlThreads / 32;
constexpr int kStageLd = 20;  // padded row of one state's 16 values in shared memory

__device__ __forceinline__ void mma_f64(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <int P>
__global__ void __launch_bounds__(kBlThreads, 1) k_bl_simple(size_t D, int p, double a, BlockOut Y, double s1,
                                                          BlockIn X1, const double *__restrict__ M1, int gram,
                                                          BlockIn L, double *partials) {
  constexpr int NT = P / 8;  // 8 x 8 tiles per side
  // dynamic shared memory: M1, then per warp the two staged 32-state panels
  // (reused for the cross-warp sum of the Gram partials at the end)
  extern __shared__ double smem_bl[];
  double *m1 = smem_bl;
  double *stage = smem_bl + P * P;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool upd = X1.v[0] != nullptr;
  for (int t = threadIdx.x; t < P * P; t += blockDim.x) {
    const int i = t / P, c = t % P;
    m1[t] = (upd && i < p && c < p) ? M1[i * p + c] : 0.0;
  }
  __syncthreads();
  double acc[NT * NT][2];
#pragma unroll
  for (int q = 0; q < NT * NT; ++q) acc[q][0] = acc[q][1] = 0.0;
  double *sl = stage + (size_t)warp * 2 * 32 * kStageLd, *sy = sl + 32 * kStageLd;
  const size_t stride = (size_t)gridDim.x * kBlThreads;
  for (size_t I0 = (size_t)blockIdx.x * kBlThreads + warp * 32; I0 < D; I0 += stride) {
    const size_t I = I0 + lane;
    const bool valid = I < D;
    double y[P];
#pragma unroll
    for (int c = 0; c < P; ++c) y[c] = (valid && c < p && a != 0.0) ? a * Y.v[c][I] : 0.0;
    if (upd) {
      double x[P];
#pragma unroll
      for (int i = 0; i < P; ++i) x[i] = (valid && i < p) ? X1.v[i][I] : 0.0;
#pragma unroll
      for (int c = 0; c < P; ++c) {
        double t = 0.0;
#pragma unroll
        for (int i = 0; i < P; ++i) t = fma(x[i], m1[i * P + c], t);
        y[c] = fma(s1, t, y[c]);
      }
    }
    if (valid && (upd || a != 1.0)) {  // a pure Gram (a = 1, no update) leaves Y as it is
#pragma unroll
      for (int c = 0; c < P; ++c)
        if (c < p) Y.v[c][I] = y[c];
    }
    if (gram) {
#pragma unroll
      for (int c = 0; c < P; ++c) {
        const double l = gram == 1 ? y[c] : ((valid && c < p) ? L.v[c][I] : 0.0);
        sl[lane * kStageLd + c] = l;
        sy[lane * kStageLd + c] = y[c];
      }
      __syncwarp();
#pragma unroll
      for (int k0 = 0; k0 < 32; k0 += 4) {
        const int st = (k0 + (lane & 3)) * kStageLd + (lane >> 2);
        double af[NT], bf[NT];
#pragma unroll
        for (int t = 0; t < NT; ++t) {
          af[t] = sl[st + 8 * t];
          bf[t] = sy[st + 8 * t];
        }
#pragma unroll
        for (int mt = 0; mt < NT; ++mt)
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) mma_f64(acc[mt * NT + nt][0], acc[mt * NT + nt][1], af[mt], bf[nt]);
      }
      __syncwarp();  // the stage is read before the next states overwrite it
    }
  }
  if (!gram) return;
  __syncthreads();  // every warp is done with its panels: they now hold the partial Grams
  double *red = stage;  // [warp][P * P]
  // C fragment: row lane >> 2, columns 2 (lane & 3) + {0, 1} of each tile
#pragma unroll
  for (int mt = 0; mt < NT; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int j = 0; j < 2; ++j)
        red[warp * P * P + (mt * 8 + (lane >> 2)) * P + nt * 8 + 2 * (lane & 3) + j] = acc[mt * NT + nt][j];
  __syncthreads();
  for (int t = threadIdx.x; t < p * p; t += blockDim.x) {
    const int i = t / p, c = t % p;
    double s = 0.0;
    for (int w = 0; w < kBlWarps; ++w) s += red[w * P * P + i * P + c];
    partials[(size_t)blockIdx.x * p * p + t] = s;
  }
}

// ---- pipelined tensor-core form -------------------------------------------
//
// Each warp streams tiles of 32 consecutive states. A tile's p values of each
// block it reads (X1, Y unless a = 0, L for gram 2) arrive as panels in shared
// memory by cp.async (16-byte chunks, double-buffered: the next tile's panels
// are in flight while this one computes). A panel is laid out [vector][state]
// with a row of kPanelLd = 36 doubles, so that every fragment read below hits
// 16 distinct 8-byte bank slots per half-warp. The update runs as FP64 mma:
// C (8 states x 8 vectors) = a Y + (X1 tile) (s1 M1 tile), M1's fragments held
// in registers; C goes back into the Y panel, the Gram fragments read the
// panels, and the Y panel goes out with coalesced 16-byte stores.
constexpr int kPanelLd = 36;
constexpr int kPipeWarps = 4;
constexpr int kPipeThreads = 32 * kPipeWarps;

__device__ __forceinline__ void cp_async16(void *dst, const void *src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)),
               "l"(src), "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Lane's share of a panel copy: chunk q = lane + 32 r holds vector q / 16,
// states 2 (q % 16) and 2 (q % 16) + 1 of the tile at I0 (zero-filled past D).
template <int P, class B>
__device__ __forceinline__ void load_panel(double *panel, const B &V, int p, size_t I0, size_t D, int lane) {
  const int hi = lane >> 4, j = lane & 15;
  const size_t I = I0 + 2 * j;
  const int bytes = I + 2 <= D ? 16 : (I < D ? 8 : 0);
#pragma unroll
  for (int r = 0; r < P / 2; ++r) {
    const int c = 2 * r + hi;  // lanes 0-15 copy vector 2r, lanes 16-31 vector 2r + 1
    const double *src = hi ? V.v[2 * r + 1] : V.v[2 * r];
    if (c < p) cp_async16(panel + c * kPanelLd + 2 * j, src + (I < D ? I : 0), bytes);
  }
}

template <int P>
__global__ void __launch_bounds__(kPipeThreads) k_bl_pipe(size_t D, int p, double a, BlockOut Y, double s1,
                                                          BlockIn X1, const double *__restrict__ M1, int gram,
                                                          BlockIn L, double *partials) {
  constexpr int NT = P / 8;      // 8-vector tiles
  constexpr int KS = P / 4;      // k steps of the update
  constexpr int PANEL = P * kPanelLd;
  extern __shared__ double smem_pipe[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const bool upd = X1.v[0] != nullptr, rdy = a != 0.0, useL = gram == 2;
  const bool store = upd || a != 1.0;
  // per warp: 2 stages x (X, Y, L) panels
  double *base = smem_pipe + (size_t)warp * 2 * 3 * PANEL;
  auto px = [&](int st) { return base + (st * 3 + 0) * PANEL; };
  auto py = [&](int st) { return base + (st * 3 + 1) * PANEL; };
  auto pl = [&](int st) { return base + (st * 3 + 2) * PANEL; };
  // rows of vectors >= p stay zero in every panel
  for (int i = lane; i < 2 * 3 * PANEL; i += 32) base[i] = 0.0;
  __syncwarp();
  // s1 M1 as B fragments: row k = input vector, column n = output vector
  double bm[KS][NT];
#pragma unroll
  for (int ks = 0; ks < KS; ++ks)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const int i = 4 * ks + (lane & 3), c = 8 * nt + (lane >> 2);
      bm[ks][nt] = (upd && i < p && c < p) ? s1 * M1[i * p + c] : 0.0;
    }
  double g[NT * NT][2];
#pragma unroll
  for (int q = 0; q < NT * NT; ++q) g[q][0] = g[q][1] = 0.0;
  const size_t ntile = (D + 31) / 32;
  const size_t nw = (size_t)gridDim.x * kPipeWarps;
  size_t t = (size_t)blockIdx.x * kPipeWarps + warp;
  auto issue = [&](size_t tt, int st) {
    if (tt < ntile) {
      const size_t I0 = tt * 32;
      if (upd) load_panel<P>(px(st), X1, p, I0, D, lane);
      if (rdy) load_panel<P>(py(st), Y, p, I0, D, lane);
      if (useL) load_panel<P>(pl(st), L, p, I0, D, lane);
    }
    cp_async_commit();  // one group per tile, empty past the end
  };
  issue(t, 0);
  for (int st = 0; t < ntile; t += nw, st ^= 1) {
    issue(t + nw, st ^ 1);  // the next tile's panels fly while this one computes
    cp_async_wait1();
    __syncwarp();
    double *X = px(st), *Yp = py(st), *Lp = useL ? pl(st) : Yp;
    if (store) {
      // C = a Y + X (s1 M1), 4 tiles of 8 states x NT tiles of 8 vectors
#pragma unroll
      for (int mt = 0; mt < 4; ++mt) {
        double c[NT][2];
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const int v = 8 * nt + 2 * (lane & 3) + j;
            c[nt][j] = rdy ? a * Yp[v * kPanelLd + 8 * mt + (lane >> 2)] : 0.0;
          }
        if (upd) {
#pragma unroll
          for (int ks = 0; ks < KS; ++ks) {
            const double af = X[(4 * ks + (lane & 3)) * kPanelLd + 8 * mt + (lane >> 2)];
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) mma_f64(c[nt][0], c[nt][1], af, bm[ks][nt]);
          }
        }
        __syncwarp();  // every lane has read its Y fragments of this state tile
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            const int v = 8 * nt + 2 * (lane & 3) + j;
            Yp[v * kPanelLd + 8 * mt + (lane >> 2)] = c[nt][j];
          }
      }
      __syncwarp();
    }
    if (gram) {
      // G += L^T Y' over the tile's 32 states
#pragma unroll
      for (int k0 = 0; k0 < 32; k0 += 4) {
        double af[NT], bf[NT];
#pragma unroll
        for (int u = 0; u < NT; ++u) {
          af[u] = Lp[(8 * u + (lane >> 2)) * kPanelLd + k0 + (lane & 3)];
          bf[u] = Yp[(8 * u + (lane >> 2)) * kPanelLd + k0 + (lane & 3)];
        }
#pragma unroll
        for (int mt = 0; mt < NT; ++mt)
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) mma_f64(g[mt * NT + nt][0], g[mt * NT + nt][1], af[mt], bf[nt]);
      }
    }
    if (store) {
      const size_t I0 = t * 32;
      const int hi = lane >> 4, j = lane & 15;
      const size_t I = I0 + 2 * j;
#pragma unroll
      for (int r = 0; r < P / 2; ++r) {
        const int c = 2 * r + hi;
        double *dst = hi ? Y.v[2 * r + 1] : Y.v[2 * r];
        if (c < p && I < D) {
          const double2 v = *reinterpret_cast<const double2 *>(Yp + c * kPanelLd + 2 * j);
          if (I + 1 < D) *reinterpret_cast<double2 *>(dst + I) = v;
          else dst[I] = v.x;
        }
      }
    }
    __syncwarp();  // the stage is free for the tile after next
  }
  if (!gram) return;
  __syncthreads();
  double *red = smem_pipe;  // [warp][P * P], over the panels (all warps are done with them)
#pragma unroll
  for (int mt = 0; mt < NT; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt)
#pragma unroll
      for (int j = 0; j < 2; ++j)
        red[warp * P * P + (mt * 8 + (lane >> 2)) * P + nt * 8 + 2 * (lane & 3) + j] = g[mt * NT + nt][j];
  __syncthreads();
  for (int u = threadIdx.x; u < p * p; u += blockDim.x) {
    const int i = u / p, c = u % p;
    double s = 0.0;
    for (int w = 0; w < kPipeWarps; ++w) s += red[w * P * P + i * P + c];
    partials[(size_t)blockIdx.x * p * p + u] = s;
  }
}

}  // namespace

int launch_bl_update(size_t D, int p, double a, const BlockOut &Y, double s1, const BlockIn &X1, const double *M1,
                     int gram, const BlockIn &L, double *partials, int max_blocks, cudaStream_t s) {
  if (p < 1 || p > 16) fail(QED_ERR_ARGUMENT, "block update: block size outside [1, 16]");
  if (!D) return 0;
  static const int sms = [] {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 148;
  }();
  const size_t want = (D + kBlThreads - 1) / kBlThreads;
  int grid = (int)std::min<size_t>(want, (size_t)sms * 2);
  if (gram && grid > max_blocks) grid = max_blocks;
  grid = std::max(grid, 1);
  // the pipelined form needs 16-byte aligned vectors (D even, aligned bases)
  bool pipe = D % 2 == 0;
  for (int c = 0; c < p; ++c) {
    if ((uintptr_t)Y.v[c] & 15u) pipe = false;
    if (X1.v[0] && ((uintptr_t)X1.v[c] & 15u)) pipe = false;
    if (gram == 2 && ((uintptr_t)L.v[c] & 15u)) pipe = false;
  }
  if (pipe) {
    auto psmem = [](int P) { return (size_t)kPipeWarps * 2 * 3 * P * kPanelLd * sizeof(double); };
    static const bool pattr = [&] {
      QED_CUDA(cudaFuncSetAttribute(k_bl_pipe<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem(8)));
      QED_CUDA(cudaFuncSetAttribute(k_bl_pipe<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psmem(16)));
      return true;
    }();
    (void)pattr;
    const size_t tiles = (D + 31) / 32;
    // two CTAs per SM fit (shared memory); the warps stride over the tiles
    int g2 = (int)std::min<size_t>((tiles + kPipeWarps - 1) / kPipeWarps, (size_t)sms * 2);
    if (gram && g2 > max_blocks) g2 = max_blocks;
    g2 = std::max(g2, 1);
    if (p <= 8)
      k_bl_pipe<8><<<g2, kPipeThreads, psmem(8), s>>>(D, p, a, Y, s1, X1, M1, gram, L, partials);
    else
      k_bl_pipe<16><<<g2, kPipeThreads, psmem(16), s>>>(D, p, a, Y, s1, X1, M1, gram, L, partials);
    QED_LAUNCH();
    return g2;
  }
  auto smem = [](int P) { return (size_t)(P * P + kBlWarps * 2 * 32 * kStageLd) * sizeof(double); };
  static const bool attr = [&] {
    QED_CUDA(cudaFuncSetAttribute(k_bl_simple<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem(8)));
    QED_CUDA(cudaFuncSetAttribute(k_bl_simple<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem(16)));
    return true;
  }();
  (void)attr;
  if (p <= 8)
    k_bl_simple<8><<<grid, kBlThreads, smem(8), s>>>(D, p, a, Y, s1, X1, M1, gram, L, partials);
  else
    k_bl_simple<16><<<grid, kBlThreads, smem(16), s>>>(D, p, a, Y, s1, X1, M1, gram, L, partials);
  QED_LAUNCH();
  return grid;
}

}  // namespace qed
