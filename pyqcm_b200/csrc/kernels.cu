// sm_100a kernels of the ED solver (see kernels.cuh for the contracts).
//
// Layout in HBM: a sector vector is the dim_dn x dim_up matrix x[dn][up],
// row-major (index up + dim_up * dn), the factorized basis order of the
// reference (src_ed/ED_basis.cpp:142-165). Up-spin hops act along rows,
// down-spin hops along columns. All arithmetic is FP64.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>

#include "common.hpp"
#include "options.hpp"
#include "kernels.cuh"
#include "winhv.hpp"

namespace qed {

namespace {

constexpr int kThreads = 256;

// C(n, k) for n, k <= 32 (C(32,16) < 2^32).
__constant__ uint32_t c_binom[33][33];
std::once_flag g_binom_once;

void ensure_binom() {
  std::call_once(g_binom_once, [] {
    uint32_t h[33][33] = {};
    for (int n = 0; n <= 32; ++n)
      for (int k = 0; k <= 32; ++k) h[n][k] = (uint32_t)binom(n, k);
    QED_CUDA(cudaMemcpyToSymbol(c_binom, h, sizeof(h)));
    // the copy runs on the legacy stream, which the solver's non-blocking
    // streams do not wait for: finish it before any kernel reads the table
    QED_CUDA(cudaDeviceSynchronize());
  });
}

// Colex rank of an N-of-L string: sum_k C(p_k, k+1) over set bits p_0 < p_1 < ...
// Equals the position in the ascending list of N-of-L strings, i.e.
// ED_halfbasis::index (src_ed/ED_basis.cpp:130-135).
__device__ __forceinline__ uint32_t colex_rank(uint32_t b) {
  uint32_t r = 0;
  int k = 1;
  while (b) {
    int p = __ffs(b) - 1;
    r += c_binom[p][k++];
    b &= b - 1;
  }
  return r;
}

__device__ __forceinline__ uint32_t colex_unrank(uint32_t I, int L, int N) {
  uint32_t b = 0;
  int p = L - 1;
  for (int k = N; k >= 1; --k) {
    while (c_binom[p][k] > I) --p;
    b |= 1u << p;
    I -= c_binom[p][k];
    --p;
  }
  return b;
}

template <int NRED>
__device__ __forceinline__ void block_reduce_store(double (&v)[NRED], double *partials, int nred) {
  __shared__ double sm[NRED > 0 ? NRED : 1][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int i = 0; i < NRED; ++i) {
    double x = v[i];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if (lane == 0) sm[i][warp] = x;
  }
  __syncthreads();
  if (threadIdx.x < nred) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += sm[threadIdx.x][w];
    partials[(size_t)blockIdx.x * Reducer::kMaxRed + threadIdx.x] = s;
  }
}

__global__ void k_finalize(const double *partials, int nblocks, double *out) {
  // one block per slot, fixed-order tree sum
  __shared__ double sm[kThreads];
  const int slot = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partials[(size_t)b * Reducer::kMaxRed + slot];
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[slot] = sm[0];
}

int grid_for(size_t n, int num_sms, int per_sm = 4) {
  size_t g = (n + kThreads - 1) / kThreads;
  size_t cap = (size_t)num_sms * per_sm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

int device_sms() {
  static const int n = [] {
    int dev = 0, c = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&c, cudaDevAttrMultiProcessorCount, dev);
    return c > 0 ? c : 148;
  }();
  return n;
}

// ---------------------------------------------------------------- basis ----

__global__ void k_unrank(int L, int N, uint32_t dim, uint32_t *out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += gridDim.x * blockDim.x)
    out[i] = colex_unrank(i, L, N);
}

__global__ void k_rank(int L, int N, size_t n, const uint32_t *s, uint32_t *r) {
  const uint32_t dim = c_binom[L][N];
  const uint32_t lim = (L >= 32) ? 0xffffffffu : ((1u << L) - 1u);
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    uint32_t b = s[i];
    r[i] = ((b & ~lim) == 0 && __popc(b) == N) ? colex_rank(b) : dim;
  }
}

__device__ __forceinline__ uint32_t between_mask(int a, int b) {
  int lo = a < b ? a : b, hi = a < b ? b : a;
  uint64_t m = ((1ull << hi) - 1ull) & ~((2ull << lo) - 1ull);
  return (uint32_t)m;
}

// One-body hops c^+_r c_c on every string (HS_half_operator ctor,
// src_ed/Operators/HS_half_operator.hpp:17-45): allowed when bit c is set and
// bit r empty; phase (-1)^(number of set bits strictly between r and c)
// (binary_state::one_body / interphase, src_ed/binary_state.cpp:23-28,
// src_ed/binary_state.hpp:42-47).
__global__ void k_build_hops(int L, int N, uint32_t dim, const uint32_t *bits, int npairs,
                             const int *pd, const int *ps, const int *pslot, uint8_t *cnt,
                             uint32_t *ell, int width) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += gridDim.x * blockDim.x) {
    uint32_t b = bits[i];
    int k = 0;
    for (int q = 0; q < npairs; ++q) {
      int r = pd[q], c = ps[q];
      if (!((b >> c) & 1u) || ((b >> r) & 1u)) continue;
      uint32_t nb = b ^ (1u << c) ^ (1u << r);
      int sgn = __popc(nb & between_mask(r, c)) & 1;
      uint32_t J = colex_rank(nb);
      if (k < width) ell[(size_t)k * dim + i] = (J << 8) | (uint32_t)(pslot[q] + sgn);
      ++k;
    }
    cnt[i] = (uint8_t)(k < width ? k : width);
  }
}

__global__ void k_diag_half(int L, uint32_t dim, const uint32_t *bits, const double *tdiag,
                            const double *vsame, double *diag) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += gridDim.x * blockDim.x) {
    uint32_t b = bits[i];
    double s = 0.0;
    for (int r = 0; r < L; ++r)
      if ((b >> r) & 1u) {
        s += tdiag[r];
        for (int c = r; c < L; ++c)
          if ((b >> c) & 1u) s += vsame[r * L + c];
      }
    diag[i] = s;
  }
}

__global__ void k_cdag_gather(int L, int spin, int a, int pm, const uint32_t *tub, uint32_t du_t,
                              const uint32_t *tdb, uint32_t dd_t, int src_nup, int src_ndn,
                              uint32_t du_s, const double *psi, double *y, double coef, int acc) {
  const size_t D = (size_t)du_t * dd_t;
  const uint32_t bit = 1u << a, below = bit - 1u;
  for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < D; I += (size_t)gridDim.x * blockDim.x) {
    uint32_t u = (uint32_t)(I % du_t), d = (uint32_t)(I / du_t);
    uint32_t tu = tub[u];
    double val = 0.0;
    if (spin == 0) {
      bool occ = (tu & bit) != 0;
      if (pm < 0 ? !occ : occ) {
        uint32_t s = tu ^ bit;  // source up string
        int ph = __popc((pm < 0 ? s : tu) & below) & 1;
        size_t src = (size_t)colex_rank(s) + (size_t)du_s * d;
        val = ph ? -psi[src] : psi[src];
      }
    } else {
      uint32_t td = tdb[d];
      bool occ = (td & bit) != 0;
      if (pm < 0 ? !occ : occ) {
        uint32_t s = td ^ bit;  // source dn string
        int ph = (__popc((pm < 0 ? s : td) & below) + __popc(tu)) & 1;
        size_t src = (size_t)u + (size_t)du_s * colex_rank(s);
        val = ph ? -psi[src] : psi[src];
      }
    }
    y[I] = (acc ? y[I] : 0.0) + coef * val;
  }
}

// ------------------------------------------------------------------ H.v ----

__device__ __forceinline__ double inter_term(const InterSpin &it, uint32_t up, uint32_t dn) {
  if (it.mode == 1) return it.u * (double)__popc(up & dn);
  double s = 0.0;
  if (it.mode == 2) {
    uint32_t w = up & dn;
    while (w) {
      int r = __ffs(w) - 1;
      s += __ldg(it.v + r);
      w &= w - 1;
    }
  } else if (it.mode == 3) {
    uint32_t wd = dn;
    while (wd) {
      int r = __ffs(wd) - 1;
      uint32_t wu = up;
      while (wu) {
        int c = __ffs(wu) - 1;
        s += __ldg(it.v + r * it.n + c);
        wu &= wu - 1;
      }
      wd &= wd - 1;
    }
  }
  return s;
}

// Dense Hamiltonian: thread I writes row I (diagonal, up hops along the row,
// dn hops across rows), the same matrix elements the H.v passes apply.
__global__ void k_dense_hamiltonian(HvOperator op, double *__restrict__ h) {
  const uint32_t du = op.up.dim, dd = op.dn.dim;
  const size_t D = (size_t)du * dd;
  for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < D; I += (size_t)gridDim.x * blockDim.x) {
    const uint32_t u = (uint32_t)(I % du), d = (uint32_t)(I / du);
    double *row = h + I * D;  // zeroed by the launcher
    row[I] = op.up.diag[u] + op.dn.diag[d] + inter_term(op.inter, op.up.bits[u], op.dn.bits[d]);
    for (int k = 0; k < op.up.cnt[u]; ++k) {
      const uint32_t e = op.up.ell[(size_t)k * du + u];
      row[(size_t)d * du + (e >> 8)] += op.up.vals[e & 255u];
    }
    for (int k = 0; k < op.dn.cnt[d]; ++k) {
      const uint32_t e = op.dn.ell[(size_t)k * dd + d];
      row[(size_t)(e >> 8) * du + u] += op.dn.vals[e & 255u];
    }
  }
}

// Row pass: one CTA per dn row (grid-stride). The row of x is staged in shared
// memory when it fits, so the up-spin gathers hit on-chip memory.
template <bool SMEM>
__global__ void __launch_bounds__(512) k_hv_rows(HvOperator op, const double *__restrict__ x,
                                                  double xs, double *y, SubList sub) {
  if (op.skip && *op.skip) return;
  extern __shared__ double xsm[];
  __shared__ double vals[256];
  const uint32_t du = op.up.dim, dd = op.dn.dim;
  for (int i = threadIdx.x; i < op.up.nvals; i += blockDim.x) vals[i] = op.up.vals[i];
  for (uint32_t d = blockIdx.x; d < dd; d += gridDim.x) {
    const double *xr = x + (size_t)d * du;
    if (SMEM) {
      __syncthreads();
      for (uint32_t u = threadIdx.x; u < du; u += blockDim.x) xsm[u] = xr[u];
    }
    __syncthreads();
    const uint32_t dnb = op.dn.bits[d];
    const double ddn = op.dn.diag[d];
    for (uint32_t u = threadIdx.x; u < du; u += blockDim.x) {
      const double diag = op.up.diag[u] + ddn + inter_term(op.inter, op.up.bits[u], dnb);
      double acc = diag * (SMEM ? xsm[u] : xr[u]);
      const int c = op.up.cnt[u];
      for (int k = 0; k < c; ++k) {
        const uint32_t e = __ldg(op.up.ell + (size_t)k * du + u);
        acc += vals[e & 255u] * (SMEM ? xsm[e >> 8] : __ldg(xr + (e >> 8)));
      }
      const size_t I = (size_t)d * du + u;
      acc *= xs;
      for (int s = 0; s < sub.n; ++s) acc -= (sub.cdev ? sub.cdev[s] : sub.c[s]) * sub.z[s][I];
      y[I] = acc;
    }
  }
}

// Column pass: work item = (column chunk, group of R rows), chunk-major so the
// CTAs in flight share one chunk of columns and the down-spin gathers of x
// rows hit L2. Each thread owns VEC adjacent columns.
template <int VEC, int R>
__global__ void __launch_bounds__(kThreads) k_hv_cols(HvOperator op, const double *__restrict__ x,
                                                       double xs, double *y, int red_mask,
                                                       double *partials) {
  if (op.skip && *op.skip) return;
  __shared__ double vals[256];
  const uint32_t du = op.up.dim, dd = op.dn.dim;
  for (int i = threadIdx.x; i < op.dn.nvals; i += blockDim.x) vals[i] = op.dn.vals[i];
  __syncthreads();
  const uint32_t W = VEC * blockDim.x;
  const uint32_t nchunk = (du + W - 1) / W, nrg = (dd + R - 1) / R;
  const size_t nitems = (size_t)nchunk * nrg;
  double red[3] = {0.0, 0.0, 0.0};
  for (size_t t = blockIdx.x; t < nitems; t += gridDim.x) {
    const uint32_t chunk = (uint32_t)(t / nrg), rg = (uint32_t)(t % nrg);
    const uint32_t u0 = chunk * W + VEC * threadIdx.x;
    if (u0 >= du) continue;
    for (int rr = 0; rr < R; ++rr) {
      const uint32_t d = rg * R + rr;
      if (d >= dd) break;
      const int c = op.dn.cnt[d];
      const size_t base = (size_t)d * du + u0;
      if (VEC == 2) {
        double2 acc = make_double2(0.0, 0.0);
        for (int k = 0; k < c; ++k) {
          const uint32_t e = __ldg(op.dn.ell + (size_t)k * dd + d);
          const double v = vals[e & 255u];
          const double2 xv = __ldg(reinterpret_cast<const double2 *>(x + (size_t)(e >> 8) * du + u0));
          acc.x += v * xv.x;
          acc.y += v * xv.y;
        }
        double2 yv = *reinterpret_cast<double2 *>(y + base);
        yv.x += xs * acc.x;
        yv.y += xs * acc.y;
        *reinterpret_cast<double2 *>(y + base) = yv;
        if (red_mask) {
          const double2 xv = __ldg(reinterpret_cast<const double2 *>(x + base));
          red[0] += xs * (xv.x * yv.x + xv.y * yv.y);
          red[1] += yv.x * yv.x + yv.y * yv.y;
          red[2] += xs * xs * (xv.x * xv.x + xv.y * xv.y);
        }
      } else {
        double acc = 0.0;
        for (int k = 0; k < c; ++k) {
          const uint32_t e = __ldg(op.dn.ell + (size_t)k * dd + d);
          acc += vals[e & 255u] * __ldg(x + (size_t)(e >> 8) * du + u0);
        }
        const double yv = y[base] + xs * acc;
        y[base] = yv;
        if (red_mask) {
          const double xv = x[base];
          red[0] += xs * xv * yv;
          red[1] += yv * yv;
          red[2] += xs * xs * xv * xv;
        }
      }
    }
  }
  if (red_mask) block_reduce_store<3>(red, partials, 3);
}

// Row pass, two dn rows per CTA step: the rows are staged interleaved in shared
// memory (one double2 per up string), so every hop-table entry and every
// shared-memory gather serves both rows, and the gathers are 16 bytes wide.
template <int UNROLL>
__global__ void __launch_bounds__(1024) k_hv_rows2(HvOperator op, const double *__restrict__ x,
                                                   double xs, double *y, SubList sub) {
  if (op.skip && *op.skip) return;
  extern __shared__ double2 xs2[];
  __shared__ double vals[256];
  const uint32_t du = op.up.dim, dd = op.dn.dim;
  for (int i = threadIdx.x; i < op.up.nvals; i += blockDim.x) vals[i] = op.up.vals[i];
  for (uint32_t d0 = 2 * blockIdx.x; d0 < dd; d0 += 2 * gridDim.x) {
    const bool two = d0 + 1 < dd;
    const double *x0 = x + (size_t)d0 * du;
    __syncthreads();
    for (uint32_t u = threadIdx.x; u < du; u += blockDim.x)
      xs2[u] = make_double2(x0[u], two ? x0[u + du] : 0.0);
    __syncthreads();
    const uint32_t b0 = op.dn.bits[d0], b1 = two ? op.dn.bits[d0 + 1] : 0u;
    const double e0 = op.dn.diag[d0], e1 = two ? op.dn.diag[d0 + 1] : 0.0;
    for (uint32_t u = threadIdx.x; u < du; u += blockDim.x) {
      const uint32_t ub = op.up.bits[u];
      const double dup = op.up.diag[u];
      const double2 xu = xs2[u];
      double a0 = (dup + e0 + inter_term(op.inter, ub, b0)) * xu.x;
      double a1 = (dup + e1 + inter_term(op.inter, ub, b1)) * xu.y;
      const int c = op.up.cnt[u];
      const uint32_t *ep = op.up.ell + u;
      int k = 0;
      for (; k + UNROLL <= c; k += UNROLL) {  // UNROLL independent gathers in flight
        uint32_t f[UNROLL];
#pragma unroll
        for (int q = 0; q < UNROLL; ++q) f[q] = __ldg(ep + (size_t)(k + q) * du);
#pragma unroll
        for (int q = 0; q < UNROLL; ++q) {
          const double2 t = xs2[f[q] >> 8];
          const double v = vals[f[q] & 255u];
          a0 += v * t.x;
          a1 += v * t.y;
        }
      }
      for (; k < c; ++k) {
        const uint32_t f0 = __ldg(ep + (size_t)k * du);
        const double2 t0 = xs2[f0 >> 8];
        const double v0 = vals[f0 & 255u];
        a0 += v0 * t0.x;
        a1 += v0 * t0.y;
      }
      const size_t I0 = (size_t)d0 * du + u;
      a0 *= xs;
      a1 *= xs;
      for (int s = 0; s < sub.n; ++s) {
        const double cs = sub.cdev ? sub.cdev[s] : sub.c[s];
        a0 -= cs * sub.z[s][I0];
        if (two) a1 -= cs * sub.z[s][I0 + du];
      }
      y[I0] = a0;
      if (two) y[I0 + du] = a1;
    }
  }
}

// Column pass with staged hop entries: the CTA decodes the hop entries of its
// R rows into shared memory once per work item, then every thread issues
// UNROLL independent 16-byte gathers of x row segments (from L2) at a time.
constexpr int kColsR = 4;
constexpr int kMaxHops = 256;

template <class T> __device__ __forceinline__ T gather_ld(const T *p, bool l2only) {
  return l2only ? __ldcg(p) : __ldg(p);
}

// Output rows [r0, r1) of the down-spin pass (every row: r0 = 0, r1 = dd); the
// gathers read every row of x.
template <int VEC, bool CG>
__global__ void __launch_bounds__(kThreads) k_hv_cols2(HvOperator op, const double *__restrict__ x,
                                                        double xs, double *y, int red_mask,
                                                        double *partials, uint32_t r0, uint32_t r1) {
  if (op.skip && *op.skip) return;
  __shared__ double cval[kColsR][kMaxHops];
  __shared__ uint32_t cidx[kColsR][kMaxHops];
  __shared__ int ccnt[kColsR];
  const uint32_t du = op.up.dim, dd = r1;
  const uint32_t W = VEC * blockDim.x;
  const uint32_t nchunk = (du + W - 1) / W, nrg = (r1 - r0 + kColsR - 1) / kColsR;
  const size_t nitems = (size_t)nchunk * nrg;
  double red[3] = {0.0, 0.0, 0.0};
  for (size_t t = blockIdx.x; t < nitems; t += gridDim.x) {
    const uint32_t chunk = (uint32_t)(t / nrg), rg = (uint32_t)(t % nrg);
    __syncthreads();  // the previous item is done with the staged entries
    if (threadIdx.x < kColsR) {
      const uint32_t d = r0 + rg * kColsR + threadIdx.x;
      ccnt[threadIdx.x] = d < dd ? (int)op.dn.cnt[d] : 0;
    }
    for (int j = threadIdx.x; j < kColsR * kMaxHops; j += blockDim.x) {
      const int rr = j / kMaxHops, k = j % kMaxHops;
      const uint32_t d = r0 + rg * kColsR + rr;
      if (d < dd && k < (int)op.dn.cnt[d]) {
        const uint32_t e = __ldg(op.dn.ell + (size_t)k * op.dn.dim + d);
        cval[rr][k] = op.dn.vals[e & 255u];
        cidx[rr][k] = e >> 8;
      }
    }
    __syncthreads();
    const uint32_t u0 = chunk * W + VEC * threadIdx.x;
    if (u0 >= du) continue;
    for (int rr = 0; rr < kColsR; ++rr) {
      const uint32_t d = r0 + rg * kColsR + rr;
      if (d >= dd) break;
      const int c = ccnt[rr];
      const size_t base = (size_t)d * du + u0;
      if (VEC == 2) {
        const double *xb = x + u0;
        double ax = 0.0, ay = 0.0;
        int k = 0;
        for (; k + 4 <= c; k += 4) {
          const double2 t0 = gather_ld(reinterpret_cast<const double2 *>(xb + (size_t)cidx[rr][k] * du), CG);
          const double2 t1 = gather_ld(reinterpret_cast<const double2 *>(xb + (size_t)cidx[rr][k + 1] * du), CG);
          const double2 t2 = gather_ld(reinterpret_cast<const double2 *>(xb + (size_t)cidx[rr][k + 2] * du), CG);
          const double2 t3 = gather_ld(reinterpret_cast<const double2 *>(xb + (size_t)cidx[rr][k + 3] * du), CG);
          ax += cval[rr][k] * t0.x + cval[rr][k + 1] * t1.x + cval[rr][k + 2] * t2.x + cval[rr][k + 3] * t3.x;
          ay += cval[rr][k] * t0.y + cval[rr][k + 1] * t1.y + cval[rr][k + 2] * t2.y + cval[rr][k + 3] * t3.y;
        }
        for (; k < c; ++k) {
          const double2 t0 = gather_ld(reinterpret_cast<const double2 *>(xb + (size_t)cidx[rr][k] * du), CG);
          ax += cval[rr][k] * t0.x;
          ay += cval[rr][k] * t0.y;
        }
        double2 yv = *reinterpret_cast<double2 *>(y + base);
        yv.x += xs * ax;
        yv.y += xs * ay;
        *reinterpret_cast<double2 *>(y + base) = yv;
        if (red_mask) {
          const double2 xv = __ldg(reinterpret_cast<const double2 *>(x + base));
          red[0] += xs * (xv.x * yv.x + xv.y * yv.y);
          red[1] += yv.x * yv.x + yv.y * yv.y;
          red[2] += xs * xs * (xv.x * xv.x + xv.y * xv.y);
        }
      } else {
        const double *xb = x + u0;
        double a = 0.0;
        int k = 0;
        for (; k + 4 <= c; k += 4) {
          const double t0 = __ldg(xb + (size_t)cidx[rr][k] * du), t1 = __ldg(xb + (size_t)cidx[rr][k + 1] * du);
          const double t2 = __ldg(xb + (size_t)cidx[rr][k + 2] * du), t3 = __ldg(xb + (size_t)cidx[rr][k + 3] * du);
          a += cval[rr][k] * t0 + cval[rr][k + 1] * t1 + cval[rr][k + 2] * t2 + cval[rr][k + 3] * t3;
        }
        for (; k < c; ++k) a += cval[rr][k] * __ldg(xb + (size_t)cidx[rr][k] * du);
        const double yv = y[base] + xs * a;
        y[base] = yv;
        if (red_mask) {
          const double xv = x[base];
          red[0] += xs * xv * yv;
          red[1] += yv * yv;
          red[2] += xs * xs * xv * xv;
        }
      }
    }
  }
  if (red_mask) block_reduce_store<3>(red, partials, 3);
}

// ------------------------------------------- staged-row H.v (packed hops) ----
//
// Both spins' hops gather from shared memory. The row pass stages two dn-rows
// of x (one double2 per up string) and applies the diagonal and the up hops;
// the column pass stages two columns of x (one double2 per dn string, all dn
// rows, brought in by TMA) and adds the down hops into y, which it reads and
// writes by TMA in chunks of rows. Hop entries are the 16-bit packed, bank-
// ordered tables of SpinTable::pk: target | sign << 14 | class << 15.

// Set by a kernel whose bounded wait on a TMA transaction gave up; the host
// reads it (check_device_waits) and reports the failure.
__device__ int g_wait_timeout = 0;

// One packed word (four hops of one magnitude class) gathered from the staged
// pairs at shared byte address base `sb`: p += sum_q (+-1) * st[target_q]. The
// target becomes a byte offset with one shift and one mask, the sign a +-1.0
// operand of the FMA (its high word from one LOP3). The gathers take 32-bit
// shared-window addresses (ld.shared with a 32-bit register), which saves the
// 64-bit address arithmetic of generic pointers (about 5 % of the H.v time).
__device__ __forceinline__ void hop_word(uint2 w, const char *sb, double2 &p) {
  const uint32_t o[4] = {(w.x << 4) & 0x3FFF0u, (w.x >> 12) & 0x3FFF0u, (w.y << 4) & 0x3FFF0u,
                         (w.y >> 12) & 0x3FFF0u};
  const uint32_t sh[4] = {((w.x << 16) & 0x80000000u) | 0x3FF00000u, (w.x & 0x80000000u) | 0x3FF00000u,
                          ((w.y << 16) & 0x80000000u) | 0x3FF00000u, (w.y & 0x80000000u) | 0x3FF00000u};
  double2 t[4];
  const uint32_t base = (uint32_t)__cvta_generic_to_shared(sb);
#pragma unroll
  for (int q = 0; q < 4; ++q)
    asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(t[q].x), "=d"(t[q].y) : "r"(base + o[q]));
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const double sg = __hiloint2double((int)sh[q], 0);
    p.x = fma(sg, t[q].x, p.x);
    p.y = fma(sg, t[q].y, p.y);
  }
}

// Hop words of one string, loaded ahead of its gathers: up to A0 / A1 words of
// each class in one batch of independent loads (the counts come one string
// earlier), so that a string costs one L2 round trip. The accumulation order
// does not depend on A0 / A1 (words alternate between two class-0 partial sums
// by their index), so every variant gives the same bits.
template <int A0, int A1> struct HopRow {
  uint2 a[A0], b[A1];
  uint32_t cw;
};

template <int A0, int A1>
__device__ __forceinline__ void load_row(const SpinTable &t, uint32_t stride, uint32_t i, uint32_t cw,
                                         HopRow<A0, A1> &h) {
  const uint32_t n0 = cw & 15u, n1 = cw >> 4;
  h.cw = cw;
#pragma unroll
  for (int k = 0; k < A0; ++k)
    if (k < (int)n0) h.a[k] = __ldg(t.pk[0] + (size_t)k * stride + i);
#pragma unroll
  for (int k = 0; k < A1; ++k)
    if (k < (int)n1) h.b[k] = __ldg(t.pk[1] + (size_t)k * stride + i);
}

// (a0, a1) += the hops of string i (both classes, magnitudes applied). The
// words past the loaded-ahead ones come two per step (A0 is even, so the even
// word of a step always goes to p0), with both loads issued first.
template <int A0, int A1>
__device__ __forceinline__ void apply_row(const HopRow<A0, A1> &h, const SpinTable &t, uint32_t stride, uint32_t i,
                                          const char *sb, double &a0, double &a1) {
  static_assert(A0 % 2 == 0, "class-0 words alternate between p0 and p1 by index");
  const int n0 = (int)(h.cw & 15u), n1 = (int)(h.cw >> 4);
  double2 p0 = make_double2(0.0, 0.0), p1 = make_double2(0.0, 0.0), q = make_double2(0.0, 0.0);
#pragma unroll
  for (int k = 0; k < A0; ++k)
    if (k < n0) hop_word(h.a[k], sb, (k & 1) ? p1 : p0);
  const uint2 *w0 = t.pk[0] + (size_t)A0 * stride + i;
  int k = A0;
  for (; k + 1 < n0; k += 2, w0 += 2 * (size_t)stride) {
    const uint2 wa = __ldg(w0), wb = __ldg(w0 + stride);
    hop_word(wa, sb, p0);
    hop_word(wb, sb, p1);
  }
  if (k < n0) hop_word(__ldg(w0), sb, p0);
#pragma unroll
  for (int j = 0; j < A1; ++j)
    if (j < n1) hop_word(h.b[j], sb, q);
  const uint2 *w1 = t.pk[1] + (size_t)A1 * stride + i;
  int j = A1;
  for (; j + 1 < n1; j += 2, w1 += 2 * (size_t)stride) {
    const uint2 wa = __ldg(w1), wb = __ldg(w1 + stride);
    hop_word(wa, sb, q);
    hop_word(wb, sb, q);
  }
  if (j < n1) hop_word(__ldg(w1), sb, q);
  a0 = fma(t.mag[0], p0.x + p1.x, fma(t.mag[1], q.x, a0));
  a1 = fma(t.mag[0], p0.y + p1.y, fma(t.mag[1], q.y, a1));
}

// Row pass: y = (diag + up hops) (xs x) - sub, two dn rows per CTA step (du even).
// Each thread walks its strings with the next string's hop words and basis data
// in flight while the current string gathers (and the counts one string further).
// RMW: y holds xs * (dn hops) x already (k_hv_cols16w) and is read back (also
// one string ahead); the reductions of the column pass (red_mask) are then
// taken here on the final y.
template <int THREADS, int A0, int A1, bool RMW>
__global__ void __launch_bounds__(THREADS, 1) k_hv_rows16(HvOperator op, const double *__restrict__ x, double xs,
                                                          double *y, SubList sub, int red_mask, double *partials) {
  if (op.skip && *op.skip) return;
  double red[3] = {0.0, 0.0, 0.0};
  extern __shared__ __align__(128) double2 st2[];
  const uint32_t du = op.up.dim, dd = op.dn.dim, hdu = du >> 1, T = THREADS;
  const char *sb = reinterpret_cast<const char *>(st2);
  if (threadIdx.x < 8) st2[du + threadIdx.x] = make_double2(0.0, 0.0);  // padding targets
  for (uint32_t d0 = 2 * blockIdx.x; d0 < dd; d0 += 2 * gridDim.x) {
    const bool two = d0 + 1 < dd;
    const double2 *r0 = reinterpret_cast<const double2 *>(x + (size_t)d0 * du);
    const double2 *r1 = reinterpret_cast<const double2 *>(x + (size_t)(d0 + (two ? 1 : 0)) * du);
    const size_t row0 = (size_t)d0 * du;
    HopRow<A0, A1> cur;
    uint32_t ub = 0, cw1 = 0;
    double dup = 0.0, yo0 = 0.0, yo1 = 0.0;
    const uint32_t u0 = threadIdx.x;  // the first string's loads overlap the staging
    if (u0 < du) {
      load_row(op.up, du, u0, op.up.cntw[u0], cur);
      ub = op.up.bits[u0];
      dup = op.up.diag[u0];
      if (RMW) {
        yo0 = y[row0 + u0];
        if (two) yo1 = y[row0 + du + u0];
      }
    }
    if (u0 + T < du) cw1 = op.up.cntw[u0 + T];
    __syncthreads();  // every thread is done with the previous pair
    for (uint32_t q = threadIdx.x; q < hdu; q += T) {
      const double2 a = r0[q];
      const double2 b = two ? r1[q] : make_double2(0.0, 0.0);
      st2[2 * q] = make_double2(a.x, b.x);
      st2[2 * q + 1] = make_double2(a.y, b.y);
    }
    __syncthreads();
    const uint32_t b0 = op.dn.bits[d0], b1 = two ? op.dn.bits[d0 + 1] : 0u;
    const double e0 = op.dn.diag[d0], e1 = two ? op.dn.diag[d0 + 1] : 0.0;
    for (uint32_t u = u0; u < du; u += T) {
      const uint32_t un = u + T;
      HopRow<A0, A1> nxt;
      uint32_t ubn = 0, cw2 = 0;
      double dupn = 0.0, yn0 = 0.0, yn1 = 0.0;
      if (un < du) {
        load_row(op.up, du, un, cw1, nxt);
        ubn = op.up.bits[un];
        dupn = op.up.diag[un];
        if (RMW) {
          yn0 = y[row0 + un];
          if (two) yn1 = y[row0 + du + un];
        }
        if (un + T < du) cw2 = op.up.cntw[un + T];
      }
      const double2 xu = st2[u];
      double a0 = (dup + e0 + inter_term(op.inter, ub, b0)) * xu.x;
      double a1 = (dup + e1 + inter_term(op.inter, ub, b1)) * xu.y;
      apply_row(cur, op.up, du, u, sb, a0, a1);
      const size_t I0 = row0 + u;
      a0 *= xs;
      a1 *= xs;
      for (int s = 0; s < sub.n; ++s) {
        const double cs = sub.cdev ? sub.cdev[s] : sub.c[s];
        a0 -= cs * sub.z[s][I0];
        if (two) a1 -= cs * sub.z[s][I0 + du];
      }
      if (RMW) {
        a0 += yo0;
        a1 += yo1;
        if (red_mask) {
          red[0] += xs * (xu.x * a0 + (two ? xu.y * a1 : 0.0));
          red[1] += a0 * a0 + (two ? a1 * a1 : 0.0);
          red[2] += xs * xs * (xu.x * xu.x + xu.y * xu.y);
        }
      }
      y[I0] = a0;
      if (two) y[I0 + du] = a1;
      cur = nxt;
      ub = ubn;
      dup = dupn;
      cw1 = cw2;
      yo0 = yn0;
      yo1 = yn1;
    }
  }
  if (RMW && red_mask) block_reduce_store<3>(red, partials, 3);
}

// ---- TMA and mbarrier helpers (1-CTA clusters; no multicast) ----

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for the phase of parity `parity` of bar to complete; gives up after
// about two seconds, records the timeout and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
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
      const uint64_t t = global_ns();
      if (it == 0) t0 = t;
      else if (t - t0 > 2000000000ull) {
        atomicExch(&g_wait_timeout, 1);
        return false;
      }
    }
  }
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int c0, int c1, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
      ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tma_store_2d(const CUtensorMap *map, int c0, int c1, const void *src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];"
               ::"l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(src))
               : "memory");
}

__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_read_all() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

constexpr int kSliceRows = 32;  // rows of one warp's TMA store
constexpr int kTmaBoxRows = 256;

// Column pass, write form: y = xs * (dn hops) x. Work item = one column pair
// (u0, u0 + 1): its x values for all dn rows are TMA-loaded into shared memory
// (box 2 x 256, zero-filled past dd, which also clears the padding targets
// dd .. dd + 7, or they are cleared once below). Each warp then takes slices of
// 32 rows, one row per lane, and sends each slice out with its own TMA store
// (box 2 x 32) from its 512-byte staging slot; no CTA barrier inside a column
// pair. The lanes load the hop words of their next row while gathering.
template <int THREADS, int A0, int A1>
__global__ void __launch_bounds__(THREADS, 1)
    k_hv_cols16w(const __grid_constant__ CUtensorMap tmx, const __grid_constant__ CUtensorMap tmy, HvOperator op,
                 double xs) {
  if (op.skip && *op.skip) return;
  extern __shared__ __align__(1024) unsigned char sm_raw[];
  const uint32_t du = op.up.dim, dd = op.dn.dim;
  const uint32_t nbox = (dd + kTmaBoxRows - 1) / kTmaBoxRows;
  const uint32_t nst = nbox * kTmaBoxRows + 8;
  constexpr uint32_t nwarps = THREADS / 32;
  double2 *st2 = reinterpret_cast<double2 *>(sm_raw);
  double2 *ob = st2 + nst;  // one slot per thread: a warp's slots are its slice buffer
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint64_t *bar = reinterpret_cast<uint64_t *>(ob + THREADS);
  double2 *buf = ob + warp * kSliceRows;
  const char *sb = reinterpret_cast<const char *>(st2);
  const uint32_t npairs = du >> 1;
  const uint32_t nslice = (dd + kSliceRows - 1) / kSliceRows;
  const uint32_t step = nwarps * kSliceRows;
  if (threadIdx.x < 8) st2[nbox * kTmaBoxRows + threadIdx.x] = make_double2(0.0, 0.0);
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init_fence();
  }
  __syncthreads();
  uint32_t px = 0;
  for (uint32_t pp = blockIdx.x; pp < npairs; pp += gridDim.x) {
    const int u0 = (int)(2 * pp);
    if (threadIdx.x == 0) {
      mbar_expect_tx(&bar[0], nbox * kTmaBoxRows * 16);
      for (uint32_t b = 0; b < nbox; ++b)
        tma_load_2d(st2 + b * kTmaBoxRows, &tmx, u0, (int)(b * kTmaBoxRows), &bar[0]);
    }
    // the first row's hop words (the table does not depend on x) while x arrives
    uint32_t d = warp * kSliceRows + lane;
    HopRow<A0, A1> cur;
    uint32_t cw1 = 0;
    if (d < dd) load_row(op.dn, dd, d, op.dn.cntw[d], cur);
    if (d + step < dd) cw1 = op.dn.cntw[d + step];
    // every thread takes the same branch, also when the wait gave up
    if (!__syncthreads_and(mbar_wait(&bar[0], px))) break;
    px ^= 1u;
    for (uint32_t sl = warp; sl < nslice; sl += nwarps, d += step) {
      HopRow<A0, A1> nxt;
      uint32_t cw2 = 0;
      if (d + step < dd) {
        load_row(op.dn, dd, d + step, cw1, nxt);
        if (d + 2 * step < dd) cw2 = op.dn.cntw[d + 2 * step];
      }
      double a0 = 0.0, a1 = 0.0;
      if (d < dd) apply_row(cur, op.dn, dd, d, sb, a0, a1);
      if (lane == 0) bulk_wait_read_all();  // the warp's previous store has read the slot
      __syncwarp();
      buf[lane] = make_double2(xs * a0, xs * a1);
      fence_proxy_async_smem();  // the lane's write is visible to the TMA store
      __syncwarp();
      if (lane == 0) {
        tma_store_2d(&tmy, u0, (int)(sl * kSliceRows), buf);  // rows past dd are clipped
        bulk_commit();
      }
      cur = nxt;
      cw1 = cw2;
    }
    __syncthreads();  // every warp is done with st2 before the next pair's loads
  }
  if (lane == 0) bulk_wait_all();  // stores complete while the staging slots are still ours
}

// ---- matrix continued fractions --------------------------------------------
//
// One CTA per (frequency, fraction): the backward recursion of the p x p complex
// floors in shared memory, each floor inverted by Gauss-Jordan elimination with
// partial pivoting on the augmented matrix [D | I].

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__global__ void __launch_bounds__(256) k_mcf_eval(const McfDesc *desc, const double *blob, int q, int nz,
                                                  const double *z, double *out) {
  const McfDesc d = desc[blockIdx.y];
  const int k = blockIdx.x, p = d.p, pp = p * p, t = threadIdx.x, nt = blockDim.x;
  const double zr = z[2 * k], zi = z[2 * k + 1];
  __shared__ double2 F[kMcfMaxP * kMcfMaxP], T1[kMcfMaxP * kMcfMaxP];
  __shared__ double2 Aug[kMcfMaxP][2 * kMcfMaxP];
  __shared__ double2 fac[kMcfMaxP];
  __shared__ int piv;
  for (int i = t; i < pp; i += nt) F[i] = make_double2(0.0, 0.0);
  __syncthreads();
  for (int j = d.M - 1; j >= 0; --j) {
    const double *A = blob + d.offA + (size_t)j * pp, *B = blob + d.offB + (size_t)j * pp;
    const bool tail = j < d.M - 1;  // B_{M-1} is the truncation residual, not used
    if (tail) {
      for (int i = t; i < pp; i += nt) {  // T1 = F B_j
        const int r = i / p, c = i % p;
        double2 acc = make_double2(0.0, 0.0);
        for (int a = 0; a < p; ++a) {
          const double b = B[a * p + c];
          acc.x += F[r * p + a].x * b;
          acc.y += F[r * p + a].y * b;
        }
        T1[i] = acc;
      }
      __syncthreads();
    }
    for (int i = t; i < 2 * pp; i += nt) {  // Aug = [z - A_j - B_j^T T1 | I]
      const int r = i / (2 * p), c = i % (2 * p);
      double2 v;
      if (c < p) {
        double2 sg = make_double2(0.0, 0.0);
        if (tail)
          for (int a = 0; a < p; ++a) {
            const double b = B[a * p + r];
            sg.x += b * T1[a * p + c].x;
            sg.y += b * T1[a * p + c].y;
          }
        v = make_double2((r == c ? zr : 0.0) - A[r * p + c] - sg.x, (r == c ? zi : 0.0) - sg.y);
      } else {
        v = make_double2(r == c - p ? 1.0 : 0.0, 0.0);
      }
      Aug[r][c] = v;
    }
    __syncthreads();
    for (int c = 0; c < p; ++c) {
      if (t == 0) {
        int best = c;
        double bm = Aug[c][c].x * Aug[c][c].x + Aug[c][c].y * Aug[c][c].y;
        for (int r = c + 1; r < p; ++r) {
          const double m = Aug[r][c].x * Aug[r][c].x + Aug[r][c].y * Aug[r][c].y;
          if (m > bm) {
            bm = m;
            best = r;
          }
        }
        piv = best;
      }
      __syncthreads();
      const int pr = piv;
      if (pr != c)
        for (int i = t; i < 2 * p; i += nt) {
          const double2 tmp = Aug[c][i];
          Aug[c][i] = Aug[pr][i];
          Aug[pr][i] = tmp;
        }
      __syncthreads();
      const double2 pv = Aug[c][c];
      const double den = pv.x * pv.x + pv.y * pv.y;
      const double2 inv = make_double2(pv.x / den, -pv.y / den);
      __syncthreads();  // every thread has read the pivot
      for (int i = t; i < 2 * p; i += nt) Aug[c][i] = cmul(Aug[c][i], inv);
      if (t < p) fac[t] = Aug[t][c];
      __syncthreads();
      for (int i = t; i < 2 * pp; i += nt) {
        const int r = i / (2 * p), col = i % (2 * p);
        if (r == c) continue;
        const double2 m = cmul(fac[r], Aug[c][col]);
        Aug[r][col].x -= m.x;
        Aug[r][col].y -= m.y;
      }
      __syncthreads();
    }
    for (int i = t; i < pp; i += nt) F[i] = Aug[i / p][p + i % p];
    __syncthreads();
  }
  // G = W^T F_0 W
  const double *W = blob + d.offW;
  double *o = out + ((size_t)blockIdx.y * nz + k) * (size_t)q * q * 2;
  for (int i = t; i < q * q; i += nt) {
    const int a = i / q, b = i % q;
    double2 acc = make_double2(0.0, 0.0);
    for (int r = 0; r < p; ++r) {
      const double wa = W[r * q + a];
      if (wa == 0.0) continue;
      double2 row = make_double2(0.0, 0.0);
      for (int c = 0; c < p; ++c) {
        const double wb = W[c * q + b];
        row.x += F[r * p + c].x * wb;
        row.y += F[r * p + c].y * wb;
      }
      acc.x += wa * row.x;
      acc.y += wa * row.y;
    }
    const size_t idx = d.transpose ? (size_t)b * q + a : (size_t)a * q + b;
    o[2 * idx] = acc.x;
    o[2 * idx + 1] = acc.y;
  }
}

// ---- block H.v on separate vectors (sectors without packed tables) ----
//
// A block of p <= 16 vectors (pointer arrays) through the ELL tables: one
// thread per state applies every hop to all p vectors, so each table entry is
// read once per state for the whole block. Row pass: Y_c = (diag + up hops) X_c;
// column pass: Y_c += (dn hops) X_c. Small sectors are launch-bound, where one
// launch per pass for the whole block is what counts.
template <int P>
__global__ void __launch_bounds__(kThreads) k_blhv_rows(HvOperator op, int p, BlockIn X, BlockOut Y) {
  const uint32_t du = op.up.dim, dd = op.dn.dim;
  const size_t D = (size_t)du * dd;
  for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < D; I += (size_t)gridDim.x * blockDim.x) {
    const uint32_t u = (uint32_t)(I % du), d = (uint32_t)(I / du);
    const double dg = op.up.diag[u] + op.dn.diag[d] + inter_term(op.inter, op.up.bits[u], op.dn.bits[d]);
    const size_t row = (size_t)d * du;
    double acc[P];
#pragma unroll
    for (int c = 0; c < P; ++c) acc[c] = c < p ? dg * X.v[c][I] : 0.0;
    const int cu = op.up.cnt[u];
    for (int k = 0; k < cu; ++k) {
      const uint32_t e = __ldg(op.up.ell + (size_t)k * du + u);
      const double v = op.up.vals[e & 255u];
      const size_t J = row + (e >> 8);
#pragma unroll
      for (int c = 0; c < P; ++c)
        if (c < p) acc[c] += v * X.v[c][J];
    }
#pragma unroll
    for (int c = 0; c < P; ++c)
      if (c < p) Y.v[c][I] = acc[c];
  }
}

template <int P>
__global__ void __launch_bounds__(kThreads) k_blhv_cols(HvOperator op, int p, BlockIn X, BlockOut Y) {
  const uint32_t du = op.up.dim, dd = op.dn.dim;
  const size_t D = (size_t)du * dd;
  for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < D; I += (size_t)gridDim.x * blockDim.x) {
    const uint32_t u = (uint32_t)(I % du), d = (uint32_t)(I / du);
    double acc[P];
#pragma unroll
    for (int c = 0; c < P; ++c) acc[c] = 0.0;
    const int cd = op.dn.cnt[d];
    for (int k = 0; k < cd; ++k) {
      const uint32_t e = __ldg(op.dn.ell + (size_t)k * dd + d);
      const double v = op.dn.vals[e & 255u];
      const size_t J = (size_t)(e >> 8) * du + u;
#pragma unroll
      for (int c = 0; c < P; ++c)
        if (c < p) acc[c] += v * X.v[c][J];
    }
#pragma unroll
    for (int c = 0; c < P; ++c)
      if (c < p) Y.v[c][I] += acc[c];
  }
}

// --------------------------------------------------------- vector kernels ----

template <int G>
__global__ void k_dots(size_t D, double *x, double xs, int write_x, VecList ys, int first,
                       double *partials) {
  if (ys.skip && *ys.skip) return;
  if (ys.xsdev && first == 0) xs = *ys.xsdev;
  double acc[G];
#pragma unroll
  for (int g = 0; g < G; ++g) acc[g] = 0.0;
  const int n = min(G, ys.n - first);
  for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < D; I += (size_t)gridDim.x * blockDim.x) {
    double xv = x[I] * xs;
    if (write_x) x[I] = xv;
#pragma unroll
    for (int g = 0; g < G; ++g)
      if (g < n) acc[g] += xv * ys.v[first + g][I];
  }
  // store into slots first..first+n
  __shared__ double sm[G][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int g = 0; g < G; ++g) {
    double v = acc[g];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) sm[g][warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < n) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += sm[threadIdx.x][w];
    partials[(size_t)blockIdx.x * Reducer::kMaxRed + first + threadIdx.x] = s;
  }
}

__global__ void k_multi_axpy(size_t D, const double *x, double xs, VecList ys, int norm_first,
                             double *partials) {
  if (ys.skip && *ys.skip) return;
  double nrm[1] = {0.0};
  for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < D; I += (size_t)gridDim.x * blockDim.x) {
    const double xv = x[I] * xs;
    for (int i = 0; i < ys.n; ++i) {
      double v = ys.v[i][I] - (ys.cdev ? ys.cdev[i] : ys.c[i]) * xv;
      ys.v[i][I] = v;
      if (i == 0 && norm_first) nrm[0] += v * v;
    }
  }
  if (norm_first) block_reduce_store<1>(nrm, partials, 1);
}

__global__ void k_axpby(size_t D, double a, double *y, double b, const double *x, int norm,
                        double *partials) {
  double nrm[1] = {0.0};
  for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < D; I += (size_t)gridDim.x * blockDim.x) {
    double v = (a != 0.0 ? a * y[I] : 0.0) + (x ? b * x[I] : 0.0);
    y[I] = v;
    nrm[0] += v * v;
  }
  if (norm) block_reduce_store<1>(nrm, partials, 1);
}

__global__ void k_axpy_dev(size_t D, double *y, const double *x, const double *a_dev, double *partials,
                           const int *skip) {
  if (skip && *skip) return;
  const double b = -*a_dev;
  double nrm[1] = {0.0};
  for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < D; I += (size_t)gridDim.x * blockDim.x) {
    const double v = y[I] + b * x[I];
    y[I] = v;
    nrm[0] += v * v;
  }
  block_reduce_store<1>(nrm, partials, 1);
}

__global__ void k_lanczos_advance(size_t D, double *y, LanczosScalars ls) {
  const double b = sqrt(*ls.b2_cur);
  const double z = (b > 0.0) ? 1.0 / b : 0.0;
  for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < D; I += (size_t)gridDim.x * blockDim.x)
    y[I] *= z;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int j = *ls.j;
    ls.alpha_hist[j] = *ls.alpha_cur;
    ls.beta_hist[j] = b;
    *ls.beta_prev = b;
    *ls.j = j + 1;
  }
}

// Sum over the CTA in a fixed order (warp shuffles, then warp 0 over the warp
// sums); every thread gets the total. sm: at least 33 doubles of shared memory.
__device__ __forceinline__ double cta_sum(double v, double *sm) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  __syncthreads();  // previous use of sm is complete
  if (lane == 0) sm[warp] = v;
  __syncthreads();
  if (warp == 0) {
    double t = lane < nw ? sm[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) sm[32] = t;
  }
  __syncthreads();
  return sm[32];
}

// One sector per CTA; the job descriptor is staged in shared memory.
__device__ __forceinline__ uint64_t splitmix64(uint64_t z);

__global__ void __launch_bounds__(kLanczosJobThreads) k_lanczos_start_jobs(const LanczosJob *__restrict__ jobs) {
  __shared__ LanczosJob J;
  __shared__ double sm[33];
  if (threadIdx.x == 0) J = jobs[blockIdx.x];
  __syncthreads();
  const uint32_t D = J.op.up.dim * J.op.dn.dim;
  double *vp = J.v[J.rot], *vc = J.v[(J.rot + 1) % 3];
  const uint64_t key = splitmix64(J.seed ^ 0x5eedull);
  double s2 = 0.0;
  for (uint32_t I = threadIdx.x; I < D; I += blockDim.x) {
    uint64_t h1 = splitmix64(key + 2 * (uint64_t)I), h2 = splitmix64(key + 2 * (uint64_t)I + 1);
    double u1 = ((h1 >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    double u2 = (h2 >> 11) * (1.0 / 9007199254740992.0);
    const double v = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    vc[I] = v;
    vp[I] = 0.0;
    s2 += v * v;
  }
  const double nrm = sqrt(cta_sum(s2, sm));
  const double z = nrm > 0.0 ? 1.0 / nrm : 0.0;
  for (uint32_t I = threadIdx.x; I < D; I += blockDim.x) vc[I] *= z;
  if (threadIdx.x == 0) *J.beta_prev = 0.0;
}

__global__ void __launch_bounds__(kLanczosJobThreads) k_lanczos_jobs(const LanczosJob *__restrict__ jobs) {
  __shared__ LanczosJob J;
  __shared__ double sm[33];
  if (threadIdx.x == 0) J = jobs[blockIdx.x];
  __syncthreads();
  const uint32_t du = J.op.up.dim, dd = J.op.dn.dim;
  const uint32_t D = du * dd;
  double *vp = J.v[J.rot], *vc = J.v[(J.rot + 1) % 3], *w = J.v[(J.rot + 2) % 3];
  for (int step = 0; step < J.nsteps; ++step) {
    const double bprev = *J.beta_prev;
    double sa = 0.0;
    for (uint32_t I = threadIdx.x; I < D; I += blockDim.x) {
      const uint32_t u = I % du, d = I / du;
      const double x = vc[I];
      double acc = (J.op.up.diag[u] + J.op.dn.diag[d] + inter_term(J.op.inter, J.op.up.bits[u], J.op.dn.bits[d])) * x;
      const double *row = vc + (size_t)d * du;
      for (int k = 0; k < J.op.up.cnt[u]; ++k) {
        const uint32_t e = J.op.up.ell[(size_t)k * du + u];
        acc += J.op.up.vals[e & 255u] * row[e >> 8];
      }
      for (int k = 0; k < J.op.dn.cnt[d]; ++k) {
        const uint32_t e = J.op.dn.ell[(size_t)k * dd + d];
        acc += J.op.dn.vals[e & 255u] * vc[(size_t)(e >> 8) * du + u];
      }
      acc -= bprev * vp[I];
      w[I] = acc;
      sa += x * acc;
    }
    const double a = cta_sum(sa, sm);  // alpha_j = <v_j, w>
    double sb = 0.0;
    for (uint32_t I = threadIdx.x; I < D; I += blockDim.x) {
      const double t = w[I] - a * vc[I];
      w[I] = t;
      sb += t * t;
    }
    const double b = sqrt(cta_sum(sb, sm));  // beta_j = |w|
    const double z = (b > 0.0) ? 1.0 / b : 0.0;
    for (uint32_t I = threadIdx.x; I < D; I += blockDim.x) w[I] *= z;
    if (threadIdx.x == 0) {
      J.out[step] = a;
      J.out[kLanczosJobMaxSteps + step] = b;
      *J.beta_prev = b;
    }
    __syncthreads();  // v_{j+1} and beta_j visible to the whole CTA
    double *t = vp;
    vp = vc;
    vc = w;
    w = t;
  }
}

__global__ void k_swap_scale(size_t D, double *q, double *p, double beta) {
  const double z = 1.0 / beta;
  for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < D; I += (size_t)gridDim.x * blockDim.x) {
    const double t = p[I];
    p[I] = q[I] * z;
    q[I] = -beta * t;
  }
}

__device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
  z += 0x9e3779b97f4a7c15ull;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

__global__ void k_random(size_t D, uint64_t seed, double *y, double *partials) {
  double nrm[1] = {0.0};
  const uint64_t key = splitmix64(seed ^ 0x5eedull);
  for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < D; I += (size_t)gridDim.x * blockDim.x) {
    // Box-Muller on two 53-bit uniforms from a counter-based hash
    uint64_t h1 = splitmix64(key + 2 * I), h2 = splitmix64(key + 2 * I + 1);
    double u1 = ((h1 >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    double u2 = (h2 >> 11) * (1.0 / 9007199254740992.0);
    double v = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    y[I] = v;
    nrm[0] += v * v;
  }
  block_reduce_store<1>(nrm, partials, 1);
}

__global__ void k_scale_dev(size_t D, double *y, const double *a_dev, const int *skip) {
  if (skip && *skip) return;
  const double a = *a_dev;
  for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < D; I += (size_t)gridDim.x * blockDim.x)
    y[I] *= a;
}

// Band-Lanczos norm step: z = sqrt(sum of partials); below the deflation
// tolerance it raises *flag (step + 1) and leaves everything else alone,
// otherwise it stores z and 1/z.
__global__ void k_finalize_norm(const double *partials, int nblocks, double dtol, double *z_out,
                                double *inv_out, int *flag, int step) {
  __shared__ double sm[kThreads];
  double s = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partials[(size_t)b * Reducer::kMaxRed];
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0 && *flag == 0) {
    const double z = sqrt(sm[0]);
    if (z < dtol) {
      *flag = step + 1;
    } else {
      *z_out = z;
      *inv_out = 1.0 / z;
    }
  }
}

__global__ void k_scale(size_t D, double *y, double a) {
  for (size_t I = blockIdx.x * (size_t)blockDim.x + threadIdx.x; I < D; I += (size_t)gridDim.x * blockDim.x)
    y[I] *= a;
}

// ------------------------------------------------ block (p-vector) kernels ----
// A block holds p vectors interleaved: element (I, c) at I * p + c. P (a power
// of two, p <= P <= 16) threads serve one basis state, thread c its column c,
// so every gather of the block H.v reads the p values of one state at once.

// out[slot] = sum over blocks of partials[b * ld + slot], slot < n, fixed order.
__global__ void k_finalize_ld(const double *partials, int nblocks, int ld, double *out) {
  __shared__ double sm[kThreads];
  const int slot = blockIdx.x;
  double s = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += partials[(size_t)b * ld + slot];
  sm[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[slot] = sm[0];
}

// Cholesky factor of a p x p Gram matrix (p <= 16, row-major): R upper
// triangular with G = R^T R, and R^{-1}; the kernel exists so that the block
// recurrence needs no host round trip for its QR. One CTA of 256 threads,
// thread (r, c) owning entry r * p + c: p right-looking elimination steps in
// shared memory (each entry receives the same subtractions, in the same order,
// as the row-by-row host factorisation), then one back substitution per column
// of R^{-1}. A diagonal that is not positive, or a pivot below pivot_min, sets
// *fail_flag = 1 and zeroes R^{-1}. With Rprev given, also B = R Rprev (upper
// triangular) into B_out and its transpose into Bt_out.
__global__ void __launch_bounds__(256) k_block_chol(int p, const double *G, double pivot_min, double *R,
                                                    double *Rinv, const double *Rprev, double *B_out,
                                                    double *Bt_out, double *fail_flag) {
  __shared__ double a[256], ri[256];
  __shared__ int bad;
  const int t = threadIdx.x, pp = p * p;
  const int r = t / p, c = t - (t / p) * p;  // valid for t < pp
  if (t < pp) a[t] = G[t];
  if (t == 0) bad = 0;
  __syncthreads();
  for (int i = 0; i < p; ++i) {
    __syncthreads();                // the updates of step i - 1 are done
    const double d = a[i * p + i];  // fully updated by steps 0..i-1
    const bool ok = d > 0.0;
    const double rii = ok ? sqrt(d) : 1.0;
    if (t == 0 && (!ok || rii < pivot_min)) bad = 1;
    __syncthreads();  // everyone has read a[i][i]
    if (t < pp && r == i) a[t] = (c == i) ? rii : (c > i ? a[t] / rii : 0.0);
    __syncthreads();  // row i of R is final
    if (t < pp && r > i && c >= r) a[t] -= a[i * p + r] * a[i * p + c];
  }
  __syncthreads();
  // R^{-1}: column c by back substitution from row c up (thread c)
  if (t < p) {
    for (int i = t; i >= 0; --i) {
      double acc = 0.0;
      for (int k = i + 1; k <= t; ++k) acc += a[i * p + k] * ri[k * p + t];
      ri[i * p + t] = (i == t) ? 1.0 / a[i * p + i] : -acc / a[i * p + i];
    }
    for (int i = t + 1; i < p; ++i) ri[i * p + t] = 0.0;
  }
  __syncthreads();
  if (t < pp) {
    const double rv = (c >= r) ? a[t] : 0.0;
    R[t] = rv;
    Rinv[t] = bad ? 0.0 : ri[t];
    if (Rprev) {
      double acc = 0.0;
      for (int k = r; k <= c; ++k) acc += a[r * p + k] * Rprev[k * p + c];
      const double b = (c >= r) ? acc : 0.0;
      B_out[t] = b;
      Bt_out[c * p + r] = b;
    }
  }
  if (t == 0 && bad) *fail_flag = 1.0;
}

// -------------------------------------------------------- Green functions ----

// G(z) of a Lehmann representation for a batch of frequencies: one CTA per
// frequency; poles are streamed through shared memory in chunks.
// (Q_matrix::Green_function + VDVH kernel, src_ed/Q_matrix.hpp:133-151,
//  src_util/VDVH_kernel.cpp:28-36)
__global__ void k_qmatrix_gf(int L, int M, const double *e, const double *V, int nz,
                             const double *z, double *G) {
  constexpr int CH = 64;
  __shared__ double vs[64 * CH];
  __shared__ double ur[CH], ui[CH];
  const int k = blockIdx.x;
  const double zr = z[2 * k], zi = z[2 * k + 1];
  const int LL = L * L;
  for (int pbase = 0; pbase < LL; pbase += blockDim.x) {
    const int pidx = pbase + threadIdx.x;
    const int a = pidx / L, b = pidx % L;
    double gr = 0.0, gi = 0.0;
    for (int i0 = 0; i0 < M; i0 += CH) {
      const int nc = min(CH, M - i0);
      __syncthreads();
      for (int t = threadIdx.x; t < nc * L; t += blockDim.x) vs[t] = V[(size_t)i0 * L + t];
      for (int t = threadIdx.x; t < nc; t += blockDim.x) {
        double dr = zr - e[i0 + t], di = zi;
        double den = dr * dr + di * di;
        ur[t] = dr / den;
        ui[t] = -di / den;
      }
      __syncthreads();
      if (pidx < LL) {
        for (int i = 0; i < nc; ++i) {
          double w = vs[i * L + a] * vs[i * L + b];
          gr += w * ur[i];
          gi += w * ui[i];
        }
      }
    }
    if (pidx < LL) {
      double *g = G + 2 * ((size_t)k * LL + b + (size_t)a * L);
      g[0] += gr;
      g[1] += gi;
    }
  }
}

// Integrand of the self-energy functional on a (frequency, wavevector) grid
// (lattice_model_instance::SEF_integrand_k, src_qcm/lattice_model_instance.cpp:618-640,
// summed as in Potthoff_functional's grid path, :520-545): for each frequency
// w and each k = (i/nkx, j/nky, l/nkz) of the reduced zone,
//   V(k) = V0 + sum_e v_e exp(2 pi i k.R_e) at (r_e, c_e)   (set_V, src_qcm/CPT.cpp:22-64)
//   I(w, k) = log |det(V(k) G(iw) - 1)|.
// One thread per (w, k): V(k), V G - 1 and its LU factorisation with partial
// pivoting live in the thread's local memory (n <= 16 complex); each CTA adds
// its threads' values in a fixed order into partials[w * nblk + block].
constexpr int kSefMaxN = 16;
constexpr int kSefThreads = 128;
__global__ void __launch_bounds__(kSefThreads) k_sef_logdet(int n, const double *__restrict__ G,
                                                            const double *__restrict__ V0, int nel,
                                                            const int *__restrict__ er, const int *__restrict__ ec,
                                                            const double *__restrict__ eR,
                                                            const double *__restrict__ ev, int nkx, int nky, int nkz,
                                                            double *partials) {
  __shared__ double red[kSefThreads];
  const int iw = blockIdx.y;
  const long nk = (long)nkx * nky * nkz;
  const long kid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double val = 0.0;
  if (kid < nk) {
    const int ix = (int)(kid / ((long)nky * nkz)), iy = (int)((kid / nkz) % nky), iz = (int)(kid % nkz);
    const double kx = (double)ix / nkx, ky = (double)iy / nky, kz = (double)iz / nkz;
    double vr[kSefMaxN * kSefMaxN], vi[kSefMaxN * kSefMaxN];  // column-major n x n
    for (int t = 0; t < n * n; ++t) {
      vr[t] = V0[2 * t];
      vi[t] = V0[2 * t + 1];
    }
    for (int e = 0; e < nel; ++e) {
      double s, c;
      sincospi(2.0 * (kx * eR[3 * e] + ky * eR[3 * e + 1] + kz * eR[3 * e + 2]), &s, &c);
      const double ar = ev[2 * e], ai = ev[2 * e + 1];
      const int t = er[e] + n * ec[e];
      vr[t] += ar * c - ai * s;
      vi[t] += ar * s + ai * c;
    }
    // M = V G - 1 (column-major); G of this frequency, column-major
    const double *g = G + 2 * (size_t)iw * n * n;
    double mr[kSefMaxN * kSefMaxN], mi[kSefMaxN * kSefMaxN];
    for (int b = 0; b < n; ++b)
      for (int a = 0; a < n; ++a) {
        double sr = (a == b) ? -1.0 : 0.0, si = 0.0;
        for (int c = 0; c < n; ++c) {
          const double xr = vr[a + n * c], xi = vi[a + n * c];
          const double yr = g[2 * (c + n * b)], yi = g[2 * (c + n * b) + 1];
          sr += xr * yr - xi * yi;
          si += xr * yi + xi * yr;
        }
        mr[a + n * b] = sr;
        mi[a + n * b] = si;
      }
    // LU with partial pivoting: log |det M| = sum log |u_jj|
    double logdet = 0.0;
    for (int j = 0; j < n; ++j) {
      int piv = j;
      double best = hypot(mr[j + n * j], mi[j + n * j]);
      for (int r = j + 1; r < n; ++r) {
        const double m = hypot(mr[r + n * j], mi[r + n * j]);
        if (m > best) {
          best = m;
          piv = r;
        }
      }
      if (piv != j)
        for (int c = 0; c < n; ++c) {
          double t = mr[j + n * c];
          mr[j + n * c] = mr[piv + n * c];
          mr[piv + n * c] = t;
          t = mi[j + n * c];
          mi[j + n * c] = mi[piv + n * c];
          mi[piv + n * c] = t;
        }
      logdet += log(best);
      if (best == 0.0) break;
      const double pr = mr[j + n * j], pi = mi[j + n * j];
      const double d = pr * pr + pi * pi;
      const double ir = pr / d, ii = -pi / d;  // 1 / pivot
      for (int r = j + 1; r < n; ++r) {
        const double lr = mr[r + n * j] * ir - mi[r + n * j] * ii;
        const double li = mr[r + n * j] * ii + mi[r + n * j] * ir;
        for (int c = j + 1; c < n; ++c) {
          mr[r + n * c] -= lr * mr[j + n * c] - li * mi[j + n * c];
          mi[r + n * c] -= lr * mi[j + n * c] + li * mr[j + n * c];
        }
      }
    }
    val = logdet;
  }
  red[threadIdx.x] = val;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int t = 0; t < blockDim.x; ++t) s += red[t];
    partials[(size_t)iw * gridDim.x + blockIdx.x] = s;
  }
}

// Projected CPT Green function on a wavevector grid, for the CDMFT host
// (lattice_model_instance::projected_Green_function, src_qcm/CPT.cpp:283-346;
// set_Gcpt, :76-86): for frequency w, the grid average of
//   G_cpt(k) = G (1 - V(k) G)^{-1},  V(k) = V0(w) + sum_e v_e exp(2 pi i k.R_e),
// k = ((a + off)/nkx, (b + off)/nky, (c + off)/nkz). One CTA per frequency;
// thread t sums the k points t, t + blockDim.x, ... into its own n x n
// accumulator (local memory, n <= 16) and writes it to partials[(w * T + t)];
// k_cpt_reduce adds the T accumulators in a fixed order. (1 - V G) is inverted
// by Gauss-Jordan elimination with partial pivoting.
constexpr int kCptThreads = 64;
__global__ void __launch_bounds__(kCptThreads) k_cpt_partial(int n, const double *__restrict__ G,
                                                              const double *__restrict__ V0, int nel,
                                                              const int *__restrict__ er, const int *__restrict__ ec,
                                                              const double *__restrict__ eR,
                                                              const double *__restrict__ ev, int nkx, int nky,
                                                              int nkz, double off, double *partials) {
  const int iw = blockIdx.x, T = blockDim.x;
  const int nn = n * n;
  const long nk = (long)nkx * nky * nkz;
  const double *g = G + 2 * (size_t)iw * nn, *v0 = V0 + 2 * (size_t)iw * nn;
  double sr[kSefMaxN * kSefMaxN], si[kSefMaxN * kSefMaxN];  // this thread's sum of G_cpt
  double ar[kSefMaxN * kSefMaxN], ai[kSefMaxN * kSefMaxN];  // 1 - V G, then its inverse
  double br[kSefMaxN * kSefMaxN], bi[kSefMaxN * kSefMaxN];  // V(k), then the identity being transformed
  for (int t = 0; t < nn; ++t) sr[t] = si[t] = 0.0;
  for (long kid = threadIdx.x; kid < nk; kid += T) {
    const int ix = (int)(kid / ((long)nky * nkz)), iy = (int)((kid / nkz) % nky), iz = (int)(kid % nkz);
    const double kx = (ix + off) / nkx, ky = (iy + off) / nky, kz = (iz + off) / nkz;
    for (int t = 0; t < nn; ++t) {
      br[t] = v0[2 * t];
      bi[t] = v0[2 * t + 1];
    }
    for (int e = 0; e < nel; ++e) {
      double s, c;
      sincospi(2.0 * (kx * eR[3 * e] + ky * eR[3 * e + 1] + kz * eR[3 * e + 2]), &s, &c);
      const int t = er[e] + n * ec[e];
      br[t] += ev[2 * e] * c - ev[2 * e + 1] * s;
      bi[t] += ev[2 * e] * s + ev[2 * e + 1] * c;
    }
    for (int b = 0; b < n; ++b)  // A = 1 - V G (column-major)
      for (int a = 0; a < n; ++a) {
        double xr = (a == b) ? 1.0 : 0.0, xi = 0.0;
        for (int c = 0; c < n; ++c) {
          const double vr = br[a + n * c], vi = bi[a + n * c];
          const double gr = g[2 * (c + n * b)], gi = g[2 * (c + n * b) + 1];
          xr -= vr * gr - vi * gi;
          xi -= vr * gi + vi * gr;
        }
        ar[a + n * b] = xr;
        ai[a + n * b] = xi;
      }
    for (int t = 0; t < nn; ++t) {  // B = identity
      br[t] = (t % (n + 1) == 0) ? 1.0 : 0.0;
      bi[t] = 0.0;
    }
    for (int j = 0; j < n; ++j) {  // Gauss-Jordan: A -> 1, B -> A^{-1}
      int piv = j;
      double best = hypot(ar[j + n * j], ai[j + n * j]);
      for (int r = j + 1; r < n; ++r) {
        const double m = hypot(ar[r + n * j], ai[r + n * j]);
        if (m > best) {
          best = m;
          piv = r;
        }
      }
      if (piv != j)
        for (int c = 0; c < n; ++c) {
          double t = ar[j + n * c]; ar[j + n * c] = ar[piv + n * c]; ar[piv + n * c] = t;
          t = ai[j + n * c]; ai[j + n * c] = ai[piv + n * c]; ai[piv + n * c] = t;
          t = br[j + n * c]; br[j + n * c] = br[piv + n * c]; br[piv + n * c] = t;
          t = bi[j + n * c]; bi[j + n * c] = bi[piv + n * c]; bi[piv + n * c] = t;
        }
      const double pr = ar[j + n * j], pi = ai[j + n * j];
      const double d = pr * pr + pi * pi;
      const double qr = pr / d, qi = -pi / d;  // 1 / pivot
      for (int c = 0; c < n; ++c) {  // row j /= pivot
        double xr = ar[j + n * c], xi = ai[j + n * c];
        ar[j + n * c] = xr * qr - xi * qi;
        ai[j + n * c] = xr * qi + xi * qr;
        xr = br[j + n * c];
        xi = bi[j + n * c];
        br[j + n * c] = xr * qr - xi * qi;
        bi[j + n * c] = xr * qi + xi * qr;
      }
      for (int r = 0; r < n; ++r) {  // eliminate column j from the other rows
        if (r == j) continue;
        const double fr = ar[r + n * j], fi = ai[r + n * j];
        if (fr == 0.0 && fi == 0.0) continue;
        for (int c = 0; c < n; ++c) {
          ar[r + n * c] -= fr * ar[j + n * c] - fi * ai[j + n * c];
          ai[r + n * c] -= fr * ai[j + n * c] + fi * ar[j + n * c];
          br[r + n * c] -= fr * br[j + n * c] - fi * bi[j + n * c];
          bi[r + n * c] -= fr * bi[j + n * c] + fi * br[j + n * c];
        }
      }
    }
    for (int b = 0; b < n; ++b)  // sum += G A^{-1}
      for (int a = 0; a < n; ++a) {
        double xr = 0.0, xi = 0.0;
        for (int c = 0; c < n; ++c) {
          const double gr = g[2 * (a + n * c)], gi = g[2 * (a + n * c) + 1];
          xr += gr * br[c + n * b] - gi * bi[c + n * b];
          xi += gr * bi[c + n * b] + gi * br[c + n * b];
        }
        sr[a + n * b] += xr;
        si[a + n * b] += xi;
      }
  }
  double *out = partials + 2 * ((size_t)iw * T + threadIdx.x) * nn;
  for (int t = 0; t < nn; ++t) {
    out[2 * t] = sr[t];
    out[2 * t + 1] = si[t];
  }
}

// Gproj[w] = (sum over the T thread accumulators, in order) / nk
__global__ void k_cpt_reduce(int nn, int T, long nk, const double *partials, double *Gproj) {
  const int iw = blockIdx.x;
  for (int t = threadIdx.x; t < 2 * nn; t += blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < T; ++q) s += partials[2 * ((size_t)iw * T + q) * nn + t];
    Gproj[2 * (size_t)iw * nn + t] = s / (double)nk;
  }
}

// Jacobi continued fractions, backward recursion (continued_fraction::evaluate,
// src_ed/continued_fraction.cpp:52-57); one thread per (fraction, frequency).
__global__ void k_cf_eval(int nf, const int *off, const int *len, const double *a, const double *b,
                          int nz, const double *z, double *F) {
  const size_t n = (size_t)nf * nz;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
    const int f = (int)(t % nf), k = (int)(t / nf);
    const double zr = z[2 * k], zi = z[2 * k + 1];
    const int o = off[f];
    double gr = 0.0, gi = 0.0;
    for (int i = len[f] - 1; i >= 0; --i) {
      // G = b_i / (z - a_i - G)
      double dr = zr - a[o + i] - gr, di = zi - gi;
      double den = dr * dr + di * di;
      double bi = b[o + i];
      gr = bi * dr / den;
      gi = -bi * di / den;
    }
    F[2 * t] = gr;
    F[2 * t + 1] = gi;
  }
}

}  // namespace

// ------------------------------------------------------------ launchers ----

void launch_unrank(int L, int N, uint32_t dim, uint32_t *out, cudaStream_t s) {
  ensure_binom();
  k_unrank<<<grid_for(dim, device_sms()), kThreads, 0, s>>>(L, N, dim, out);
  QED_LAUNCH();
}

void launch_rank(int L, int N, size_t n, const uint32_t *strings, uint32_t *ranks, cudaStream_t s) {
  ensure_binom();
  k_rank<<<grid_for(n, device_sms()), kThreads, 0, s>>>(L, N, n, strings, ranks);
  QED_LAUNCH();
}

void launch_build_hops(int L, int N, uint32_t dim, const uint32_t *bits, int npairs,
                       const int *pd, const int *ps, const int *pslot, uint8_t *cnt, uint32_t *ell,
                       int width, cudaStream_t s) {
  ensure_binom();
  k_build_hops<<<grid_for(dim, device_sms()), kThreads, 0, s>>>(L, N, dim, bits, npairs, pd, ps,
                                                                 pslot, cnt, ell, width);
  QED_LAUNCH();
}

void launch_diag_half(int L, uint32_t dim, const uint32_t *bits, const double *tdiag,
                      const double *vsame, double *diag, cudaStream_t s) {
  k_diag_half<<<grid_for(dim, device_sms()), kThreads, 0, s>>>(L, dim, bits, tdiag, vsame, diag);
  QED_LAUNCH();
}

void launch_cdag_gather(int L, int spin, int a, int pm, const uint32_t *tub, uint32_t du_t,
                        const uint32_t *tdb, uint32_t dd_t, int src_nup, int src_ndn, uint32_t du_s,
                        const double *psi, double *y, double coef, int accumulate, cudaStream_t s) {
  ensure_binom();
  size_t D = (size_t)du_t * dd_t;
  k_cdag_gather<<<grid_for(D, device_sms(), 8), kThreads, 0, s>>>(
      L, spin, a, pm, tub, du_t, tdb, dd_t, src_nup, src_ndn, du_s, psi, y, coef, accumulate);
  QED_LAUNCH();
}

void launch_dense_hamiltonian(const HvOperator &op, double *h, cudaStream_t s) {
  const size_t D = (size_t)op.up.dim * op.dn.dim;
  if (!D) return;
  QED_CUDA(cudaMemsetAsync(h, 0, D * D * sizeof(double), s));
  k_dense_hamiltonian<<<grid_for(D, device_sms()), kThreads, 0, s>>>(op, h);
  QED_LAUNCH();
}

namespace {
constexpr size_t kRowSmemMax = 112 * 1024;
constexpr size_t kRowSmem2Max = 220 * 1024;  // below the 227 KB per-CTA limit
}

// Launch variant of the H.v passes of sectors without the staged kernels (the
// solver option hv_variant; bit 0: column-pass gathers cached in L2 only; bit 1:
// row pass with four gathers in flight; bit 2: staged kernels off). Default 2
// (on the 4x4 sector with the staged kernels off: 5.47 ms per H.v against 5.57 ms
// for 0). The staged kernels pick their launch shape by timing (below).
int hv_variant() {
  thread_local unsigned long long gen = ~0ull;  // read once per thread and option change
  thread_local int v = 2;
  const unsigned long long g = options_generation();
  if (g != gen) {
    v = (int)opt_int("hv_variant");
    gen = g;
  }
  return v;
}

namespace {

constexpr size_t kSmemOptin = 227 * 1024;  // per-CTA dynamic shared memory limit (sm_100)
constexpr size_t kStagedMaxThreads = 1024;  // the largest launch shape of the staged kernels

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

// Shared memory of k_hv_rows16 / k_hv_cols16 for this operator (0: not applicable).
size_t rows16_smem(const HvOperator &op) {
  const uint32_t du = op.up.dim;
  if (!op.up.cntw || du % 2 || du < 512 || op.dn.dim < 2) return 0;
  const size_t b = (size_t)(du + 8) * sizeof(double2);
  return b <= kRowSmem2Max ? b : 0;
}

size_t cols16_smem(const HvOperator &op) {
  const uint32_t du = op.up.dim, dd = op.dn.dim;
  if (!op.dn.cntw || du % 2 || du < 2 || dd < 512) return 0;
  const size_t nst = (size_t)(dd + kTmaBoxRows - 1) / kTmaBoxRows * kTmaBoxRows + 8;
  const size_t b = nst * sizeof(double2) + kStagedMaxThreads * sizeof(double2) + 2 * sizeof(uint64_t);
  return b <= kSmemOptin - 1024 ? b : 0;
}

bool staged_disabled() { return (hv_variant() & 4) != 0; }

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    QED_CUDA(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !p) fail(QED_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

// TMA map of a dd x du row-major FP64 matrix with a box of 2 columns x box_rows
// rows (16 bytes wide: du even keeps the row stride and every box start, at an
// even column, on 16-byte boundaries); reads past the last row fill zeros.
CUtensorMap column_pair_map(const double *base, uint32_t du, uint32_t dd, uint32_t box_rows) {
  CUtensorMap m;
  cuuint64_t dims[2] = {du, dd};
  cuuint64_t strides[1] = {(cuuint64_t)du * sizeof(double)};
  cuuint32_t box[2] = {2, box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = tensor_map_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(base), dims,
                                    strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) fail(QED_ERR_CUDA, "cuTensorMapEncodeTiled failed with code " + std::to_string((int)r));
  return m;
}

}  // namespace

int hv_cols_grid(const HvOperator &op) {
  const uint32_t du = op.up.dim, dd = op.dn.dim;
  const uint32_t W = ((du % 2 == 0) ? 2 : 1) * kThreads;
  const size_t nitems = (size_t)((du + W - 1) / W) * ((dd + kColsR - 1) / kColsR);
  const int g = (int)std::max<size_t>(1, std::min<size_t>(nitems, (size_t)device_sms() * 8));
  // the staged pass runs one CTA per column pair, at most one per SM
  const int g16 = (int)std::max<size_t>(1, std::min<size_t>(du / 2, (size_t)device_sms()));
  return std::max(g, g16);
}

std::atomic<bool> g_staged_used{false};  // set by the first staged H.v launch

bool staged_kernels_used() { return g_staged_used.load(std::memory_order_relaxed); }

void read_wait_flag_async(int *host_flag, cudaStream_t s) {
  QED_CUDA(cudaMemcpyFromSymbolAsync(host_flag, g_wait_timeout, sizeof(int), 0, cudaMemcpyDeviceToHost, s));
}

void check_wait_flag(int flag) {
  if (flag) fail(QED_ERR_CUDA, "a kernel's wait on its TMA transfers gave up after 2 s (results are invalid)");
}

void launch_hv_rows(const HvOperator &op, const double *x, double xs, double *y,
                    const SubList &sub, cudaStream_t s) {
  const uint32_t du = op.up.dim, dd = op.dn.dim;
  if (const size_t sm16 = staged_disabled() ? 0 : rows16_smem(op); sm16 && aligned16(x)) {
    static const bool attr16 = [] {
      QED_CUDA(cudaFuncSetAttribute(k_hv_rows16<512, 6, 4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kRowSmem2Max));
      return true;
    }();
    (void)attr16;
    const int grid = (int)std::min<size_t>((dd + 1) / 2, (size_t)device_sms());
    k_hv_rows16<512, 6, 4, false><<<grid, 512, sm16, s>>>(op, x, xs, y, sub, 0, nullptr);
    QED_LAUNCH();
    return;
  }
  const size_t smem = (size_t)du * sizeof(double);
  int threads = du >= 512 ? 512 : (du >= 256 ? 256 : 128);
  const size_t smem2 = 2 * smem;  // two rows interleaved
  if (smem2 <= kRowSmem2Max && dd >= 2) {
    static const bool attr2 = [] {
      QED_CUDA(cudaFuncSetAttribute(k_hv_rows2<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kRowSmem2Max));
      QED_CUDA(cudaFuncSetAttribute(k_hv_rows2<4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kRowSmem2Max));
      return true;
    }();
    (void)attr2;
    const int t2 = du >= 1024 ? 1024 : threads;
    const int per_sm = smem2 > 110 * 1024 ? 1 : (smem2 > 72 * 1024 ? 2 : 3);
    int grid = (int)std::min<size_t>((dd + 1) / 2, (size_t)device_sms() * per_sm);
    if (hv_variant() & 2)
      k_hv_rows2<4><<<grid, t2, smem2, s>>>(op, x, xs, y, sub);
    else
      k_hv_rows2<2><<<grid, t2, smem2, s>>>(op, x, xs, y, sub);
  } else if (smem <= kRowSmemMax) {
    static const bool attr = [] {
      QED_CUDA(cudaFuncSetAttribute(k_hv_rows<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)kRowSmemMax));
      return true;
    }();
    (void)attr;
    int per_sm = smem > 100 * 1024 ? 2 : 4;
    int grid = (int)std::min<size_t>(dd, (size_t)device_sms() * per_sm);
    k_hv_rows<true><<<grid, threads, smem, s>>>(op, x, xs, y, sub);
  } else {
    int grid = (int)std::min<size_t>(dd, (size_t)device_sms() * 4);
    k_hv_rows<false><<<grid, threads, 0, s>>>(op, x, xs, y, sub);
  }
  QED_LAUNCH();
}

int launch_hv_cols(const HvOperator &op, const double *x, double xs, double *y, int red_mask,
                   Reducer &r, cudaStream_t s) {
  const bool vec2 = (op.up.dim % 2 == 0);
  int grid = hv_cols_grid(op);
  if (red_mask && grid > r.max_blocks) grid = r.max_blocks;
  const bool cg = hv_variant() & 1;
  const uint32_t dd = op.dn.dim;
  if (vec2 && cg)
    k_hv_cols2<2, true><<<grid, kThreads, 0, s>>>(op, x, xs, y, red_mask, r.partials, 0u, dd);
  else if (vec2)
    k_hv_cols2<2, false><<<grid, kThreads, 0, s>>>(op, x, xs, y, red_mask, r.partials, 0u, dd);
  else
    k_hv_cols2<1, false><<<grid, kThreads, 0, s>>>(op, x, xs, y, red_mask, r.partials, 0u, dd);
  QED_LAUNCH();
  return grid;
}

void launch_hv_cols_rows(const HvOperator &op, const double *x, double xs, double *y, uint32_t r0, uint32_t r1,
                         cudaStream_t s) {
  if (r1 <= r0) return;
  const int grid = hv_cols_grid(op);
  if (op.up.dim % 2 == 0)
    k_hv_cols2<2, false><<<grid, kThreads, 0, s>>>(op, x, xs, y, 0, nullptr, r0, r1);
  else
    k_hv_cols2<1, false><<<grid, kThreads, 0, s>>>(op, x, xs, y, 0, nullptr, r0, r1);
  QED_LAUNCH();
}

// ---- staged H.v launch shapes and their autotuner ----
//
// The staged kernels come in launch shapes (threads per CTA, hop words loaded
// ahead per class) that give the same bits; which is fastest depends on the
// sector. The first staged H.v of each (dim_up, dim_dn) runs every shape a few
// times on the call's own vectors (y is fully rewritten by every run), times it
// with CUDA events and keeps the fastest for that shape.
namespace {

using RowsFn = void (*)(HvOperator, const double *, double, double *, SubList, int, double *);
using ColsFn = void (*)(CUtensorMap, CUtensorMap, HvOperator, double);

struct StagedShape {
  int threads;
  RowsFn rows;
  ColsFn cols;
  const char *name;
};

const StagedShape kShapes[] = {
    {512, k_hv_rows16<512, 6, 4, true>, k_hv_cols16w<512, 6, 4>, "512t/6+4"},
    {768, k_hv_rows16<768, 4, 2, true>, k_hv_cols16w<768, 4, 2>, "768t/4+2"},
    {1024, k_hv_rows16<1024, 2, 1, true>, k_hv_cols16w<1024, 2, 1>, "1024t/2+1"},
    {384, k_hv_rows16<384, 8, 5, true>, k_hv_cols16w<384, 8, 5>, "384t/8+5"},
};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

struct TuneRecord {
  int choice = 0;
  float ms[kNumShapes] = {};
  bool identical = true;  // every shape wrote the same bits of y
};

// Order-independent fingerprint of the bits of y: the sum over i of
// splitmix64(bits(y_i) ^ golden-ratio * i) mod 2^64 (Vigna's splitmix64
// finaliser); two vectors that differ in any bit or position give different
// sums except with probability about 2^-64.
__global__ void k_bits_fingerprint(const double *__restrict__ y, size_t n, unsigned long long *h) {
  unsigned long long acc = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    unsigned long long z = (unsigned long long)__double_as_longlong(y[i]) ^ (i * 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    acc += z ^ (z >> 31);
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(h, acc);
}
std::mutex g_tune_mtx;
std::map<std::pair<uint32_t, uint32_t>, TuneRecord> g_tune;

void set_shape_attributes() {
  static std::once_flag once;
  std::call_once(once, [] {
    for (const auto &v : kShapes) {
      QED_CUDA(cudaFuncSetAttribute(v.rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRowSmem2Max));
      QED_CUDA(cudaFuncSetAttribute(v.cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(kSmemOptin - 1024)));
    }
  });
}

int launch_staged(int v, const HvOperator &op, const double *x, double xs, double *y, const SubList &sub,
                  int red_mask, Reducer &r, size_t smr, size_t smc, cudaStream_t s) {
  const StagedShape &sh = kShapes[v];
  const uint32_t du = op.up.dim, dd = op.dn.dim;
  const int gc = (int)std::min<size_t>(du / 2, (size_t)device_sms());
  const CUtensorMap mx = column_pair_map(x, du, dd, kTmaBoxRows);
  const CUtensorMap my = column_pair_map(y, du, dd, kSliceRows);
  sh.cols<<<gc, sh.threads, smc, s>>>(mx, my, op, xs);
  QED_LAUNCH();
  int gr = (int)std::min<size_t>((dd + 1) / 2, (size_t)device_sms());
  if (red_mask && gr > r.max_blocks) gr = r.max_blocks;
  sh.rows<<<gr, sh.threads, smr, s>>>(op, x, xs, y, sub, red_mask, r.partials);
  QED_LAUNCH();
  return gr;
}

int staged_shape(const HvOperator &op, const double *x, double *y, Reducer &r, size_t smr, size_t smc,
                 cudaStream_t s, bool may_tune) {
  const std::pair<uint32_t, uint32_t> key{op.up.dim, op.dn.dim};
  {
    std::lock_guard<std::mutex> l(g_tune_mtx);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second.choice;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  QED_CUDA(cudaStreamIsCapturing(s, &cs));
  if (!may_tune || cs != cudaStreamCaptureStatusNone) return 0;
  TuneRecord rec;
  cudaEvent_t e0, e1;
  QED_CUDA(cudaEventCreate(&e0));
  QED_CUDA(cudaEventCreate(&e1));
  unsigned long long *fp = nullptr;  // one fingerprint of y per shape
  QED_CUDA(cudaMallocAsync((void **)&fp, kNumShapes * sizeof(unsigned long long), s));
  QED_CUDA(cudaMemsetAsync(fp, 0, kNumShapes * sizeof(unsigned long long), s));
  const size_t D = (size_t)op.up.dim * op.dn.dim;
  SubList none;
  float best = 0.0f;
  for (int v = 0; v < kNumShapes; ++v) {
    launch_staged(v, op, x, 1.0, y, none, 0, r, smr, smc, s);  // warm-up
    QED_CUDA(cudaEventRecord(e0, s));
    for (int k = 0; k < 3; ++k) launch_staged(v, op, x, 1.0, y, none, 0, r, smr, smc, s);
    QED_CUDA(cudaEventRecord(e1, s));
    k_bits_fingerprint<<<2 * device_sms(), 256, 0, s>>>(y, D, fp + v);
    QED_LAUNCH();
    QED_CUDA(cudaEventSynchronize(e1));
    float ms = 0.0f;
    QED_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    rec.ms[v] = ms / 3.0f;
    if (v == 0 || rec.ms[v] < best) {
      best = rec.ms[v];
      rec.choice = v;
    }
  }
  unsigned long long h[kNumShapes];
  QED_CUDA(cudaMemcpyAsync(h, fp, sizeof(h), cudaMemcpyDeviceToHost, s));
  QED_CUDA(cudaFreeAsync(fp, s));
  QED_CUDA(cudaStreamSynchronize(s));
  for (int v = 1; v < kNumShapes; ++v) rec.identical = rec.identical && h[v] == h[0];
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::lock_guard<std::mutex> l(g_tune_mtx);
  return g_tune.emplace(key, rec).first->second.choice;
}

int launch_hv_impl(const HvOperator &op, const double *x, double xs, double *y, const SubList &sub, int red_mask,
                   Reducer &r, cudaStream_t s, bool may_tune) {
  if (op.win && window_usable(op, x, y, sub)) return launch_hv_windows(op, x, xs, y, sub, red_mask, r, s);
  const size_t smr = staged_disabled() ? 0 : rows16_smem(op);
  const size_t smc = smr ? cols16_smem(op) : 0;
  bool staged = smr && smc && aligned16(x) && aligned16(y);
  for (int k = 0; k < sub.n && staged; ++k)
    if (sub.z[k] == y) staged = false;  // the column pass would overwrite a term of the row pass
  if (!staged) {
    launch_hv_rows(op, x, xs, y, sub, s);
    return launch_hv_cols(op, x, xs, y, red_mask, r, s);
  }
  set_shape_attributes();
  g_staged_used.store(true, std::memory_order_relaxed);
  const int v = staged_shape(op, x, y, r, smr, smc, s, may_tune);
  return launch_staged(v, op, x, xs, y, sub, red_mask, r, smr, smc, s);
}

}  // namespace

int launch_hv(const HvOperator &op, const double *x, double xs, double *y, const SubList &sub, int red_mask,
              Reducer &r, cudaStream_t s) {
  return launch_hv_impl(op, x, xs, y, sub, red_mask, r, s, true);
}

std::string hv_tuning_report() {
  std::lock_guard<std::mutex> l(g_tune_mtx);
  std::string out = "[";
  for (const auto &kv : g_tune) {
    if (out.size() > 1) out += ", ";
    out += "{\"dim_up\": " + std::to_string(kv.first.first) + ", \"dim_dn\": " + std::to_string(kv.first.second) +
           ", \"choice\": \"" + kShapes[kv.second.choice].name +
           "\", \"bit_identical\": " + (kv.second.identical ? "true" : "false") + ", \"ms\": {";
    for (int v = 0; v < kNumShapes; ++v)
      out += std::string(v ? ", " : "") + "\"" + kShapes[v].name + "\": " + std::to_string(kv.second.ms[v]);
    out += "}}";
  }
  return out + "]";
}

void launch_block_hv(const HvOperator &op, int p, const BlockIn &X, const BlockOut &Y, Reducer &r, cudaStream_t s) {
  if (p < 1 || p > 16) fail(QED_ERR_ARGUMENT, "block H.v: block size outside [1, 16]");
  const size_t D = (size_t)op.up.dim * op.dn.dim;
  if (!D) return;
  bool staged = op.win || (!staged_disabled() && rows16_smem(op) && cols16_smem(op));
  for (int c = 0; c < p && staged; ++c) staged = aligned16(X.v[c]) && aligned16(Y.v[c]);
  if (staged) {  // large sectors: the staged single-vector kernels, one vector at a time
    SubList none;
    for (int c = 0; c < p; ++c) launch_hv(op, X.v[c], 1.0, Y.v[c], none, 0, r, s);
    return;
  }
  const int grid = grid_for(D, device_sms(), 8);
  if (p <= 4) {
    k_blhv_rows<4><<<grid, kThreads, 0, s>>>(op, p, X, Y);
    QED_LAUNCH();
    k_blhv_cols<4><<<grid, kThreads, 0, s>>>(op, p, X, Y);
  } else if (p <= 8) {
    k_blhv_rows<8><<<grid, kThreads, 0, s>>>(op, p, X, Y);
    QED_LAUNCH();
    k_blhv_cols<8><<<grid, kThreads, 0, s>>>(op, p, X, Y);
  } else {
    k_blhv_rows<16><<<grid, kThreads, 0, s>>>(op, p, X, Y);
    QED_LAUNCH();
    k_blhv_cols<16><<<grid, kThreads, 0, s>>>(op, p, X, Y);
  }
  QED_LAUNCH();
}

int launch_dots(size_t D, double *x, double xs, int write_x, const VecList &ys, Reducer &r,
                cudaStream_t s) {
  int grid = std::min(grid_for(D, device_sms(), 4), r.max_blocks);
  constexpr int G = 8;
  if (ys.n == 0 && write_x) {
    k_scale<<<grid, kThreads, 0, s>>>(D, x, xs);
    QED_LAUNCH();
    return grid;
  }
  for (int first = 0; first < ys.n; first += G) {
    // x is scaled in place only on the first sweep; later sweeps read the scaled x.
    const bool wx = write_x && first == 0;
    const double sc = (write_x && first > 0) ? 1.0 : xs;
    k_dots<G><<<grid, kThreads, 0, s>>>(D, x, sc, wx, ys, first, r.partials);
    QED_LAUNCH();
  }
  return grid;
}

int launch_multi_axpy(size_t D, const double *x, double xs, const VecList &ys, int norm_first,
                      Reducer &r, cudaStream_t s) {
  int grid = std::min(grid_for(D, device_sms(), 4), r.max_blocks);
  k_multi_axpy<<<grid, kThreads, 0, s>>>(D, x, xs, ys, norm_first, r.partials);
  QED_LAUNCH();
  return grid;
}

int launch_axpby(size_t D, double a, double *y, double b, const double *x, int norm, Reducer &r,
                 cudaStream_t s) {
  int grid = std::min(grid_for(D, device_sms(), 4), r.max_blocks);
  k_axpby<<<grid, kThreads, 0, s>>>(D, a, y, b, x, norm, r.partials);
  QED_LAUNCH();
  return grid;
}

int launch_axpy_dev(size_t D, double *y, const double *x, const double *a_dev, Reducer &r, cudaStream_t s,
                    const int *skip) {
  int grid = std::min(grid_for(D, device_sms(), 4), r.max_blocks);
  k_axpy_dev<<<grid, kThreads, 0, s>>>(D, y, x, a_dev, r.partials, skip);
  QED_LAUNCH();
  return grid;
}

void launch_lanczos_advance(size_t D, double *y, const LanczosScalars &ls, cudaStream_t s) {
  k_lanczos_advance<<<grid_for(D, device_sms(), 4), kThreads, 0, s>>>(D, y, ls);
  QED_LAUNCH();
}

void launch_lanczos_start_jobs(const LanczosJob *jobs, int njobs, cudaStream_t s) {
  if (njobs <= 0) return;
  k_lanczos_start_jobs<<<njobs, kLanczosJobThreads, 0, s>>>(jobs);
  QED_LAUNCH();
}

void launch_lanczos_jobs(const LanczosJob *jobs, int njobs, cudaStream_t s) {
  if (njobs <= 0) return;
  k_lanczos_jobs<<<njobs, kLanczosJobThreads, 0, s>>>(jobs);
  QED_LAUNCH();
}

namespace {
}  // namespace

void launch_finalize_ld(const double *partials, int nblocks, int ld, int n, double *out, cudaStream_t s) {
  k_finalize_ld<<<n, kThreads, 0, s>>>(partials, nblocks, ld, out);
  QED_LAUNCH();
}

void launch_cpt_projected(int n, int nw, const double *G, const double *V0, int nel, const int *er, const int *ec,
                          const double *eR, const double *ev, int nkx, int nky, int nkz, double off,
                          double *partials, double *Gproj, cudaStream_t s) {
  if (n < 1 || n > kSefMaxN) fail(QED_ERR_UNSUPPORTED, "projected Green function: dimension above 16");
  if (nw <= 0) return;
  k_cpt_partial<<<nw, kCptThreads, 0, s>>>(n, G, V0, nel, er, ec, eR, ev, nkx, nky, nkz, off, partials);
  QED_LAUNCH();
  k_cpt_reduce<<<nw, 64, 0, s>>>(n * n, kCptThreads, (long)nkx * nky * nkz, partials, Gproj);
  QED_LAUNCH();
}

int cpt_partials_size(int n, int nw) { return 2 * n * n * kCptThreads * nw; }

int launch_sef_logdet(int n, int nw, const double *G, const double *V0, int nel, const int *er, const int *ec,
                      const double *eR, const double *ev, int nkx, int nky, int nkz, double *partials,
                      cudaStream_t s) {
  if (n < 1 || n > kSefMaxN) fail(QED_ERR_UNSUPPORTED, "SEF grid integrand: Green function dimension above 16");
  const long nk = (long)nkx * nky * nkz;
  const int nblk = (int)((nk + kSefThreads - 1) / kSefThreads);
  if (nw <= 0 || nk <= 0) return nblk;
  if (nw > 65535) fail(QED_ERR_ARGUMENT, "SEF grid integrand: more than 65535 frequencies");
  k_sef_logdet<<<dim3(nblk, nw), kSefThreads, 0, s>>>(n, G, V0, nel, er, ec, eR, ev, nkx, nky, nkz, partials);
  QED_LAUNCH();
  return nblk;
}

void launch_block_chol(int p, const double *G, double pivot_min, double *R, double *Rinv, const double *Rprev,
                       double *B_out, double *Bt_out, double *fail_flag, cudaStream_t s) {
  if (p < 1 || p > 16) fail(QED_ERR_ARGUMENT, "launch_block_chol: block size outside [1, 16]");
  k_block_chol<<<1, 256, 0, s>>>(p, G, pivot_min, R, Rinv, Rprev, B_out, Bt_out, fail_flag);
  QED_LAUNCH();
}

void launch_swap_scale(size_t D, double *q, double *p, double beta, cudaStream_t s) {
  k_swap_scale<<<grid_for(D, device_sms(), 4), kThreads, 0, s>>>(D, q, p, beta);
  QED_LAUNCH();
}

int launch_random(size_t D, uint64_t seed, double *y, Reducer &r, cudaStream_t s) {
  int grid = std::min(grid_for(D, device_sms(), 4), r.max_blocks);
  k_random<<<grid, kThreads, 0, s>>>(D, seed, y, r.partials);
  QED_LAUNCH();
  return grid;
}

void launch_scale_dev(size_t D, double *y, const double *a_dev, const int *skip, cudaStream_t s) {
  k_scale_dev<<<grid_for(D, device_sms(), 4), kThreads, 0, s>>>(D, y, a_dev, skip);
  QED_LAUNCH();
}

void launch_finalize_norm(const double *partials, int nblocks, double dtol, double *z_out, double *inv_out,
                          int *flag, int step, cudaStream_t s) {
  k_finalize_norm<<<1, kThreads, 0, s>>>(partials, nblocks, dtol, z_out, inv_out, flag, step);
  QED_LAUNCH();
}

void launch_scale(size_t D, double *y, double a, cudaStream_t s) {
  k_scale<<<grid_for(D, device_sms(), 4), kThreads, 0, s>>>(D, y, a);
  QED_LAUNCH();
}

void finalize_sums(Reducer &r, int nblocks, int nred, cudaStream_t s) {
  k_finalize<<<nred, kThreads, 0, s>>>(r.partials, nblocks, r.out);
  QED_LAUNCH();
  QED_CUDA(cudaMemcpyAsync(r.host, r.out, nred * sizeof(double), cudaMemcpyDeviceToHost, s));
}

void launch_finalize(const double *partials, int nblocks, int nred, double *out, cudaStream_t s) {
  k_finalize<<<nred, kThreads, 0, s>>>(partials, nblocks, out);
  QED_LAUNCH();
}

// ---- H.v + dots without any device allocation -------------------------------
//
// For callers that cannot allocate device memory at call time: a process whose
// device memory is owned by another runtime's pool, a real-time loop that cannot
// take cudaMalloc's implicit synchronisation, or code that must not grow the
// footprint after set-up. The scratch below is part of the library image: every
// GPU that loads the library holds it (682 KB) until the process exits.

namespace {

// Per-block partial sums of the reducing column pass: kHvColsMaxBlocks rows of
// Reducer::kMaxRed doubles (1184 x 72 x 8 B = 682 KB).
static __device__ __align__(256) double g_noalloc_partials[kHvColsMaxBlocks * Reducer::kMaxRed];

// Device address of g_noalloc_partials, looked up once per device with that
// device current. In host code the array's name is only a host-side stand-in,
// so kernels must be given this address, never the symbol itself.
double *noalloc_partials_address() {
  static std::mutex mtx;
  static double *addr[64] = {};
  int dev = 0;
  QED_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) fail(QED_ERR_ARGUMENT, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(mtx);
  if (!addr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || !p)
      fail(QED_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    addr[dev] = static_cast<double *>(p);
  }
  return addr[dev];
}

}  // namespace

void launch_hv_dots_noalloc(const HvOperator &op, const double *x, double *y, double *dots,
                            cudaStream_t s) {
  // The grid the column pass launches (grid-stride, at most 8 CTAs per SM);
  // each CTA needs one row of the scratch.
  const size_t want = (size_t)hv_cols_grid(op);
  if (want > (size_t)kHvColsMaxBlocks)
    fail(QED_ERR_MEMORY, "H.v without allocation: the column pass needs " + std::to_string(want) +
                             " partial-sum rows, the fixed scratch holds " +
                             std::to_string(kHvColsMaxBlocks));
  Reducer r;
  r.partials = noalloc_partials_address();
  r.max_blocks = kHvColsMaxBlocks;
  SubList none;
  // no tuning here (it would create events): a shape tuned earlier, else the first
  const int nb = launch_hv_impl(op, x, 1.0, y, none, 7, r, s, false);
  // Every block of the reducing launch overwrites its own row, and the sum reads
  // only those rows, so nothing has to be cleared between calls.
  launch_finalize(r.partials, nb, 3, dots, s);
}

void launch_qmatrix_gf(int L, int M, const double *e, const double *V, int nz, const double *z,
                       double *G, cudaStream_t s) {
  if (nz <= 0 || M <= 0) return;
  if (L > 64) fail(QED_ERR_UNSUPPORTED, "Green function dimension above 64");
  k_qmatrix_gf<<<nz, kThreads, 0, s>>>(L, M, e, V, nz, z, G);
  QED_LAUNCH();
}

void launch_cf_eval(int nf, const int *off, const int *len, const double *a, const double *b,
                    int nz, const double *z, double *F, cudaStream_t s) {
  if (nf <= 0 || nz <= 0) return;
  size_t n = (size_t)nf * nz;
  k_cf_eval<<<grid_for(n, device_sms(), 8), kThreads, 0, s>>>(nf, off, len, a, b, nz, z, F);
  QED_LAUNCH();
}

void launch_mcf_eval(int nf, const McfDesc *desc, const double *blob, int q, int nz, const double *z, double *out,
                     cudaStream_t s) {
  if (nf <= 0 || nz <= 0) return;
  if (q > 32) fail(QED_ERR_UNSUPPORTED, "matrix continued fractions of more than 32 orbitals");
  k_mcf_eval<<<dim3(nz, nf), 256, 0, s>>>(desc, blob, q, nz, z, out);
  QED_LAUNCH();
}

}  // namespace qed
