// Symmetry-adapted (mixed) basis Hamiltonian on the device: see mixed.hpp.
#include "mixed.hpp"

#include <cmath>
#include <mutex>

#include "kernels.cuh"
#include "options.hpp"
#include "qed_b200.h"

namespace qed {

MixedTerms mixed_terms(const Model &m, const std::map<std::string, double> &value) {
  const int n = m.n_orb;
  auto mask = [n](int i) -> uint64_t { return i >= n ? (uint64_t)1 << (i - n + 32) : (uint64_t)1 << i; };
  std::map<std::pair<int, int>, double> off;
  std::map<uint64_t, double> diag;
  for (const auto &kv : value) {
    const Operator &op = *m.term.at(kv.first);
    for (const Element &e : op.elements) {
      const double x = kv.second * e.v;
      if (op.is_interaction) diag[mask(e.r) + mask(e.c)] += x;  // r == c doubles the bit, as the reference does
      else if (e.r == e.c) diag[mask(e.r)] += x;
      else off[{e.r, e.c}] += x;
    }
  }
  MixedTerms t;
  for (const auto &kv : off) {
    if (kv.second == 0.0) continue;
    t.r.push_back(kv.first.first);
    t.c.push_back(kv.first.second);
    t.v.push_back(kv.second);
  }
  for (const auto &kv : diag) {
    if (kv.second == 0.0) continue;
    t.dmask.push_back(kv.first);
    t.dval.push_back(kv.second);
  }
  return t;
}

namespace {

constexpr int kMarkTile = 4096;   // factorized states per block of the mark scan
constexpr int kMarkThreads = 256; // 16 states per thread

__constant__ uint32_t c_mbinom[33][33];  // C(n, k), n, k <= 32

struct OffTerms {
  int n;
  const int *r, *c;
  const double *v;
};

// colex rank of an L-bit string: sum over its set bits p_1 < p_2 < ... of C(p_i, i)
__device__ __forceinline__ uint32_t colex_rank(uint32_t s) {
  uint32_t rank = 0;
  int i = 1;
  while (s) {
    const int p = __ffs(s) - 1;
    rank += c_mbinom[p][i++];
    s &= s - 1;
  }
  return rank;
}

__device__ __forceinline__ uint64_t orb_mask(int i, int n) {
  return i >= n ? (uint64_t)1 << (i - n + 32) : (uint64_t)1 << i;
}

__global__ void k_mixed_mark(SymGroup G, int irrep, const uint32_t *__restrict__ ustr, uint32_t du,
                             const uint32_t *__restrict__ dstr, uint64_t nf, uint8_t *__restrict__ lenf) {
  for (uint64_t f = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; f < nf; f += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = (uint64_t)ustr[f % du] | ((uint64_t)dstr[f / du] << 32);
    const RepMap m = sym_representative(G, b, irrep);
    lenf[f] = (m.length > 0 && m.rep == b) ? (uint8_t)m.length : (uint8_t)0;
  }
}

// Per tile of kMarkTile factorized states: how many are basis states.
__global__ void __launch_bounds__(kMarkThreads) k_mixed_tile_count(const uint8_t *__restrict__ lenf, uint64_t nf,
                                                                   uint32_t *__restrict__ tile_count) {
  const uint64_t base = (uint64_t)blockIdx.x * kMarkTile;
  uint32_t c = 0;
  for (int k = threadIdx.x; k < kMarkTile; k += kMarkThreads) {
    const uint64_t f = base + k;
    if (f < nf && lenf[f]) ++c;
  }
  __shared__ uint32_t red[kMarkThreads / 32];
  for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t s = 0;
    for (int w = 0; w < kMarkThreads / 32; ++w) s += red[w];
    tile_count[blockIdx.x] = s;
  }
}

// Writes the basis in factorized order: each thread takes 16 consecutive
// states of the tile, the block scans the per-thread counts.
__global__ void __launch_bounds__(kMarkThreads) k_mixed_scatter(const uint8_t *__restrict__ lenf, uint64_t nf,
                                                                const uint64_t *__restrict__ tile_off,
                                                                const uint32_t *__restrict__ ustr, uint32_t du,
                                                                const uint32_t *__restrict__ dstr,
                                                                int32_t *__restrict__ fmap,
                                                                uint64_t *__restrict__ states,
                                                                uint8_t *__restrict__ len) {
  constexpr int per = kMarkTile / kMarkThreads;
  const uint64_t f0 = (uint64_t)blockIdx.x * kMarkTile + (uint64_t)threadIdx.x * per;
  uint32_t c = 0;
  for (int k = 0; k < per; ++k)
    if (f0 + k < nf && lenf[f0 + k]) ++c;
  __shared__ uint32_t scan[kMarkThreads];
  scan[threadIdx.x] = c;
  __syncthreads();
  for (int o = 1; o < kMarkThreads; o <<= 1) {  // inclusive Hillis-Steele scan
    const uint32_t add = threadIdx.x >= o ? scan[threadIdx.x - o] : 0u;
    __syncthreads();
    scan[threadIdx.x] += add;
    __syncthreads();
  }
  uint64_t idx = tile_off[blockIdx.x] + scan[threadIdx.x] - c;
  for (int k = 0; k < per; ++k) {
    const uint64_t f = f0 + k;
    if (f >= nf) break;
    const uint8_t l = lenf[f];
    if (!l) {
      fmap[f] = -1;
      continue;
    }
    fmap[f] = (int32_t)idx;
    states[idx] = (uint64_t)ustr[f % du] | ((uint64_t)dstr[f / du] << 32);
    len[idx] = l;
    ++idx;
  }
}

// Row J's off-diagonal entries: count (fill == false) or write them.
template <bool fill>
__global__ void k_mixed_rows(SymGroup G, int irrep, OffTerms t, const uint64_t *__restrict__ states,
                             const uint8_t *__restrict__ len, uint64_t D, const int32_t *__restrict__ fmap,
                             uint32_t du, uint32_t *__restrict__ count, const uint64_t *__restrict__ row_ptr,
                             uint32_t *__restrict__ col, double *__restrict__ val) {
  const int n = G.N;
  for (uint64_t J = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; J < D; J += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = states[J];
    const double lj = (double)len[J];
    uint32_t k = 0;
    uint64_t out = fill ? row_ptr[J] : 0;
    for (int e = 0; e < t.n; ++e) {
      const uint64_t mc = orb_mask(t.c[e], n), mr = orb_mask(t.r[e], n);
      if (!(b & mc) || (b & mr)) continue;  // Pauli: c_c needs the orbital, c+_r an empty one
      const uint64_t lo = mc < mr ? mc : mr, hi = mc < mr ? mr : mc;
      const int sign = (__popcll(b & (hi - (lo << 1))) & 1) ? -1 : 1;
      const RepMap m = sym_representative(G, b - mc + mr, irrep);
      if (m.length == 0) continue;
      const uint64_t f = (uint64_t)colex_rank((uint32_t)m.rep) + (uint64_t)du * colex_rank((uint32_t)(m.rep >> 32));
      const int32_t K = fmap[f];
      if (K < 0) continue;
      if (fill) {
        col[out] = (uint32_t)K;
        val[out] = (m.phase ? -1.0 : 1.0) * t.v[e] * sign * sqrt(lj / (double)len[K]);
        ++out;
      } else {
        ++k;
      }
    }
    if (!fill) count[J] = k;
  }
}

__global__ void k_mixed_diag(const uint64_t *__restrict__ states, uint64_t D, const uint64_t *__restrict__ dmask,
                             const double *__restrict__ dval, int nd, double *__restrict__ dg) {
  for (uint64_t J = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; J < D; J += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = states[J];
    double d = 0.0;
    for (int k = 0; k < nd; ++k)
      if ((b & dmask[k]) == dmask[k]) d += dval[k];
    dg[J] = d;
  }
}

// Where a row's off-diagonal entries come from. CsrRows: the stored matrix
// (each lane takes every eighth stored entry). OtfRows: computed on the fly,
// with no stored matrix (each lane takes every eighth one-body element and
// evaluates it on the row's state exactly as k_mixed_rows does: Pauli test,
// fermion sign, representative of the image, its basis index, phase and
// orbit-length factor), for sectors whose matrix would not fit or when asked.
struct CsrRows {
  const uint64_t *row_ptr;
  const uint32_t *col;
  const double *val;
  __device__ __forceinline__ double lane_sum(uint64_t J, int lane, const double *__restrict__ x) const {
    double s = 0.0;
    const uint64_t a = row_ptr[J], e = row_ptr[J + 1];
    for (uint64_t k = a + lane; k < e; k += 8) s += val[k] * __ldg(x + col[k]);
    return s;
  }
};

struct OtfRows {
  SymGroup G;
  int irrep;
  OffTerms t;
  const uint64_t *states;
  const uint8_t *len;
  const int32_t *fmap;
  uint32_t du;
  __device__ __forceinline__ double lane_sum(uint64_t J, int lane, const double *__restrict__ x) const {
    const int n = G.N;
    const uint64_t b = states[J];
    const double lj = (double)len[J];
    double s = 0.0;
    for (int e = lane; e < t.n; e += 8) {
      const uint64_t mc = orb_mask(t.c[e], n), mr = orb_mask(t.r[e], n);
      if (!(b & mc) || (b & mr)) continue;
      const uint64_t lo = mc < mr ? mc : mr, hi = mc < mr ? mr : mc;
      const int sign = (__popcll(b & (hi - (lo << 1))) & 1) ? -1 : 1;
      const RepMap m = sym_representative(G, b - mc + mr, irrep);
      if (m.length == 0) continue;
      const uint64_t f = (uint64_t)colex_rank((uint32_t)m.rep) + (uint64_t)du * colex_rank((uint32_t)(m.rep >> 32));
      const int32_t K = fmap[f];
      if (K < 0) continue;
      s += (m.phase ? -1.0 : 1.0) * t.v[e] * sign * sqrt(lj / (double)len[K]) * __ldg(x + K);
    }
    return s;
  }
};

// y = H x: eight lanes per row stride over its entries, then a shuffle sum. A
// warp takes four consecutive rows per pass; the loop bound is the warp's first
// row, the same for all its lanes, so every shuffle sees the whole warp.
template <class Rows>
__global__ void k_mixed_spmv(const Rows R, const double *__restrict__ dg, const double *__restrict__ x,
                             double *__restrict__ y, uint64_t D) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t n_warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 7;
  const int group = (threadIdx.x & 31) >> 3;
  for (uint64_t J0 = warp * 4; J0 < D; J0 += n_warps * 4) {
    const uint64_t J = J0 + group;
    double s = 0.0;
    if (J < D) s = R.lane_sum(J, lane, x);
    s += __shfl_xor_sync(0xffffffffu, s, 4);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    if (J < D && lane == 0) y[J] = dg[J] * x[J] + s;
  }
}

// One ground-state Lanczos step on the mixed basis: w = H v - beta v_prev with
// the per-block partial sums of <v, w> at partials[block * ld] (the layout the
// factorized path's reductions use), rows as in k_mixed_spmv.
template <class Rows>
__global__ void __launch_bounds__(256) k_mixed_lanczos_w(const Rows R, const double *__restrict__ dg,
                                                         const double *__restrict__ v,
                                                         const double *__restrict__ vprev,
                                                         const double *__restrict__ beta_dev,
                                                         double *__restrict__ w, uint64_t D,
                                                         double *__restrict__ partials, int ld) {
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t n_warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 7;
  const int group = (threadIdx.x & 31) >> 3;
  const double beta = *beta_dev;
  double acc = 0.0;
  for (uint64_t J0 = warp * 4; J0 < D; J0 += n_warps * 4) {
    const uint64_t J = J0 + group;
    double s = 0.0;
    if (J < D) s = R.lane_sum(J, lane, v);
    s += __shfl_xor_sync(0xffffffffu, s, 4);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    if (J < D && lane == 0) {
      const double vj = v[J];
      const double wj = dg[J] * vj + s - beta * vprev[J];
      w[J] = wj;
      acc += vj * wj;
    }
  }
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  __shared__ double red[8];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
    partials[(size_t)blockIdx.x * ld] = t;
  }
}

// y = xs H x - sum_k c_k z_k with the reductions of the factorized column pass
// (block partials at partials[block * Reducer::kMaxRed + i]); rows as in
// k_mixed_spmv. *skip != 0: the whole call does nothing.
template <class Rows>
__global__ void __launch_bounds__(256) k_mixed_full(const Rows R, const double *__restrict__ dg,
                                                    const double *__restrict__ x, double xs, double *y, uint64_t D,
                                                    SubList sub, int red_mask, double *partials, const int *skip) {
  if (skip && *skip) return;
  const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
  const uint64_t n_warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
  const int lane = threadIdx.x & 7;
  const int group = (threadIdx.x & 31) >> 3;
  double red[3] = {0.0, 0.0, 0.0};
  for (uint64_t J0 = warp * 4; J0 < D; J0 += n_warps * 4) {
    const uint64_t J = J0 + group;
    double s = 0.0;
    if (J < D) s = R.lane_sum(J, lane, x);
    s += __shfl_xor_sync(0xffffffffu, s, 4);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    if (J < D && lane == 0) {
      const double xj = x[J];
      double yj = xs * (dg[J] * xj + s);
      for (int k = 0; k < sub.n; ++k) yj -= (sub.cdev ? sub.cdev[k] : sub.c[k]) * sub.z[k][J];
      y[J] = yj;
      red[0] += xs * xj * yj;
      red[1] += yj * yj;
      red[2] += xs * xs * xj * xj;
    }
  }
  if (!red_mask) return;
  __shared__ double sm[3][8];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    double v = red[i];
    for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) sm[i][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += sm[threadIdx.x][k];
    partials[(size_t)blockIdx.x * Reducer::kMaxRed + threadIdx.x] = t;
  }
}

struct OrbCoef {
  double c[kMaxSymOrb];
};

// basis index of state b in a sector: through the colex ranks of its two words
__device__ __forceinline__ int32_t mixed_index(const int32_t *fmap, uint32_t du, uint64_t b) {
  return fmap[(uint64_t)colex_rank((uint32_t)b) + (uint64_t)du * colex_rank((uint32_t)(b >> 32))];
}

// phi[J] = (c+ psi)[J]: the target state J carries the created particle; each
// occupied orbital a of the orbital's support, emptied, gives a source state
// whose representative (in the source irrep) holds the amplitude.
__global__ void k_mixed_create(SymGroup G, int r_src, int r_tgt, int spin, int n_sites, OrbCoef cf,
                               const uint64_t *__restrict__ tstates, const uint8_t *__restrict__ tlen, uint64_t Dt,
                               const int32_t *__restrict__ sfmap, uint32_t sdu, const uint8_t *__restrict__ slen,
                               const double *__restrict__ psi, double *__restrict__ phi) {
  const int N = G.N;
  for (uint64_t J = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; J < Dt; J += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = tstates[J];
    const double lj = (double)tlen[J];
    double acc = 0.0;
    for (int a = 0; a < n_sites; ++a) {
      if (cf.c[a] == 0.0) continue;
      const uint64_t m = orb_mask(a + spin * N, N);
      if (!(b & m)) continue;
      const RepMap rm = sym_representative(G, b ^ m, r_src);
      if (rm.length == 0) continue;
      const int32_t I = mixed_index(sfmap, sdu, rm.rep);
      if (I < 0) continue;
      int ph = rm.phase + ((__popcll(b & (m - 1)) & 1) ? G.g : 0);
      ph %= 2 * G.g;
      acc += (ph == 0 ? 1.0 : -1.0) * cf.c[a] * sqrt(lj / (double)rm.length) * psi[I];
    }
    phi[J] = acc;
  }
}

// phi[J] = (c psi)[J]: every source state b' whose orbital a, emptied, lands in
// J's orbit is b' = h(J) + a for a group element h (each distinct image h(J)
// once) and an orbital a that h(J) leaves empty; b' contributes when it is its
// own representative in the source irrep.
__global__ void k_mixed_destroy(SymGroup G, int r_src, int r_tgt, int spin, int n_sites, OrbCoef cf,
                                const uint64_t *__restrict__ tstates, uint64_t Dt, const int32_t *__restrict__ sfmap,
                                uint32_t sdu, const uint8_t *__restrict__ slen, const double *__restrict__ psi,
                                double *__restrict__ phi) {
  const int N = G.N;
  for (uint64_t J = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; J < Dt; J += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t bj = tstates[J];
    uint64_t seen[kMaxGroup];
    int nseen = 0;
    double acc = 0.0;
    for (int h = 0; h < G.g; ++h) {
      int q;
      const uint64_t sh = sym_apply(G, h, 0, bj, q);
      bool dup = false;
      for (int k = 0; k < nseen; ++k) dup |= seen[k] == sh;
      if (dup) continue;
      seen[nseen++] = sh;
      for (int a = 0; a < n_sites; ++a) {
        if (cf.c[a] == 0.0) continue;
        const uint64_t m = orb_mask(a + spin * N, N);
        if (sh & m) continue;
        const uint64_t bs = sh | m;  // the source state
        const RepMap rs = sym_representative(G, bs, r_src);
        if (rs.length == 0 || rs.rep != bs) continue;
        const int32_t I = mixed_index(sfmap, sdu, bs);
        if (I < 0) continue;
        const RepMap rt = sym_representative(G, sh, r_tgt);  // rep bj; its phase and length
        if (rt.length == 0) continue;
        int ph = rt.phase + ((__popcll(bs & (m - 1)) & 1) ? G.g : 0);
        ph %= 2 * G.g;
        acc += (ph == 0 ? 1.0 : -1.0) * cf.c[a] * sqrt((double)slen[I] / (double)rt.length) * psi[I];
      }
    }
    phi[J] = acc;
  }
}

unsigned grid_for(uint64_t n, int threads) {
  static const int sms = [] {
    int dev = 0, v = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v;
  }();
  const uint64_t want = (n + threads - 1) / threads;
  const uint64_t cap = (uint64_t)sms * 16;
  return (unsigned)(want < 1 ? 1 : (want > cap ? cap : want));
}

void upload_binomials() {
  static std::once_flag once;
  std::call_once(once, [] {
    uint32_t h[33][33] = {};
    for (int n = 0; n <= 32; ++n)
      for (int k = 0; k <= n; ++k) h[n][k] = (uint32_t)binom(n, k);
    QED_CUDA(cudaMemcpyToSymbol(c_mbinom, h, sizeof(h)));
    QED_CUDA(cudaDeviceSynchronize());
  });
}

}  // namespace

MixedHamiltonian::MixedHamiltonian(const SymmetryGroup &G, const MixedTerms &t, int irrep, int n_up, int n_dn,
                                   cudaStream_t s) {
  const int N = G.tab.N;
  if (irrep < 0 || irrep >= G.g()) fail(QED_ERR_ARGUMENT, "irrep out of range");
  if (n_up < 0 || n_dn < 0 || n_up > N || n_dn > N) fail(QED_ERR_ARGUMENT, "bad sector for the mixed basis");
  upload_binomials();
  const uint64_t du = binom(N, n_up), dd = binom(N, n_dn), nf = du * dd;
  if (du > 0xffffffffull || dd > 0xffffffffull || nf > 0x7fffffffull)
    fail(QED_ERR_UNSUPPORTED, "sector too large for the mixed-basis index map");
  this->irrep = irrep;
  this->n_up = n_up;
  this->n_dn = n_dn;
  this->du = (uint32_t)du;
  this->dd = (uint32_t)dd;
  group = G.tab;
  DevBuf<uint32_t> us(du), ds(dd);
  launch_unrank(N, n_up, (uint32_t)du, us.p, s);
  launch_unrank(N, n_dn, (uint32_t)dd, ds.p, s);
  DevBuf<uint8_t> lenf(nf);
  k_mixed_mark<<<grid_for(nf, 256), 256, 0, s>>>(G.tab, irrep, us.p, (uint32_t)du, ds.p, nf, lenf.p);
  QED_LAUNCH();
  const uint64_t ntiles = (nf + kMarkTile - 1) / kMarkTile;
  DevBuf<uint32_t> tcount(ntiles);
  k_mixed_tile_count<<<(unsigned)ntiles, kMarkThreads, 0, s>>>(lenf.p, nf, tcount.p);
  QED_LAUNCH();
  std::vector<uint32_t> htc(ntiles);
  tcount.download(htc.data(), ntiles, s);
  QED_CUDA(cudaStreamSynchronize(s));
  std::vector<uint64_t> toff(ntiles);
  uint64_t total = 0;
  for (uint64_t k = 0; k < ntiles; ++k) {
    toff[k] = total;
    total += htc[k];
  }
  D = total;
  DevBuf<uint64_t> dtoff;
  dtoff.upload(toff, s);
  states.alloc(D);
  len.alloc(D);
  fmap.alloc(nf);
  k_mixed_scatter<<<(unsigned)ntiles, kMarkThreads, 0, s>>>(lenf.p, nf, dtoff.p, us.p, (uint32_t)du, ds.p, fmap.p,
                                                            states.p, len.p);
  QED_LAUNCH();
  row_ptr.alloc(D + 1);
  dg.alloc(D);
  if (D == 0) {
    const uint64_t zero = 0;
    row_ptr.upload(&zero, 1, s);
    QED_CUDA(cudaStreamSynchronize(s));
    return;
  }
  term_r.upload(t.r, s);
  term_c.upload(t.c, s);
  term_v.upload(t.v, s);
  n_terms = (int)t.r.size();
  const OffTerms ot{n_terms, term_r.p, term_c.p, term_v.p};
  DevBuf<uint32_t> cnt(D);
  k_mixed_rows<false><<<grid_for(D, 128), 128, 0, s>>>(G.tab, irrep, ot, states.p, len.p, D, fmap.p, (uint32_t)du,
                                                       cnt.p, nullptr, nullptr, nullptr);
  QED_LAUNCH();
  std::vector<uint32_t> hc(D);
  cnt.download(hc.data(), D, s);
  QED_CUDA(cudaStreamSynchronize(s));
  std::vector<uint64_t> rp(D + 1);
  rp[0] = 0;
  for (size_t J = 0; J < D; ++J) rp[J + 1] = rp[J] + hc[J];
  nnz = rp[D];
  // the stored matrix (12 bytes per entry + the row pointers) or, above the
  // size budget or when asked, entries recomputed at every product; sectors
  // that may be diagonalised in full keep the stored form
  const double csr_bytes = 12.0 * (double)nnz + 8.0 * (double)(D + 1);
  on_the_fly = (long)D >= opt_int("max_dim_full") &&
               (opt_bool("mixed_on_the_fly") || csr_bytes > opt_double("mixed_csr_max_gb") * 1e9);
  if (!on_the_fly) {
    row_ptr.upload(rp, s);
    col.alloc(nnz);
    val.alloc(nnz);
    if (nnz)
      k_mixed_rows<true><<<grid_for(D, 128), 128, 0, s>>>(G.tab, irrep, ot, states.p, len.p, D, fmap.p,
                                                          (uint32_t)du, nullptr, row_ptr.p, col.p, val.p);
    QED_LAUNCH();
  }
  DevBuf<uint64_t> dm;
  DevBuf<double> dv;
  dm.upload(t.dmask, s);
  dv.upload(t.dval, s);
  k_mixed_diag<<<grid_for(D, 256), 256, 0, s>>>(states.p, D, dm.p, dv.p, (int)t.dmask.size(), dg.p);
  QED_LAUNCH();
  QED_CUDA(cudaStreamSynchronize(s));
}

namespace {
CsrRows csr_rows(const MixedHamiltonian &H) { return CsrRows{H.row_ptr.p, H.col.p, H.val.p}; }
OtfRows otf_rows(const MixedHamiltonian &H) {
  return OtfRows{H.group, H.irrep, OffTerms{H.n_terms, H.term_r.p, H.term_c.p, H.term_v.p}, H.states.p, H.len.p,
                 H.fmap.p, H.du};
}
}  // namespace

int MixedHamiltonian::lanczos_w(const double *v, const double *vprev, const double *beta_dev, double *w,
                                double *partials, int ld, int max_blocks, cudaStream_t s) const {
  unsigned nb = grid_for(D * 8, 256);
  if (nb > (unsigned)max_blocks) nb = (unsigned)max_blocks;
  if (on_the_fly)
    k_mixed_lanczos_w<<<nb, 256, 0, s>>>(otf_rows(*this), dg.p, v, vprev, beta_dev, w, D, partials, ld);
  else
    k_mixed_lanczos_w<<<nb, 256, 0, s>>>(csr_rows(*this), dg.p, v, vprev, beta_dev, w, D, partials, ld);
  QED_LAUNCH();
  return (int)nb;
}

void MixedHamiltonian::apply(const double *x, double *y, cudaStream_t s) const {
  if (!D) return;
  if (on_the_fly)
    k_mixed_spmv<<<grid_for(D * 8, 256), 256, 0, s>>>(otf_rows(*this), dg.p, x, y, D);
  else
    k_mixed_spmv<<<grid_for(D * 8, 256), 256, 0, s>>>(csr_rows(*this), dg.p, x, y, D);
  QED_LAUNCH();
}

int MixedHamiltonian::apply_full(const double *x, double xs, double *y, const SubList &sub, int red_mask,
                                 Reducer &r, cudaStream_t s, const int *skip) const {
  if (!D) return 0;
  unsigned nb = grid_for(D * 8, 256);
  if (red_mask && nb > (unsigned)r.max_blocks) nb = (unsigned)r.max_blocks;
  if (on_the_fly)
    k_mixed_full<<<nb, 256, 0, s>>>(otf_rows(*this), dg.p, x, xs, y, D, sub, red_mask, r.partials, skip);
  else
    k_mixed_full<<<nb, 256, 0, s>>>(csr_rows(*this), dg.p, x, xs, y, D, sub, red_mask, r.partials, skip);
  QED_LAUNCH();
  return (int)nb;
}

std::vector<double> MixedHamiltonian::dense(cudaStream_t s) const {
  if (on_the_fly) fail(QED_ERR_INTERNAL, "dense form of an on-the-fly mixed Hamiltonian");
  std::vector<uint64_t> rp(D + 1);
  std::vector<uint32_t> c(nnz);
  std::vector<double> v(nnz), d(D), out(D * D, 0.0);
  row_ptr.download(rp.data(), D + 1, s);
  if (nnz) {
    col.download(c.data(), nnz, s);
    val.download(v.data(), nnz, s);
  }
  dg.download(d.data(), D, s);
  QED_CUDA(cudaStreamSynchronize(s));
  for (size_t J = 0; J < D; ++J) {
    out[J + D * J] += d[J];
    for (uint64_t k = rp[J]; k < rp[J + 1]; ++k) out[J + D * c[k]] += v[k];
  }
  return out;
}

void mixed_cdag(const MixedHamiltonian &src, const MixedHamiltonian &tgt, int pm, int spin, int n_sites,
                const double *coef, const double *psi, double *phi, cudaStream_t s) {
  if (!tgt.D) return;
  if (n_sites > kMaxSymOrb) fail(QED_ERR_UNSUPPORTED, "more than 32 sites");
  OrbCoef cf{};
  for (int a = 0; a < n_sites; ++a) cf.c[a] = coef[a];
  if (pm == 1)
    k_mixed_create<<<grid_for(tgt.D, 128), 128, 0, s>>>(src.group, src.irrep, tgt.irrep, spin, n_sites, cf,
                                                        tgt.states.p, tgt.len.p, tgt.D, src.fmap.p, src.du, src.len.p,
                                                        psi, phi);
  else
    k_mixed_destroy<<<grid_for(tgt.D, 128), 128, 0, s>>>(src.group, src.irrep, tgt.irrep, spin, n_sites, cf,
                                                         tgt.states.p, tgt.D, src.fmap.p, src.du, src.len.p, psi,
                                                         phi);
  QED_LAUNCH();
}

}  // namespace qed
