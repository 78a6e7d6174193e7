// Window form of the spin-factorized H.v (see winhv.hpp): planner, host check,
// code generator, NVRTC module cache and launcher.
#include "winhv.hpp"

#include <dlfcn.h>
#include <nvrtc.h>

#include <algorithm>
#include <array>
#include <atomic>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <sstream>

#include "common.hpp"
#include "options.hpp"

namespace qed {

namespace {

// Bits strictly between sites a and b (the sites the fermion sign counts).
uint32_t between_bits(int a, int b) {
  const int lo = std::min(a, b), hi = std::max(a, b);
  return (uint32_t)(((1ull << hi) - 1ull) & ~((2ull << lo) - 1ull));
}

// The w-bit patterns with k set bits, ascending: member j of a group with k
// particles inside the window has pattern patterns(w, k)[j] there.
std::vector<uint32_t> patterns(int w, int k) {
  std::vector<uint32_t> v;
  for (uint32_t a = 0; a < (1u << w); ++a)
    if (__builtin_popcount(a) == k) v.push_back(a);
  return v;
}

// One term of a window matrix: member j gathers (-1)^neg amp[q] x[member src].
struct Term {
  int q, src;
  bool neg;
};

// The window's matrix for k particles inside it, row by row; the terms of a row
// come in increasing pair order. Hop c+_r c_c is allowed when bit c is set and
// bit r empty; it reaches the pattern with c and r exchanged, with the parity of
// the set bits strictly between r and c (k_build_hops applies the same rule to
// whole strings; the window holds every bit between r and c).
std::vector<std::vector<Term>> window_terms(const WindowPlan &P, const WindowPlan::Window &W, int k) {
  const std::vector<uint32_t> pat = patterns(W.w, k);
  std::vector<int> idx(1u << W.w, -1);
  for (size_t j = 0; j < pat.size(); ++j) idx[pat[j]] = (int)j;
  std::vector<std::vector<Term>> out(pat.size());
  for (size_t j = 0; j < pat.size(); ++j) {
    const uint32_t a = pat[j];
    for (int q : W.pairs) {
      const int r = P.pd[q] - W.lo, c = P.ps[q] - W.lo;
      if (!((a >> c) & 1u) || ((a >> r) & 1u)) continue;
      const uint32_t na = a ^ (1u << c) ^ (1u << r);
      out[j].push_back({q, idx[na], (__builtin_popcount(na & between_bits(r, c)) & 1) != 0});
    }
  }
  return out;
}

size_t count_terms(const std::vector<std::vector<Term>> &t) {
  size_t n = 0;
  for (const auto &r : t) n += r.size();
  return n;
}

}  // namespace

bool plan_windows(int L, int N, const std::vector<uint32_t> &bits, const std::vector<int> &pd,
                  const std::vector<int> &ps, WindowPlan &P) {
  P = WindowPlan();
  P.L = L;
  P.N = N;
  P.dim = (uint32_t)bits.size();
  P.pd = pd;
  P.ps = ps;
  const int np = (int)pd.size();
  if (!P.dim || P.dim > kWinMaxDim || np == 0 || np > kWinMaxPairs || ps.size() != pd.size() || L > 32)
    return false;
  for (size_t i = 1; i < bits.size(); ++i)
    if (bits[i] <= bits[i - 1]) return false;
  // windows: greedy cover of the pairs' spans, by their lower site
  const int w = std::min(L, kWinMaxSites);
  std::vector<int> order(np);
  std::iota(order.begin(), order.end(), 0);
  auto lo_of = [&](int q) { return std::min(pd[q], ps[q]); };
  auto hi_of = [&](int q) { return std::max(pd[q], ps[q]); };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return lo_of(a) < lo_of(b); });
  std::vector<int> owner(np, -1);
  for (int q : order) {
    const int a = lo_of(q), b = hi_of(q);
    if (a == b || b - a >= w) return false;
    for (size_t k = 0; k < P.win.size() && owner[q] < 0; ++k)
      if (P.win[k].lo <= a && b < P.win[k].lo + P.win[k].w) owner[q] = (int)k;
    if (owner[q] < 0) {
      if ((int)P.win.size() == kWinMaxWindows) return false;
      WindowPlan::Window W;
      W.lo = std::min(a, L - w);
      W.w = w;
      P.win.push_back(W);
      owner[q] = (int)P.win.size() - 1;
    }
  }
  for (int q = 0; q < np; ++q) P.win[owner[q]].pairs.push_back(q);
  P.tile_stride = (int)((P.dim + 2 + 1) & ~1u);
  // Row of a string = its colex rank, sum over its set bits p_1 < ... < p_N of
  // C(p_t, t) (the basis is the N-subsets in increasing order). For a window the
  // bits below it (nB of them) and above it give a per-group constant; the
  // window's own bits q_1 < ... < q_k give sum_i C(lo + q_i, nB + i), which
  // depends on the member pattern and nB only. Groups are blocked by (k, nB)
  // so that this part is uniform across a warp (table cu, in constant memory).
  const int nw = (int)P.win.size();
  std::vector<std::vector<std::array<int, 3>>> entries(nw * kWinWarps);  // (k, cu base, tab base)
  for (int wi = 0; wi < nw; ++wi) {
    const WindowPlan::Window &W = P.win[wi];
    const uint32_t mask = ((1u << W.w) - 1u) << W.lo;
    std::map<uint32_t, int> gid;
    std::vector<uint32_t> gf;
    for (uint32_t i = 0; i < P.dim; ++i) {
      const uint32_t f = bits[i] & ~mask;
      if (gid.emplace(f, (int)gf.size()).second) gf.push_back(f);
    }
    const int ng = (int)gf.size();
    std::vector<int> gk(ng), gb(ng);
    for (int g = 0; g < ng; ++g) {
      gk[g] = N - __builtin_popcount(gf[g]);
      gb[g] = __builtin_popcount(gf[g] & ((1u << W.lo) - 1u));
      if (gk[g] < 0 || gk[g] > W.w) return false;
    }
    std::vector<size_t> cost_k(W.w + 1);
    for (int k = 0; k <= W.w; ++k) cost_k[k] = count_terms(window_terms(P, W, k));
    // uniform parts per (k, nB), byte offsets
    std::map<std::pair<int, int>, int> cu_base;
    auto uniform_base = [&](int k, int nb) {
      auto it = cu_base.find({k, nb});
      if (it != cu_base.end()) return it->second;
      const int base = (int)P.cu.size();
      for (uint32_t a : patterns(W.w, k)) {
        uint64_t r = 0;
        int t = nb;
        for (int q = 0; q < W.w; ++q)
          if ((a >> q) & 1u) r += binom(W.lo + q, ++t);
        P.cu.push_back((uint32_t)(8 * r));
      }
      cu_base[{k, nb}] = base;
      return base;
    };
    // per-group constant: the bits outside the window (those above it come
    // after the k window bits in the rank's order)
    auto group_const = [&](int g) {
      uint64_t r = 0;
      int t = 0;
      for (int p = 0; p < L; ++p)
        if ((gf[g] >> p) & 1u) {
          ++t;
          r += binom(p, p < W.lo ? t : t + gk[g]);
        }
      return r;
    };
    std::vector<int> ord(ng);
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
      return gk[a] != gk[b] ? gk[a] < gk[b] : gb[a] < gb[b];
    });
    struct Blk {
      int k, ub;
      uint32_t base;
      double cost;
    };
    std::vector<Blk> blks;
    for (int s = 0; s < ng;) {
      const int k = gk[ord[s]], nb = gb[ord[s]];
      int e = s;
      while (e < ng && e - s < 32 && gk[ord[e]] == k && gb[ord[e]] == nb) ++e;
      if (wi == 0 || cost_k[k] > 0) {
        const int ub = uniform_base(k, nb);
        const uint32_t base = (uint32_t)P.tab.size();
        P.tab.resize(P.tab.size() + 32, kWinPadLane);
        for (int l = 0; l < e - s; ++l) P.tab[base + l] = (uint32_t)(8 * group_const(ord[s + l]));
        blks.push_back({k, ub, base, (double)cost_k[k] + 3.0 * binom(W.w, k)});
      }
      s = e;
    }
    // longest block first onto the least loaded warp
    std::stable_sort(blks.begin(), blks.end(), [](const Blk &a, const Blk &b) { return a.cost > b.cost; });
    std::vector<double> load(kWinWarps, 0.0);
    for (const Blk &b : blks) {
      const int wq = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      load[wq] += b.cost;
      entries[wi * kWinWarps + wq].push_back({b.k, b.ub, (int)b.base});
    }
  }
  if (P.cu.size() > kWinMaxUniform) return false;  // constant memory of the module
  P.sched.assign((size_t)nw * (kWinWarps + 1), 0);
  std::vector<int> ent;
  for (int wi = 0; wi < nw; ++wi) {
    for (int wq = 0; wq < kWinWarps; ++wq) {
      P.sched[wi * (kWinWarps + 1) + wq] = (int)(ent.size() / 3);
      for (const auto &e : entries[wi * kWinWarps + wq]) ent.insert(ent.end(), e.begin(), e.end());
    }
    P.sched[wi * (kWinWarps + 1) + kWinWarps] = (int)(ent.size() / 3);
  }
  P.sched.insert(P.sched.end(), ent.begin(), ent.end());
  return true;
}

void window_apply_host(const WindowPlan &P, const std::vector<double> &amp, const double *x, double *y) {
  std::fill(y, y + P.dim, 0.0);
  const int nw = (int)P.win.size();
  const int *ent = P.sched.data() + (size_t)nw * (kWinWarps + 1);
  for (int wi = 0; wi < nw; ++wi) {
    const int e0 = P.sched[wi * (kWinWarps + 1)], e1 = P.sched[wi * (kWinWarps + 1) + kWinWarps];
    for (int e = e0; e < e1; ++e) {
      const int k = ent[3 * e], ub = ent[3 * e + 1];
      const uint32_t base = (uint32_t)ent[3 * e + 2];
      const auto terms = window_terms(P, P.win[wi], k);
      for (int lane = 0; lane < 32; ++lane) {
        const uint32_t cg = P.tab[base + lane];
        if (cg == kWinPadLane) continue;
        auto row = [&](int j) { return (cg + P.cu[ub + j]) / 8; };
        for (size_t j = 0; j < terms.size(); ++j) {
          double a = 0.0;
          for (const Term &t : terms[j]) a += (t.neg ? -amp[t.q] : amp[t.q]) * x[row(t.src)];
          y[row((int)j)] += a;
        }
      }
    }
  }
}

// ------------------------------------------------------------ code generator --

namespace {

// Definitions shared by the generated kernels. SubList has the layout of the
// host struct of the same name (kernels.cuh); Amp carries one amplitude per
// hopping pair (kernel parameter, read from the constant bank).
const char *kPrelude = R"(
typedef unsigned int u32;
typedef unsigned long long u64;
struct Amp { double v[256]; };
struct SubList { int n; double c[32]; const double *z[32]; const double *cdev; };
extern __shared__ __align__(16) double sm[];
#define XT(o) (*reinterpret_cast<const double *>(reinterpret_cast<const char *>(sm) + (o)))
#define YT(ts, o) (*reinterpret_cast<double *>(reinterpret_cast<char *>(sm) + (ts) + (o)))
__device__ __forceinline__ u32 smem_addr(const void *p) { return (u32)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }
)";

// Inter-spin density-density term, the rule of inter_term (kernels.cu).
const char *kInter = R"(
__device__ __forceinline__ double w_inter(int mode, int n, double u, const double *__restrict__ v, u32 up, u32 dn) {
  if (mode == 1) return u * (double)__popc(up & dn);
  double s = 0.0;
  if (mode == 2) {
    u32 w = up & dn;
    while (w) { const int r = __ffs(w) - 1; s += __ldg(v + r); w &= w - 1; }
  } else if (mode == 3) {
    u32 wd = dn;
    while (wd) {
      const int r = __ffs(wd) - 1;
      u32 wu = up;
      while (wu) { const int c = __ffs(wu) - 1; s += __ldg(v + r * n + c); wu &= wu - 1; }
      wd &= wd - 1;
    }
  }
  return s;
}
)";

// Up-spin pass (first): y = xs ((diag + up hops) x) - sum_k c_k z_k. A CTA
// takes whole dn rows: the row is copied into the x tile (16-byte cp.async when
// aligned), the windows write the hop sums into the accumulator tile, and the
// epilogue combines them with the diagonal and the subtraction terms (loads of
// four elements per thread issued before any is used). y is only written.
const char *kUpPass = R"(
#define EU 4
extern "C" __global__ void __launch_bounds__(256, 1)
win_up_pass(const double *__restrict__ x, double *__restrict__ y, double xs, u32 du, u32 dd,
            const u32 *__restrict__ tab, const int *__restrict__ sched, const __grid_constant__ Amp A,
            const int *skip, const double *__restrict__ diag_up, const double *__restrict__ diag_dn,
            const u32 *__restrict__ bits_up, const u32 *__restrict__ bits_dn, int imode, int in, double iu,
            const double *__restrict__ iv, const __grid_constant__ SubList sub, int vec16) {
  if (skip && *skip) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (u32 d = blockIdx.x; d < dd; d += gridDim.x) {
    const size_t row = (size_t)d * du;
    if (vec16)
      for (u32 q = threadIdx.x; q < du / 2; q += 256) cp_async16(sm + 2 * q, x + row + 2 * q);
    else
      for (u32 i = threadIdx.x; i < du; i += 256) cp_async8(sm + i, x + row + i);
    cp_async_wait_all();
    __syncthreads();
    u_windows(warp, lane, tab, sched, A);
    const u32 bd = bits_dn[d];
    const double ed = diag_dn[d];
    for (u32 i0 = threadIdx.x; i0 < du; i0 += 256 * EU) {
      double a[EU];
#pragma unroll
      for (int e = 0; e < EU; ++e) {
        const u32 i = i0 + 256 * e;
        if (i < du) {
          const double dg = __ldg(diag_up + i) + ed + w_inter(imode, in, iu, iv, __ldg(bits_up + i), bd);
          a[e] = (dg * sm[i] + YT(U_TSB, 8u * i)) * xs;
        }
      }
      for (int s = 0; s < sub.n; ++s) {
        const double cs = sub.cdev ? sub.cdev[s] : sub.c[s];
        const double *z = sub.z[s] + row;
#pragma unroll
        for (int e = 0; e < EU; ++e)
          if (i0 + 256 * e < du) a[e] -= cs * z[i0 + 256 * e];
      }
#pragma unroll
      for (int e = 0; e < EU; ++e)
        if (i0 + 256 * e < du) y[row + i0 + 256 * e] = a[e];
    }
    __syncthreads();
  }
}
)";

// Down-spin pass (second): y += (dn hops)(xs x), with the reductions <x, y>,
// <y, y>, <x, x> of the result (xs applied as the up-spin pass does). CTA b
// takes columns b, b + G, b + 2G (G CTAs), so that neighbouring CTAs read
// neighbouring columns at the same time and share each 32-byte sector of x
// and y in L2. A column of x and of y (the up-spin pass's result) are copied
// into the x tile and the accumulator (cp.async, 8 bytes each, all in flight
// at once), the windows add their products, and the epilogue stores the
// column and takes the reductions from the two tiles.
const char *kDnPass = R"(
extern "C" __global__ void __launch_bounds__(256, 1)
win_dn_pass(const double *__restrict__ x, double *y, double xs, u32 du, u32 dd,
            const u32 *__restrict__ tab, const int *__restrict__ sched, const __grid_constant__ Amp A,
            const int *skip, int red_mask, double *partials) {
  if (skip && *skip) return;
  __shared__ double rs[3][8];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double r0 = 0.0, r1 = 0.0, r2 = 0.0;
  for (u32 u = blockIdx.x; u < du; u += gridDim.x) {
    for (u32 i = threadIdx.x; i < dd; i += 256) {
      cp_async8(sm + i, x + (size_t)i * du + u);
      cp_async8(&YT(D_TSB, 8u * i), y + (size_t)i * du + u);
    }
    cp_async_wait_all();
    __syncthreads();
    if (xs != 1.0) {
      for (u32 i = threadIdx.x; i < dd; i += 256) sm[i] *= xs;
      __syncthreads();
    }
    d_windows(warp, lane, tab, sched, A);
    for (u32 i = threadIdx.x; i < dd; i += 256) {
      const double v = YT(D_TSB, 8u * i), xv = sm[i];
      r0 += xv * v;
      r1 += v * v;
      r2 += xv * xv;
      y[(size_t)i * du + u] = v;
    }
    __syncthreads();
  }
  if (red_mask) {
    double v[3] = {r0, r1, r2};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      double t = v[k];
      for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
      if (lane == 0) rs[k][warp] = t;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
      double s = 0.0;
      for (int w = 0; w < 8; ++w) s += rs[threadIdx.x][w];
      partials[(size_t)blockIdx.x * 72 + threadIdx.x] = s;
    }
  }
}
)";

std::string coef(const Term &t) { return std::string(t.neg ? "-A.v[" : "A.v[") + std::to_string(t.q) + "]"; }

// The window functions of one spin (prefix S: "u" or "d") and its dispatcher
// S_windows, which runs every window of the plan with a CTA barrier after each.
void emit_spin(std::ostringstream &o, const char *S, const WindowPlan &P) {
  // The up spin's windows write the accumulator (the first window stores, zero
  // for strings without hops in it); the down spin's add to the up-spin result.
  const bool first_stores = S[0] == 'u';
  const std::string tsb = std::string(S[0] == 'u' ? "U_TSB" : "D_TSB");
  o << "#define " << tsb << " " << 8u * (unsigned)P.tile_stride << "u\n";
  o << "__constant__ u32 " << S << "_cu[" << std::max<size_t>(P.cu.size(), 1) << "] = {";
  for (size_t i = 0; i < P.cu.size(); ++i) o << (i ? "," : "") << P.cu[i] << "u";
  o << (P.cu.empty() ? "0u" : "") << "};\n";
  const int nw = (int)P.win.size();
  std::vector<std::vector<bool>> have(nw);
  for (int wi = 0; wi < nw; ++wi) {
    const WindowPlan::Window &W = P.win[wi];
    have[wi].assign(W.w + 1, false);
    const bool stores = first_stores && wi == 0;
    for (int k = 0; k <= W.w; ++k) {
      const auto terms = window_terms(P, W, k);
      if (!stores && count_terms(terms) == 0) continue;
      have[wi][k] = true;
      const int m = (int)terms.size();
      // member j's tile byte offset: the lane's group constant cg plus the
      // block's uniform part cu[ub + j] (constant memory)
      o << "__device__ __forceinline__ void " << S << "_w" << wi << "_k" << k
        << "(u32 cg, int ub, const Amp &A) {\n";
      // operands are loaded where first used, so that fewer are live at once
      std::vector<bool> loaded(m, false);
      for (int j = 0; j < m; ++j) {
        for (const Term &t : terms[j])
          if (!loaded[t.src]) {
            loaded[t.src] = true;
            o << "  const double x" << t.src << " = XT(cg + " << S << "_cu[ub + " << t.src << "]);\n";
          }
        const std::string at = "cg + " + std::string(S) + "_cu[ub + " + std::to_string(j) + "]";
        if (terms[j].empty()) {
          if (stores) o << "  YT(" << tsb << ", " << at << ") = 0.0;\n";
          continue;
        }
        o << "  { double a = __dmul_rn(" << coef(terms[j][0]) << ", x" << terms[j][0].src << ");";
        for (size_t h = 1; h < terms[j].size(); ++h)
          o << " a = __fma_rn(" << coef(terms[j][h]) << ", x" << terms[j][h].src << ", a);";
        o << " YT(" << tsb << ", " << at << ")" << (stores ? " = a; }\n" : " += a; }\n");
      }
      o << "}\n";
    }
  }
  o << "__device__ __forceinline__ void " << S
    << "_windows(int warp, int lane, const u32 *__restrict__ tab, const int *__restrict__ sched, const Amp &A) {\n"
    << "  const int *ent = sched + " << nw * (kWinWarps + 1) << ";\n";
  for (int wi = 0; wi < nw; ++wi) {
    o << "  for (int e = sched[" << wi * (kWinWarps + 1) << " + warp]; e < sched[" << wi * (kWinWarps + 1)
      << " + warp + 1]; ++e) {\n"
      << "    const int k = ent[3 * e], ub = ent[3 * e + 1];\n"
      << "    const u32 cg = __ldg(tab + ent[3 * e + 2] + lane);\n"
      << "    if (cg == " << kWinPadLane << "u) continue;\n    switch (k) {\n";
    for (int k = 0; k <= P.win[wi].w; ++k)
      if (have[wi][k]) o << "      case " << k << ": " << S << "_w" << wi << "_k" << k << "(cg, ub, A); break;\n";
    o << "      default: break;\n    }\n  }\n  __syncthreads();\n";
  }
  o << "}\n";
}

}  // namespace

std::string window_source(const WindowPlan &up, const WindowPlan &dn) {
  std::ostringstream o;
  o << kPrelude << kInter;
  emit_spin(o, "u", up);
  emit_spin(o, "d", dn);
  o << kDnPass << kUpPass;
  return o.str();
}

// ------------------------------------------------------- NVRTC and modules --

namespace {

// NVRTC, opened on first use so that the library loads where it is absent (the
// window kernels are then not used).
struct Nvrtc {
  bool ok = false;
  std::string why;
  nvrtcResult (*create)(nvrtcProgram *, const char *, const char *, int, const char *const *,
                        const char *const *) = nullptr;
  nvrtcResult (*compile)(nvrtcProgram, int, const char *const *) = nullptr;
  nvrtcResult (*log_size)(nvrtcProgram, size_t *) = nullptr;
  nvrtcResult (*log)(nvrtcProgram, char *) = nullptr;
  nvrtcResult (*cubin_size)(nvrtcProgram, size_t *) = nullptr;
  nvrtcResult (*cubin)(nvrtcProgram, char *) = nullptr;
  nvrtcResult (*destroy)(nvrtcProgram *) = nullptr;
};

const Nvrtc &nvrtc() {
  static const Nvrtc n = [] {
    Nvrtc n;
    std::vector<std::string> names = {"libnvrtc.so.12", "libnvrtc.so"};
    const char *home = getenv("CUDA_HOME");
    names.push_back(std::string(home ? home : "/usr/local/cuda") + "/lib64/libnvrtc.so.12");
    void *h = nullptr;
    for (const auto &s : names)
      if ((h = dlopen(s.c_str(), RTLD_NOW | RTLD_LOCAL))) break;
    if (!h) {
      n.why = "libnvrtc.so.12 not found";
      return n;
    }
    auto sym = [&](const char *name) { return dlsym(h, name); };
    n.create = reinterpret_cast<decltype(n.create)>(sym("nvrtcCreateProgram"));
    n.compile = reinterpret_cast<decltype(n.compile)>(sym("nvrtcCompileProgram"));
    n.log_size = reinterpret_cast<decltype(n.log_size)>(sym("nvrtcGetProgramLogSize"));
    n.log = reinterpret_cast<decltype(n.log)>(sym("nvrtcGetProgramLog"));
    n.cubin_size = reinterpret_cast<decltype(n.cubin_size)>(sym("nvrtcGetCUBINSize"));
    n.cubin = reinterpret_cast<decltype(n.cubin)>(sym("nvrtcGetCUBIN"));
    n.destroy = reinterpret_cast<decltype(n.destroy)>(sym("nvrtcDestroyProgram"));
    n.ok = n.create && n.compile && n.log_size && n.log && n.cubin_size && n.cubin && n.destroy;
    if (!n.ok) n.why = "libnvrtc lacks an entry point";
    return n;
  }();
  return n;
}

// Compiles `src` for sm_100a; returns the cubin (empty on failure) and the log.
std::vector<char> compile_cubin(const std::string &src, std::string &log, bool verbose) {
  const Nvrtc &N = nvrtc();
  if (!N.ok) {
    log = N.why;
    return {};
  }
  nvrtcProgram p = nullptr;
  if (N.create(&p, src.c_str(), "qed_window_hv.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) {
    log = "nvrtcCreateProgram failed";
    return {};
  }
  std::vector<const char *> opts = {"--gpu-architecture=sm_100a", "--std=c++17", "-lineinfo"};
  if (verbose) opts.push_back("--ptxas-options=-v");
  const nvrtcResult rc = N.compile(p, (int)opts.size(), opts.data());
  size_t ls = 0;
  N.log_size(p, &ls);
  log.assign(ls, '\0');
  if (ls) N.log(p, &log[0]);
  while (!log.empty() && log.back() == '\0') log.pop_back();
  std::vector<char> bin;
  if (rc == NVRTC_SUCCESS) {
    size_t n = 0;
    N.cubin_size(p, &n);
    bin.resize(n);
    if (n) N.cubin(p, bin.data());
  }
  N.destroy(&p);
  return bin;
}

std::string structure_key(const WindowPlan &P) {
  std::ostringstream o;
  o << P.L << ',' << P.N << ':';
  for (size_t q = 0; q < P.pd.size(); ++q) o << P.pd[q] << '-' << P.ps[q] << ' ';
  return o.str();
}

struct HostAmp {
  double v[256];
};
static_assert(sizeof(HostAmp) == 2048, "Amp layout");
static_assert(sizeof(SubList) == 8 + 32 * 8 + 32 * 8 + 8, "SubList layout of the generated kernels");

}  // namespace

struct WinModule {
  cudaLibrary_t lib = nullptr;
  cudaKernel_t kdn = nullptr, kup = nullptr;
  DevBuf<uint32_t> tab_up, tab_dn;
  DevBuf<int> sched_up, sched_dn;
  uint32_t du = 0, dd = 0;
  size_t smem_up = 0, smem_dn = 0;
  ~WinModule() {
    if (lib) cudaLibraryUnload(lib);
  }
};

std::string window_compile_log(const WindowPlan &up, const WindowPlan &dn, bool *ok) {
  std::string log;
  const std::vector<char> bin = compile_cubin(window_source(up, dn), log, true);
  if (ok) *ok = !bin.empty();
  return log;
}

std::shared_ptr<const WinModule> window_module(const WindowPlan &up, const WindowPlan &dn, std::string *why) {
  // modules live for the process (the map is never destroyed: no device frees
  // after the runtime has shut down)
  static std::mutex *mtx = new std::mutex;
  static auto *cache = new std::map<std::string, std::shared_ptr<const WinModule>>;
  static auto *failed = new std::map<std::string, std::string>;
  const std::string key = structure_key(up) + "|" + structure_key(dn);
  int dev = 0;
  QED_CUDA(cudaGetDevice(&dev));
  const std::string dkey = key + "@" + std::to_string(dev);
  std::lock_guard<std::mutex> l(*mtx);
  if (auto it = cache->find(dkey); it != cache->end()) return it->second;
  if (auto it = failed->find(key); it != failed->end()) {
    if (why) *why = it->second;
    return nullptr;
  }
  std::string log;
  const std::vector<char> bin = compile_cubin(window_source(up, dn), log, false);
  if (bin.empty()) {
    (*failed)[key] = "window kernels did not compile: " + log.substr(0, 2000);
    if (why) *why = (*failed)[key];
    return nullptr;
  }
  auto m = std::make_shared<WinModule>();
  QED_CUDA(cudaLibraryLoadData(&m->lib, bin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
  QED_CUDA(cudaLibraryGetKernel(&m->kdn, m->lib, "win_dn_pass"));
  QED_CUDA(cudaLibraryGetKernel(&m->kup, m->lib, "win_up_pass"));
  m->du = up.dim;
  m->dd = dn.dim;
  m->smem_up = 2 * (size_t)up.tile_stride * sizeof(double);
  m->smem_dn = 2 * (size_t)dn.tile_stride * sizeof(double);
  QED_CUDA(cudaKernelSetAttributeForDevice(m->kup, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m->smem_up, dev));
  QED_CUDA(cudaKernelSetAttributeForDevice(m->kdn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)m->smem_dn, dev));
  cudaStream_t s = alloc_stream();
  m->tab_up.upload(up.tab, s);
  m->tab_dn.upload(dn.tab, s);
  m->sched_up.upload(up.sched, s);
  m->sched_dn.upload(dn.sched, s);
  QED_CUDA(cudaStreamSynchronize(s));
  (*cache)[dkey] = m;
  return m;
}

bool window_usable(const HvOperator &op, const double *x, const double *y, const SubList &sub) {
  if (!op.win || x == y) return false;
  const WinBinding &b = *static_cast<const WinBinding *>(op.win);
  if (!b.mod || b.mod->du != op.up.dim || b.mod->dd != op.dn.dim) return false;
  for (int k = 0; k < sub.n; ++k)
    if (sub.z[k] == y) return false;  // the down-spin pass overwrites y before the up-spin pass reads z
  return true;
}

namespace {
std::atomic<long long> g_window_launches{0};
}

long long window_launches() { return g_window_launches.load(std::memory_order_relaxed); }

int launch_hv_windows(const HvOperator &op, const double *x, double xs, double *y, const SubList &sub,
                      int red_mask, Reducer &r, cudaStream_t s) {
  g_window_launches.fetch_add(1, std::memory_order_relaxed);
  const WinBinding &b = *static_cast<const WinBinding *>(op.win);
  const WinModule &M = *b.mod;
  HostAmp au{}, ad{};
  for (size_t q = 0; q < b.amp_up.size() && q < 256; ++q) au.v[q] = b.amp_up[q];
  for (size_t q = 0; q < b.amp_dn.size() && q < 256; ++q) ad.v[q] = b.amp_dn[q];
  uint32_t du = op.up.dim, dd = op.dn.dim;
  const int sms = op.num_sms > 0 ? op.num_sms : 148;
  const double *xp = x;
  double *yp = y;
  const uint32_t *tdn = M.tab_dn.p, *tup = M.tab_up.p;
  const int *sdn = M.sched_dn.p, *sup = M.sched_up.p;
  const int *skip = op.skip;
  const double *dup = op.up.diag, *ddn = op.dn.diag, *iv = op.inter.v;
  const uint32_t *bup = op.up.bits, *bdn = op.dn.bits;
  int imode = op.inter.mode, in = op.inter.n, rm = red_mask;
  double iu = op.inter.u;
  double *part = r.partials;
  int vec16 = (du % 2 == 0 && ((uintptr_t)x & 15u) == 0) ? 1 : 0;
  SubList sl = sub;
  {
    const int grid = (int)std::min<uint32_t>(dd, (uint32_t)sms);
    void *args[] = {&xp, &yp, &xs, &du, &dd, &tup, &sup, &au, &skip, &dup, &ddn, &bup, &bdn,
                    &imode, &in, &iu, &iv, &sl, &vec16};
    QED_CUDA(cudaLaunchKernel((const void *)M.kup, dim3(grid), dim3(256), args, M.smem_up, s));
  }
  int grid = (int)std::min<uint32_t>(du, (uint32_t)sms);
  if (red_mask && grid > r.max_blocks) grid = r.max_blocks;
  void *args[] = {&xp, &yp, &xs, &du, &dd, &tdn, &sdn, &ad, &skip, &rm, &part};
  QED_CUDA(cudaLaunchKernel((const void *)M.kdn, dim3(grid), dim3(256), args, M.smem_dn, s));
  return grid;
}

}  // namespace qed
