// Device sector Hamiltonian and Krylov drivers (see solver.hpp).
#include "solver.hpp"
#include "mixed.hpp"

#include <algorithm>
#include <functional>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>

#include "bank_order.hpp"
#include "eigen.hpp"
#include "options.hpp"
#include "profile.hpp"

namespace qed {

// ---------------------------------------------------------------- Workspace --

namespace {
thread_local cudaStream_t tls_stream = nullptr;  // stream of this thread's Workspace
}

cudaStream_t alloc_stream() { return tls_stream; }

Workspace::Workspace() {
  QED_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  tls_stream = stream;
  red.max_blocks = 4096;
  partials.alloc((size_t)red.max_blocks * Reducer::kMaxRed);
  out.alloc(Reducer::kMaxRed);
  QED_CUDA(cudaMallocHost(&host, Reducer::kMaxRed * sizeof(double)));
  QED_CUDA(cudaMallocHost(&wait_flag, sizeof(int)));
  *wait_flag = 0;
  red.partials = partials.p;
  red.out = out.p;
  red.host = host;
  sync();
}

Workspace::~Workspace() {
  // free the stream-ordered buffers while the stream still exists
  partials.release();
  out.release();
  if (stream) cudaStreamSynchronize(stream);
  if (host) cudaFreeHost(host);
  if (pin) cudaFreeHost(pin);
  if (wait_flag) cudaFreeHost(wait_flag);
  if (tls_stream == stream) tls_stream = nullptr;
  if (stream) cudaStreamDestroy(stream);
}

const double *Workspace::sums(int nblocks, int nred) {
  finalize_sums(red, nblocks, nred, stream);
  sync();
  return host;
}

void Workspace::sync() {
  // the wait flag of the staged kernels rides along with the stream's work
  const bool check = staged_kernels_used();
  if (check) read_wait_flag_async(wait_flag, stream);
  QED_CUDA(cudaStreamSynchronize(stream));
  if (check) check_wait_flag(*wait_flag);
}

double *Workspace::pinned(size_t n) {
  if (n > pin_n) {
    sync();  // the old buffer may still be a copy's destination
    if (pin) cudaFreeHost(pin);
    pin = nullptr;
    pin_n = 0;
    QED_CUDA(cudaMallocHost(&pin, n * sizeof(double)));
    pin_n = n;
  }
  return pin;
}

// ------------------------------------------------------------- SectorOp ------

namespace {

constexpr double kSmall = 1.0e-12;  // SMALL_VALUE (src_util/vector_num.hpp:23)
// Spin tables of at least this many strings also get the packed copy that the
// staged-row H.v kernels read (smaller sectors never take those kernels).
constexpr uint64_t kPackMinDim = 512;

// Host build of a small spin table: the same strings (increasing), ELL entries
// (in the order of k_build_hops, which applies c+_r c_c when bit c is set and
// bit r empty with the parity of the set bits strictly between r and c), bank
// ordering / packing and diagonal (in the summation order of k_diag_half) as the
// device path.
}  // namespace

HostHalf host_half_tables(int L, int N, uint32_t dim, const std::vector<double> &tdiag,
                          const std::vector<double> &vsame, const std::vector<int> &pd, const std::vector<int> &ps,
                          const std::vector<int> &pslot, const std::vector<double> &vals, int width, bool bank_order) {
  HostHalf T;
  std::vector<uint32_t> &hb = T.bits;
  hb.reserve(dim);
  uint64_t sv = N >= 64 ? ~0ull : (1ull << N) - 1ull;
  while (dim) {  // N-subsets of L bits in increasing order (Gosper's successor)
    hb.push_back((uint32_t)sv);
    if (hb.size() == dim) break;
    const uint64_t c = sv & (~sv + 1ull), r = sv + c;
    sv = (((r ^ sv) >> 2) / c) | r;
  }
  std::vector<uint32_t> he((size_t)width * dim, 0u);
  std::vector<uint8_t> hc(dim, 0);
  std::vector<double> &hd = T.diag;
  hd.assign(dim, 0.0);
  for (uint32_t i = 0; i < dim; ++i) {
    const uint32_t b = hb[i];
    int k = 0;
    for (size_t q = 0; q < pd.size(); ++q) {
      const int r = pd[q], c = ps[q];
      if (!((b >> c) & 1u) || ((b >> r) & 1u)) continue;
      const uint32_t nb = b ^ (1u << c) ^ (1u << r);
      const int lo = std::min(r, c), hi = std::max(r, c);
      const uint32_t between = (uint32_t)(((1ull << hi) - 1ull) & ~((2ull << lo) - 1ull));
      const int sgn = __builtin_popcount(nb & between) & 1;
      const uint32_t J = (uint32_t)(std::lower_bound(hb.begin(), hb.end(), nb) - hb.begin());
      if (k < width) he[(size_t)k * dim + i] = (J << 8) | (uint32_t)(pslot[q] + sgn);
      ++k;
    }
    hc[i] = (uint8_t)std::min(k, width);
    double sd = 0.0;
    for (int r = 0; r < L; ++r)
      if ((b >> r) & 1u) {
        sd += tdiag[r];
        for (int c = r; c < L; ++c)
          if ((b >> c) & 1u) sd += vsame[(size_t)r * L + c];
      }
    hd[i] = sd;
  }
  // the bank-ordered copy: packed for the staged kernels, and the ELL itself for the up spin
  T.vals = vals;
  T.width = width;
  const bool want_pack = dim >= kPackMinDim && dim + 8 <= (1u << 14);
  if (width > 0 && (bank_order || want_pack) && dim >= 64 && vals.size() < 256) {
    std::vector<uint32_t> eo(he);
    std::vector<uint8_t> co(hc);
    const int zero_slot = (int)vals.size();
    int w2 = width;
    std::vector<double> vz(vals);
    vz.push_back(0.0);
    if (order_for_banks(eo, co, dim, w2, zero_slot)) {
      T.packed = want_pack && pack_hops16(eo, co, dim, vz, zero_slot, T.ph);
      if (bank_order) {
        T.vals = vz;
        T.width = w2;
        he.swap(eo);
        hc.swap(co);
      }
    }
  }
  T.ell = std::move(he);
  T.cnt = std::move(hc);
  return T;
}

void hop_pairs(int L, const std::vector<double> &t, std::vector<int> &pd, std::vector<int> &ps,
               std::vector<int> &pslot, std::vector<double> &vals) {
  pd.clear();
  ps.clear();
  pslot.clear();
  vals.clear();
  std::map<double, int> slot_of;
  for (int r = 0; r < L; ++r)
    for (int c = 0; c < L; ++c) {
      if (r == c) continue;
      double v = t[(size_t)r * L + c];
      if (std::fabs(v) < kSmall) continue;
      auto it = slot_of.find(v);
      int slot;
      if (it == slot_of.end()) {
        slot = (int)vals.size();
        vals.push_back(v);
        vals.push_back(-v);
        slot_of[v] = slot;
      } else {
        slot = it->second;
      }
      pd.push_back(r);
      ps.push_back(c);
      pslot.push_back(slot);
    }
}

namespace {

// Host build of a small spin table (host_half_tables), uploaded at once.
void build_half_host(HalfTables &h, int L, int N, const std::vector<double> &tdiag,
                     const std::vector<double> &vsame, const std::vector<int> &pd, const std::vector<int> &ps,
                     const std::vector<int> &pslot, const std::vector<double> &vals, int width, Workspace &ws,
                     bool bank_order) {
  HostHalf T = host_half_tables(L, N, h.dim, tdiag, vsame, pd, ps, pslot, vals, width, bank_order);
  h.width = T.width;
  h.nvals = (int)T.vals.size();
  h.bits.upload(T.bits, ws.stream);
  h.cnt.upload(T.cnt, ws.stream);
  h.vals.alloc(std::max<size_t>(T.vals.size(), 1));
  if (!T.vals.empty()) h.vals.upload(T.vals, ws.stream);
  if (T.width > 0) h.ell.upload(T.ell, ws.stream);
  h.diag.upload(T.diag, ws.stream);
  if (T.packed) {
    for (int c = 0; c < 2; ++c) {
      if (T.ph.pk[c].empty()) T.ph.pk[c].assign(4, 0);  // a valid pointer for an empty class
      h.pk[c].upload(T.ph.pk[c], ws.stream);
    }
    h.cntw.upload(T.ph.cnt, ws.stream);
    h.mag[0] = T.ph.mag[0];
    h.mag[1] = T.ph.mag[1];
  }
  h.hbits = std::move(T.bits);
  ws.sync();
}

void build_half(HalfTables &h, int L, int N, const std::vector<double> &t,
                const std::vector<double> &vsame, Workspace &ws, bool bank_order) {
  h.L = L;
  h.N = N;
  uint64_t dim = (N < 0 || N > L) ? 0 : binom(L, N);
  if (dim >= (1ull << 24)) fail(QED_ERR_UNSUPPORTED, "half basis dimension above 2^24");
  h.dim = (uint32_t)dim;
  if (!dim) return;
  // directed hop pairs (dst r, src c) with value slots; value table dedupes |t|
  std::vector<int> pd, ps, pslot;
  std::vector<double> vals;
  hop_pairs(L, t, pd, ps, pslot, vals);
  if (vals.size() > 256) fail(QED_ERR_UNSUPPORTED, "more than 128 distinct hopping amplitudes per spin");
  h.pd = pd;
  h.ps = ps;
  h.pv.resize(pd.size());
  for (size_t q = 0; q < pd.size(); ++q) h.pv[q] = t[(size_t)pd[q] * L + ps[q]];
  int width = std::min<int>((int)pd.size(), N * (L - N));
  if (width > 255) fail(QED_ERR_UNSUPPORTED, "more than 255 hops per basis string");
  std::vector<double> tdiag(L);
  for (int r = 0; r < L; ++r) tdiag[r] = t[(size_t)r * L + r];
  // Spin tables of at most host_table_max_dim strings are built on the host and
  // uploaded once (one stream synchronisation instead of five, no kernel
  // launches): a batch of small clusters builds tens of thousands of them.
  if ((long)dim <= opt_int("host_table_max_dim")) {
    build_half_host(h, L, N, tdiag, vsame, pd, ps, pslot, vals, width, ws, bank_order);
    return;
  }
  h.bits.alloc(dim);
  launch_unrank(L, N, h.dim, h.bits.p, ws.stream);
  h.width = width;
  h.nvals = (int)vals.size();
  h.cnt.alloc(dim);
  h.vals.alloc(std::max<size_t>(vals.size(), 1));
  if (!vals.empty()) h.vals.upload(vals, ws.stream);
  if (width > 0) {
    h.ell.alloc((size_t)width * dim);
    DevBuf<int> dpd(pd.size()), dps(ps.size()), dsl(pslot.size());
    dpd.upload(pd, ws.stream);
    dps.upload(ps, ws.stream);
    dsl.upload(pslot, ws.stream);
    launch_build_hops(L, N, h.dim, h.bits.p, (int)pd.size(), dpd.p, dps.p, dsl.p, h.cnt.p, h.ell.p,
                      width, ws.stream);
    ws.sync();  // the pair arrays are freed on scope exit
    const bool want_pack = dim >= kPackMinDim && dim + 8 <= (1u << 14);
    if ((bank_order || want_pack) && dim >= 64 && vals.size() < 256) {
      std::vector<uint32_t> he((size_t)width * dim);
      std::vector<uint8_t> hc(dim);
      h.ell.download(he.data(), he.size(), ws.stream);
      h.cnt.download(hc.data(), hc.size(), ws.stream);
      ws.sync();
      const int zero_slot = (int)vals.size();
      int w2 = width;
      std::vector<double> vz(vals);
      vz.push_back(0.0);
      if (order_for_banks(he, hc, (uint32_t)dim, w2, zero_slot)) {
        // the staged-row kernels read the packed copy of the ordered table
        PackedHops ph;
        if (want_pack && pack_hops16(he, hc, (uint32_t)dim, vz, zero_slot, ph)) {
          for (int c = 0; c < 2; ++c) {
            if (ph.pk[c].empty()) ph.pk[c].assign(4, 0);  // a valid pointer for an empty class
            h.pk[c].upload(ph.pk[c], ws.stream);
          }
          h.cntw.upload(ph.cnt, ws.stream);
          h.mag[0] = ph.mag[0];
          h.mag[1] = ph.mag[1];
        }
        if (bank_order) {  // the ELL itself is reordered for the up spin only
          vals = vz;
          h.nvals = (int)vals.size();
          h.vals.upload(vals, ws.stream);
          h.width = w2;
          h.ell.alloc((size_t)w2 * dim);
          h.ell.upload(he, ws.stream);
          h.cnt.upload(hc, ws.stream);
        }
        ws.sync();
      }
    }
  } else {
    QED_CUDA(cudaMemsetAsync(h.cnt.p, 0, dim, ws.stream));
  }
  DevBuf<double> dt(L), dv(vsame.size());
  dt.upload(tdiag, ws.stream);
  dv.upload(vsame, ws.stream);
  h.diag.alloc(dim);
  launch_diag_half(L, h.dim, h.bits.p, dt.p, dv.p, h.diag.p, ws.stream);
  h.hbits.resize(dim);
  h.bits.download(h.hbits.data(), dim, ws.stream);
  ws.sync();
}

SpinTable view(const HalfTables &h) {
  SpinTable s;
  s.bits = h.bits.p;
  s.cnt = h.cnt.p;
  s.ell = h.ell.p;
  s.vals = h.vals.p;
  s.diag = h.diag.p;
  s.dim = h.dim;
  s.nvals = h.nvals;
  if (h.cntw.n) {
    for (int c = 0; c < 2; ++c) {
      s.pk[c] = reinterpret_cast<const uint2 *>(h.pk[c].p);
      s.mag[c] = h.mag[c];
    }
    s.cntw = h.cntw.p;
  }
  return s;
}

}  // namespace

SectorOp::SectorOp(const SpinData &t, const Sector &s, Workspace &ws, HalfCache *cache) : sec(s), L(t.n) {
  PhaseScope ps(kPhSectorSetup);
  if (s.N >= Sector::odd || s.S >= Sector::odd)
    fail(QED_ERR_UNSUPPORTED, "sector " + s.name() + " does not conserve N and S");
  if ((s.N + s.S) % 2) fail(QED_ERR_ARGUMENT, "sector " + s.name() + " is not valid");
  if (L > 32) fail(QED_ERR_UNSUPPORTED, "more than 32 orbitals per spin");
  auto table = [&](int spin, int N) -> std::shared_ptr<const HalfTables> {
    auto make = [&] {
      auto h = std::make_shared<HalfTables>();
      build_half(*h, L, N, spin ? t.t_dn : t.t_up, spin ? t.v_dd : t.v_uu, ws, spin == 0);
      return std::shared_ptr<const HalfTables>(h);
    };
    if (!cache) return make();
    std::lock_guard<std::mutex> l(cache->m);
    auto &slot = cache->tab[{spin, N}];
    if (!slot) slot = make();  // built on this thread's stream and synchronised
    return slot;
  };
  up = table(0, s.Nup());
  dn = table(1, s.Ndw());
  D = (size_t)up->dim * dn->dim;
  // inter-spin density-density terms
  const int n = L;
  bool any = false, offdiag = false;
  for (int r = 0; r < n; ++r)
    for (int c = 0; c < n; ++c)
      if (t.v_du[(size_t)r * n + c] != 0.0) {
        any = true;
        if (r != c) offdiag = true;
      }
  op.inter.n = n;
  if (!any) {
    op.inter.mode = 0;
  } else if (!offdiag) {
    double u0 = t.v_du[0];
    bool uniform = true;
    for (int r = 0; r < n; ++r)
      if (t.v_du[(size_t)r * n + r] != u0) uniform = false;
    if (uniform) {
      op.inter.mode = 1;
      op.inter.u = u0;
    } else {
      std::vector<double> dg(n);
      for (int r = 0; r < n; ++r) dg[r] = t.v_du[(size_t)r * n + r];
      vinter.upload(dg, ws.stream);
      op.inter.mode = 2;
      op.inter.v = vinter.p;
    }
  } else {
    vinter.upload(t.v_du, ws.stream);
    op.inter.mode = 3;
    op.inter.v = vinter.p;
  }
  op.up = view(*up);
  op.dn = view(*dn);
  int dev = 0;
  QED_CUDA(cudaGetDevice(&dev));
  QED_CUDA(cudaDeviceGetAttribute(&op.num_sms, cudaDevAttrMultiProcessorCount, dev));
  bind_windows();
  ws.sync();
}

void SectorOp::bind_windows() {
  if (!opt_bool("hv_windows") || D < (size_t)opt_int("hv_windows_min_dim") || up->pd.empty() || dn->pd.empty())
    return;
  WindowPlan pu, pdn;
  if (!plan_windows(up->L, up->N, up->hbits, up->pd, up->ps, pu) ||
      !plan_windows(dn->L, dn->N, dn->hbits, dn->pd, dn->ps, pdn))
    return;
  std::string why;
  std::shared_ptr<const WinModule> mod;
  try {
    mod = window_module(pu, pdn, &why);
  } catch (const Error &) {
    (void)cudaGetLastError();  // clear the failed call's error for the next launch check
    mod = nullptr;             // the module did not load: the staged kernels take the sector
  }
  if (!mod) return;  // the staged kernels take the sector
  win = std::make_shared<WinBinding>();
  win->mod = mod;
  win->amp_up = up->pv;
  win->amp_dn = dn->pv;
  op.win = win.get();
}

KrylovOp::KrylovOp(const MixedHamiltonian &h) : D(h.D), mixed(&h) {}

int KrylovOp::apply(const double *x, double xs, double *y, const SubList &sub, int red_mask, Reducer &r,
                    cudaStream_t s, const int *skip) const {
  if (mixed) return mixed->apply_full(x, xs, y, sub, red_mask, r, s, skip);
  HvOperator op = fact->op;
  op.skip = skip;
  return launch_hv(op, x, xs, y, sub, red_mask, r, s);
}

void KrylovOp::apply_block(int p, const BlockIn &X, const BlockOut &Y, Reducer &r, cudaStream_t s) const {
  if (fact) {
    launch_block_hv(fact->op, p, X, Y, r, s);
    return;
  }
  SubList none;
  for (int c = 0; c < p; ++c) mixed->apply_full(X.v[c], 1.0, Y.v[c], none, 0, r, s);
}

void SectorOp::apply(const double *x, double *y, Workspace &ws) const {
  if (!D) return;
  SubList none;
  launch_hv(op, x, 1.0, y, none, 0, ws.red, ws.stream);
}

// ------------------------------------------------------ Lanczos (ground state) --

namespace {
// Random start vector, normalised (Hamiltonian::states -> random(),
// src_util/vector_num.cpp:114-119); deterministic in `seed`. Small sectors take
// it from the per-sector start kernel of the batched eigenvalue pass, so that
// the eigenvector pass replays the same v_0.
void start_vector(size_t D, uint64_t seed, double *v, Workspace &ws) {
  if (D <= lanczos_job_max_dim()) {
    DevBuf<double> prev(D), bp(1);
    LanczosJob J;
    J.op.up.dim = (uint32_t)D;
    J.op.dn.dim = 1;
    J.v[0] = prev.p;
    J.v[1] = v;
    J.v[2] = prev.p;
    J.beta_prev = bp.p;
    J.out = nullptr;
    J.seed = seed;
    J.nsteps = 0;
    J.rot = 0;
    DevBuf<LanczosJob> dj(1);
    dj.upload(&J, 1, ws.stream);
    launch_lanczos_start_jobs(dj.p, 1, ws.stream);
    ws.sync();
    return;
  }
  const int nb = launch_random(D, seed, v, ws.red, ws.stream);
  const double n2 = ws.sums(nb, 1)[0];
  launch_scale(D, v, 1.0 / std::sqrt(n2), ws.stream);
}
}  // namespace

// The Ritz test of LanczosEigenvalue (src_ed/Hamiltonian/Lanczos.hpp:73-90)
// needs the lowest eigenvalue of the j x j tridiagonal and the last component
// of its eigenvector at every step. Far from convergence both come from O(j)
// updates (inverse iteration from the previous step's eigenvector, certified by
// an LDL^T inertia count, or Sturm bisection + backward recurrence), accurate
// to about 1e-12 relative where the lowest eigenvalue is separated. Only when
// that estimate lands within 0.1 % of the tolerance does the O(j^2) QL
// last-row method (the reference's dstev result) decide the stop, so that the
// iteration count does not hinge on the fast estimate's last digits.
//
// The recurrence itself runs on the device in chunks: alpha_j, beta_j stay in
// device memory (the row pass reads beta_{j-1} from there), and the host reads
// a whole chunk of (alpha, beta) once, then applies the Ritz test step by step
// in the reference's order. Steps computed past the stopping step are dropped,
// so the tridiagonal, the energy and the iteration count are those of the
// one-step-at-a-time recurrence.
// The fast estimate agrees with the QL value to about 1 % near the tolerance
// (O(j) inverse iteration converged to a residual of 1e-14 ||T||), so a gate of
// 8x leaves a wide margin while the O(j^2) QL runs only on the last steps.
constexpr double kQlBand = 1e-3;

namespace {
// constructed on first use: the library installs the hook from another
// translation unit's static initialiser, which may run before this one's
ParallelFor &parallel_for_hook() {
  static ParallelFor f;
  return f;
}
}  // namespace

void set_parallel_for(ParallelFor f) { parallel_for_hook() = std::move(f); }

size_t lanczos_job_max_dim() {
  const long v = opt_int("lanczos_job_max_dim");
  return (size_t)std::max<long>(0, std::min<long>(v, (long)kLanczosCtaMaxDimCap));
}

void lanczos_energy_batch(std::vector<LanczosBatchItem> &items, Workspace &ws) {
  PhaseScope ps(kPhGsLanczos);
  const int n = (int)items.size();
  if (!n) return;
  PhaseScope ps_batch(n > 1 ? kPhGsBatch : kPhGsLanczos);
  const double accur = opt_double("accur_lanczos");
  const long max_iter = opt_int("max_iter_lanczos");
  cudaStream_t s = ws.stream;
  constexpr int kChunk = kLanczosJobMaxSteps;
  // one arena for the three vectors of every sector (32-byte aligned blocks)
  std::vector<size_t> off(n);
  size_t tot = 0;
  for (int i = 0; i < n; ++i) {
    if (items[i].H->D > lanczos_job_max_dim()) fail(QED_ERR_INTERNAL, "lanczos_energy_batch: sector too large");
    off[i] = tot;
    tot += 3 * ((items[i].H->D + 3) / 4 * 4);
  }
  DevBuf<double> arena(std::max<size_t>(tot, 1)), bprev(n), out((size_t)n * 2 * kChunk);
  DevBuf<LanczosJob> djobs(n);
  std::vector<LanczosJob> jobs(n);
  struct Run {
    RitzTracker tracker;
    double lambda0 = 0.0;
    int rot = 0, chunk = 0;
  };
  std::vector<Run> run(n);
  for (int i = 0; i < n; ++i) {
    const size_t D = items[i].H->D;
    const size_t Dp = (D + 3) / 4 * 4;
    LanczosJob &J = jobs[i];
    J.op = items[i].H->op;
    for (int r = 0; r < 3; ++r) J.v[r] = arena.p + off[i] + r * Dp;
    J.beta_prev = bprev.p + i;
    J.out = out.p + (size_t)i * 2 * kChunk;
    J.seed = items[i].seed;
    J.nsteps = 0;
    J.rot = 0;
    *items[i].out = LanczosResult();
    // a first short chunk: tiny sectors stop after about D steps
    run[i].chunk = (int)std::min<size_t>(std::max<size_t>(D, 2), 8);
  }
  djobs.upload(jobs.data(), n, s);
  launch_lanczos_start_jobs(djobs.p, n, s);
  // largest sectors first: CTAs start in table order, so the longest jobs of a
  // chunk do not wait behind the short ones (each job's arithmetic does not
  // depend on its place in the table)
  std::vector<int> active(n);
  for (int i = 0; i < n; ++i) active[i] = i;
  std::stable_sort(active.begin(), active.end(), [&](int a, int b) { return items[a].H->D > items[b].H->D; });
  std::vector<LanczosJob> batch;
  std::vector<double> hout;
  while (!active.empty()) {
    const int na = (int)active.size();
    batch.resize(na);
    for (int a = 0; a < na; ++a) {
      const int i = active[a];
      batch[a] = jobs[i];
      batch[a].nsteps = run[i].chunk;
      batch[a].rot = run[i].rot;
      batch[a].out = out.p + (size_t)a * 2 * kChunk;
    }
    djobs.upload(batch.data(), na, s);
    launch_lanczos_jobs(djobs.p, na, s);
    hout.resize((size_t)na * 2 * kChunk);
    out.download(hout.data(), hout.size(), s);
    ws.sync();
    PhaseScope ps_ritz(kPhRitz);
    std::vector<char> done(na, 0);
    std::vector<std::string> err(na);
    std::vector<int> code(na, 0);
    auto test = [&](int a) {  // the Ritz tests of one sector's chunk, in step order
      const int i = active[a];
      Run &R = run[i];
      LanczosResult &res = *items[i].out;
      const double *ha = hout.data() + (size_t)a * 2 * kChunk, *hb = ha + kChunk;
      bool stop = false;
      try {
        for (int k = 0; k < R.chunk && !stop; ++k) {
          res.alpha.push_back(ha[k]);
          res.beta.push_back(hb[k]);
          double last = 1.0;
          tridiag_lowest_track((int)res.alpha.size(), res.alpha.data(), res.beta.data(), R.tracker, &R.lambda0,
                               &last);
          double ritz = std::fabs(last * hb[k]);
          if (std::fabs(ritz - accur) < kQlBand * accur) {
            if (!tridiag_lowest_last((int)res.alpha.size(), res.alpha.data(), res.beta.data(), &R.lambda0, &last))
              fail(QED_ERR_LANCZOS, "tridiagonal eigensolver did not converge" + items[i].where);
            ritz = std::fabs(last * hb[k]);
          }
          if ((long)res.alpha.size() > max_iter)
            fail(QED_ERR_LANCZOS, "Lanczos procedure exceeded " + std::to_string(max_iter) + " iterations" +
                                      items[i].where);
          if (!(ritz > accur)) stop = true;
        }
      } catch (const Error &e) {
        code[a] = e.code;
        err[a] = e.what();
        return;
      } catch (const std::exception &e) {  // nothing may escape into a pool thread
        code[a] = QED_ERR_INTERNAL;
        err[a] = e.what();
        return;
      }
      R.rot = (R.rot + R.chunk) % 3;
      R.chunk = kChunk;
      if (stop) {
        res.energy = R.lambda0;
        res.iterations = (int)res.alpha.size();
        done[a] = 1;
      }
    };
    const ParallelFor &pf = parallel_for_hook();
    if (pf && na > 1)
      pf(na, test);
    else
      for (int a = 0; a < na; ++a) test(a);
    std::vector<int> still;
    for (int a = 0; a < na; ++a) {
      if (code[a]) fail(code[a], err[a]);
      if (!done[a]) still.push_back(active[a]);
    }
    active.swap(still);
  }
}

// CUDA graphs of one launch sequence per key (here: the Krylov buffers' rotation
// at the start of a chunk). run() captures the sequence on its first use for a
// key (the captured launches are then replayed once, so the stream does the work
// exactly once either way) and replays the instantiated graph afterwards;
// captured_now tells the caller which happened. Graphs are released with the
// object.
struct ChunkGraphs {
  cudaGraphExec_t exec[3] = {nullptr, nullptr, nullptr};
  bool captured_now = false;
  ChunkGraphs() = default;
  ChunkGraphs(const ChunkGraphs &) = delete;
  ChunkGraphs &operator=(const ChunkGraphs &) = delete;
  ~ChunkGraphs() {
    for (auto &e : exec)
      if (e) cudaGraphExecDestroy(e);
  }
  template <class F> void run(int key, cudaStream_t s, F &&record) {
    captured_now = false;
    if (!exec[key]) {
      cudaGraph_t g = nullptr;
      QED_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      try {
        record();
      } catch (...) {
        cudaStreamEndCapture(s, &g);
        if (g) cudaGraphDestroy(g);
        throw;
      }
      QED_CUDA(cudaStreamEndCapture(s, &g));
      const cudaError_t e = cudaGraphInstantiate(&exec[key], g, 0);
      cudaGraphDestroy(g);
      QED_CUDA(e);
      captured_now = true;
    }
    QED_CUDA(cudaGraphLaunch(exec[key], s));
  }
};

LanczosResult lanczos_energy(const SectorOp &H, Workspace &ws, uint64_t seed) {
  if (H.D <= lanczos_job_max_dim()) {
    LanczosResult res;
    std::vector<LanczosBatchItem> one(1);
    one[0].H = &H;
    one[0].seed = seed;
    one[0].out = &res;
    lanczos_energy_batch(one, ws);
    return res;
  }
  PhaseScope ps(kPhGsLanczos);
  LanczosResult res;
  const size_t D = H.D;
  const double accur = opt_double("accur_lanczos");
  const long max_iter = opt_int("max_iter_lanczos");
  cudaStream_t s = ws.stream;
  constexpr int kChunk = 16;
  static_assert(2 * kChunk <= Reducer::kMaxRed, "chunk read back through the pinned reduction buffer");
  DevBuf<double> A(D), B(D), C(D);
  start_vector(D, seed, B.p, ws);
  QED_CUDA(cudaMemsetAsync(A.p, 0, D * sizeof(double), s));  // v_{-1} = 0
  const size_t cap = (size_t)std::max<long>(max_iter, 1) + 2 * kChunk;
  DevBuf<double> sc(3 + 2 * cap);
  DevBuf<int> jd(1);
  QED_CUDA(cudaMemsetAsync(sc.p, 0, 3 * sizeof(double), s));
  QED_CUDA(cudaMemsetAsync(jd.p, 0, sizeof(int), s));
  LanczosScalars ls;
  ls.alpha_cur = sc.p;
  ls.b2_cur = sc.p + 1;
  ls.beta_prev = sc.p + 2;
  ls.alpha_hist = sc.p + 3;
  ls.beta_hist = sc.p + 3 + cap;
  ls.j = jd.p;
  SubList sub;  // w = H v_j - beta_{j-1} v_{j-1}, beta from device memory
  sub.n = 1;
  sub.cdev = ls.beta_prev;
  double *pa = A.p, *pb = B.p, *pc = C.p;
  std::vector<double> &alpha = res.alpha, &beta = res.beta;
  double lambda0 = 0.0;
  RitzTracker tracker;
  size_t launched = 0;
  // One Lanczos step on the current buffers, then the rotation
  // v_{j-1} <- v_j <- v_{j+1}. Every scalar lives in device memory (ls), so a
  // chunk of steps is the same launch sequence whatever the step index: after
  // the first chunk, the full chunks are replayed from CUDA graphs, one per
  // rotation of (pa, pb, pc) at the chunk's start (kChunk = 16 steps shift the
  // rotation by one).
  auto one_step = [&] {
    sub.z[0] = pa;
    int nb = launch_hv(H.op, pb, 1.0, pc, sub, 1, ws.red, s);
    launch_finalize(ws.red.partials, nb, 1, ls.alpha_cur, s);      // alpha_j = <v_j, w>
    nb = launch_axpy_dev(D, pc, pb, ls.alpha_cur, ws.red, s);      // w -= alpha_j v_j
    launch_finalize(ws.red.partials, nb, 1, ls.b2_cur, s);          // |w|^2
    launch_lanczos_advance(D, pc, ls, s);                           // v_{j+1} = w / beta_j
    double *t = pa;
    pa = pb;
    pb = pc;
    pc = t;
  };
  ChunkGraphs graphs;
  const bool use_graphs = opt_bool("lanczos_graphs") && (long)D >= opt_int("lanczos_graphs_min_dim");
  int rot = 0;  // rotations of (pa, pb, pc) since the start, mod 3
  // a first short chunk: tiny sectors stop after about D steps
  int chunk = (int)std::min<size_t>(std::max<size_t>(D, 2), 8);
  bool stop = false;
  while (!stop) {
    if (launched + chunk > cap) fail(QED_ERR_INTERNAL, "Lanczos history overflow");
    if (use_graphs && chunk == kChunk && launched > 0) {
      graphs.run(rot, s, [&] {
        for (int k = 0; k < kChunk; ++k) one_step();
      });
      if (!graphs.captured_now) {  // replayed: advance the host's view of the rotation
        for (int k = 0; k < kChunk; ++k) {
          double *t = pa;
          pa = pb;
          pb = pc;
          pc = t;
        }
      }
    } else {
      for (int k = 0; k < chunk; ++k) one_step();
    }
    rot = (rot + chunk) % 3;
    QED_CUDA(cudaMemcpyAsync(ws.host, ls.alpha_hist + launched, chunk * sizeof(double),
                             cudaMemcpyDeviceToHost, s));
    QED_CUDA(cudaMemcpyAsync(ws.host + kChunk, ls.beta_hist + launched, chunk * sizeof(double),
                             cudaMemcpyDeviceToHost, s));
    ws.sync();
    launched += chunk;
    PhaseScope ps_ritz(kPhRitz);
    for (int k = 0; k < chunk && !stop; ++k) {
      const double a = ws.host[k], b = ws.host[kChunk + k];
      alpha.push_back(a);
      beta.push_back(b);
      double last = 1.0;
      tridiag_lowest_track((int)alpha.size(), alpha.data(), beta.data(), tracker, &lambda0, &last);
      double ritz = std::fabs(last * b);
      if (std::fabs(ritz - accur) < kQlBand * accur) {
        if (!tridiag_lowest_last((int)alpha.size(), alpha.data(), beta.data(), &lambda0, &last))
          fail(QED_ERR_LANCZOS, "tridiagonal eigensolver did not converge");
        ritz = std::fabs(last * b);
      }
      if ((long)alpha.size() > max_iter)
        fail(QED_ERR_LANCZOS, "Lanczos procedure exceeded " + std::to_string(max_iter) + " iterations");
      if (!(ritz > accur)) stop = true;
    }
    chunk = kChunk;
  }
  res.energy = lambda0;
  res.iterations = (int)alpha.size();
  return res;
}

// LanczosEigenvector (src_ed/Hamiltonian/Lanczos.hpp:109-143): psi = sum_j Z_j0 v_j
// with the v_j regenerated from the same start vector and the stored alpha/beta.
void lanczos_eigenvector(const SectorOp &H, Workspace &ws, const LanczosResult &res,
                         uint64_t seed, DevBuf<double> &psi) {
  PhaseScope ps(kPhGsVector);
  const size_t D = H.D;
  cudaStream_t s = ws.stream;
  const std::vector<double> &alpha = res.alpha, &beta = res.beta;
  const int M = (int)alpha.size();
  std::vector<double> d(alpha), e(beta), Z;
  e.resize(M > 0 ? M - 1 : 0);
  if (!tridiag_eig(M, d, e, &Z)) fail(QED_ERR_LANCZOS, "tridiagonal eigensolver did not converge");
  psi.alloc(D);
  DevBuf<double> A(D), B(D), C(D);
  start_vector(D, seed, B.p, ws);
  launch_axpby(D, 0.0, psi.p, Z[0], B.p, 0, ws.red, s);
  double *pa = A.p, *pb = B.p, *pc = C.p;
  for (int j = 1; j < M; ++j) {
    SubList sub;
    sub.n = 1;
    sub.c[0] = alpha[j - 1];
    sub.z[0] = pb;
    if (j >= 2) {
      sub.n = 2;
      sub.c[1] = beta[j - 2];
      sub.z[1] = pa;
    }
    launch_hv(H.op, pb, 1.0, pc, sub, 0, ws.red, s);
    launch_scale(D, pc, 1.0 / beta[j - 1], s);
    launch_axpby(D, 1.0, psi.p, Z[j], pc, 0, ws.red, s);
    std::swap(pa, pb);
    std::swap(pb, pc);
  }
  ws.sync();
}

LanczosResult lanczos_ground_state(const SectorOp &H, Workspace &ws, DevBuf<double> &psi,
                                   uint64_t seed) {
  LanczosResult res = lanczos_energy(H, ws, seed);
  lanczos_eigenvector(H, ws, res, seed, psi);
  return res;
}

// Ground-state energy of one sector in the symmetry-adapted basis: the recurrence,
// chunking and Ritz-residual stop of lanczos_energy, with the mixed-basis CSR
// product (w = H v_j - beta_{j-1} v_{j-1} and the <v_j, w> partials in one kernel).
LanczosResult lanczos_energy_mixed(const MixedHamiltonian &H, Workspace &ws, uint64_t seed) {
  PhaseScope ps(kPhGsLanczos);
  LanczosResult res;
  const size_t D = H.D;
  if (D == 0) fail(QED_ERR_ARGUMENT, "empty sector");
  const double accur = opt_double("accur_lanczos");
  const long max_iter = opt_int("max_iter_lanczos");
  cudaStream_t s = ws.stream;
  constexpr int kChunk = 16;
  DevBuf<double> A(D), B(D), C(D);
  start_vector(D, seed, B.p, ws);
  QED_CUDA(cudaMemsetAsync(A.p, 0, D * sizeof(double), s));
  const size_t cap = (size_t)std::max<long>(max_iter, 1) + 2 * kChunk;
  DevBuf<double> sc(3 + 2 * cap);
  DevBuf<int> jd(1);
  QED_CUDA(cudaMemsetAsync(sc.p, 0, 3 * sizeof(double), s));
  QED_CUDA(cudaMemsetAsync(jd.p, 0, sizeof(int), s));
  LanczosScalars ls;
  ls.alpha_cur = sc.p;
  ls.b2_cur = sc.p + 1;
  ls.beta_prev = sc.p + 2;
  ls.alpha_hist = sc.p + 3;
  ls.beta_hist = sc.p + 3 + cap;
  ls.j = jd.p;
  double *pa = A.p, *pb = B.p, *pc = C.p;
  std::vector<double> &alpha = res.alpha, &beta = res.beta;
  double lambda0 = 0.0;
  RitzTracker tracker;
  size_t launched = 0;
  int chunk = (int)std::min<size_t>(std::max<size_t>(D, 2), 8);
  bool stop = false;
  while (!stop) {
    if (launched + chunk > cap) fail(QED_ERR_INTERNAL, "Lanczos history overflow");
    for (int k = 0; k < chunk; ++k) {
      int nb = H.lanczos_w(pb, pa, ls.beta_prev, pc, ws.red.partials, Reducer::kMaxRed, ws.red.max_blocks, s);
      launch_finalize(ws.red.partials, nb, 1, ls.alpha_cur, s);  // alpha_j = <v_j, w>
      nb = launch_axpy_dev(D, pc, pb, ls.alpha_cur, ws.red, s);  // w -= alpha_j v_j
      launch_finalize(ws.red.partials, nb, 1, ls.b2_cur, s);      // |w|^2
      launch_lanczos_advance(D, pc, ls, s);                       // v_{j+1} = w / beta_j
      double *t = pa;
      pa = pb;
      pb = pc;
      pc = t;
    }
    QED_CUDA(cudaMemcpyAsync(ws.host, ls.alpha_hist + launched, chunk * sizeof(double), cudaMemcpyDeviceToHost, s));
    QED_CUDA(cudaMemcpyAsync(ws.host + kChunk, ls.beta_hist + launched, chunk * sizeof(double),
                             cudaMemcpyDeviceToHost, s));
    ws.sync();
    launched += chunk;
    for (int k = 0; k < chunk && !stop; ++k) {
      const double a = ws.host[k], b = ws.host[kChunk + k];
      alpha.push_back(a);
      beta.push_back(b);
      double last = 1.0;
      tridiag_lowest_track((int)alpha.size(), alpha.data(), beta.data(), tracker, &lambda0, &last);
      double ritz = std::fabs(last * b);
      if (std::fabs(ritz - accur) < kQlBand * accur) {
        if (!tridiag_lowest_last((int)alpha.size(), alpha.data(), beta.data(), &lambda0, &last))
          fail(QED_ERR_LANCZOS, "tridiagonal eigensolver did not converge");
        ritz = std::fabs(last * b);
      }
      if ((long)alpha.size() > max_iter)
        fail(QED_ERR_LANCZOS, "Lanczos procedure exceeded " + std::to_string(max_iter) + " iterations");
      if (!(ritz > accur)) stop = true;
    }
    chunk = kChunk;
  }
  res.energy = lambda0;
  res.iterations = (int)alpha.size();
  return res;
}

// The ground-state vector of a mixed-basis sector: the replay of
// lanczos_eigenvector (LanczosEigenvector, src_ed/Hamiltonian/Lanczos.hpp:109-143)
// with the CSR product.
void lanczos_eigenvector_mixed(const MixedHamiltonian &H, Workspace &ws, const LanczosResult &res, uint64_t seed,
                               DevBuf<double> &psi) {
  PhaseScope ps(kPhGsVector);
  const size_t D = H.D;
  cudaStream_t s = ws.stream;
  const std::vector<double> &alpha = res.alpha, &beta = res.beta;
  // The replay divides by beta_{j-1} for j < M. The energy recurrence stops at
  // the first step whose beta vanishes (its Ritz residual is then 0), so only the
  // last beta can be zero; cut the replay at the first beta that is not
  // positive anyway (an exhausted Krylov space of a 1- or 2-state irrep).
  int M = (int)alpha.size();
  for (int j = 1; j < M; ++j)
    if (!(beta[j - 1] > 0.0)) {
      M = j;
      break;
    }
  std::vector<double> d(alpha.begin(), alpha.begin() + M), e(beta), Z;
  e.resize(M > 0 ? M - 1 : 0);
  if (!tridiag_eig(M, d, e, &Z)) fail(QED_ERR_LANCZOS, "tridiagonal eigensolver did not converge");
  psi.alloc(D);
  DevBuf<double> A(D), B(D), C(D);
  start_vector(D, seed, B.p, ws);
  launch_axpby(D, 0.0, psi.p, Z[0], B.p, 0, ws.red, s);
  double *pa = A.p, *pb = B.p, *pc = C.p;
  for (int j = 1; j < M; ++j) {
    H.apply(pb, pc, s);                                         // H v_{j-1}
    launch_axpby(D, 1.0, pc, -alpha[j - 1], pb, 0, ws.red, s);  // - alpha_{j-1} v_{j-1}
    if (j >= 2) launch_axpby(D, 1.0, pc, -beta[j - 2], pa, 0, ws.red, s);  // - beta_{j-2} v_{j-2}
    launch_scale(D, pc, 1.0 / beta[j - 1], s);
    launch_axpby(D, 1.0, psi.p, Z[j], pc, 0, ws.red, s);
    std::swap(pa, pb);
    std::swap(pb, pc);
  }
  ws.sync();
}

// ------------------------------------------------------ full diagonalisation --

void dense_eigensystem(const SectorOp &H, Workspace &ws, std::vector<double> &w,
                       std::vector<double> &U) {
  PhaseScope ps(kPhDense);
  const size_t D = H.D;
  DevBuf<double> h(D * D);
  launch_dense_hamiltonian(H.op, h.p, ws.stream);
  std::vector<double> A(D * D);
  h.download(A.data(), D * D, ws.stream);
  ws.sync();
  if (!sym_eig((int)D, A, w, &U)) fail(QED_ERR_INTERNAL, "dense eigensolver did not converge");
}

// ------------------------------------------------------------ LanczosGreen --

void lanczos_green(const KrylovOp &H, Workspace &ws, double *psi, double *q,
                   std::vector<double> &a, std::vector<double> &b) {
  const size_t D = H.D;
  const double accur = opt_double("accur_continued_fraction");
  const size_t max_iter = (size_t)opt_int("max_iter_CF");
  cudaStream_t s = ws.stream;
  a.clear();
  b.assign(1, 1.0);
  QED_CUDA(cudaMemsetAsync(q, 0, D * sizeof(double), s));
  double prod = 1.0;
  while (prod > accur && std::fabs(b.back()) > accur && a.size() < max_iter) {
    if (!a.empty()) launch_swap_scale(D, q, psi, b.back(), s);
    SubList sub;  // q <- H psi + q  (row pass subtracts -1 * q in place)
    sub.n = 1;
    sub.c[0] = -1.0;
    sub.z[0] = q;
    int nb = H.apply(psi, 1.0, q, sub, 1, ws.red, s);
    const double z = ws.sums(nb, 1)[0];
    a.push_back(z);
    nb = launch_axpby(D, 1.0, q, -z, psi, 1, ws.red, s);
    const double zz = std::sqrt(ws.sums(nb, 1)[0]);
    b.push_back(zz);
    prod *= std::fabs(zz);
  }
}

// ------------------------------------------------------------ band Lanczos --

namespace {

// Pool of device vectors of one length, recycled by slot index.
struct VecPool {
  size_t D;
  std::vector<DevBuf<double>> bufs;
  std::vector<int> free_list;
  explicit VecPool(size_t d) : D(d) {}
  int get() {
    if (!free_list.empty()) {
      int k = free_list.back();
      free_list.pop_back();
      return k;
    }
    bufs.emplace_back(D);
    return (int)bufs.size() - 1;
  }
  void put(int k) {
    if (k >= 0) free_list.push_back(k);
  }
  double *p(int k) { return bufs[k].p; }
};

}  // namespace

namespace {

// Upper-triangular R with G = R^T R (G p x p row-major symmetric); false if a
// pivot is not positive. Rinv receives R^{-1} (upper triangular, row-major).
bool cholesky_upper(int p, const double *G, std::vector<double> &R, std::vector<double> &Rinv) {
  R.assign((size_t)p * p, 0.0);
  for (int i = 0; i < p; ++i) {
    double d = G[i * p + i];
    for (int k = 0; k < i; ++k) d -= R[k * p + i] * R[k * p + i];
    if (!(d > 0.0)) return false;
    const double rii = std::sqrt(d);
    R[i * p + i] = rii;
    for (int j = i + 1; j < p; ++j) {
      double t = G[i * p + j];
      for (int k = 0; k < i; ++k) t -= R[k * p + i] * R[k * p + j];
      R[i * p + j] = t / rii;
    }
  }
  Rinv.assign((size_t)p * p, 0.0);
  for (int i = p - 1; i >= 0; --i) {  // back substitution, row by row from the bottom
    Rinv[i * p + i] = 1.0 / R[i * p + i];
    for (int j = i + 1; j < p; ++j) {
      double t = 0.0;
      for (int k = i + 1; k <= j; ++k) t += R[i * p + k] * Rinv[k * p + j];
      Rinv[i * p + j] = -t / R[i * p + i];
    }
  }
  return true;
}

// Block form of the band-Lanczos recurrence for large sectors: V_0 = QR(phi),
// W = H V_k - V_{k-1} B_k^T, A_k = V_k^T W, W -= V_k A_k, W = V_{k+1} B_{k+1}
// (Cholesky QR, twice). Without deflation band Lanczos builds, in exact
// arithmetic, the same Krylov space one vector at a time (the candidates of its
// window are H v orthogonalised against the band), and its projected matrix is
// this block tridiagonal T with upper-triangular B blocks, i.e. banded with
// half-bandwidth p. Its dimension only stops at multiples of p (the convergence
// test runs at j % p == 0, and M0 is a multiple of p), so the stopping rule is
// the same. Returns false, leaving phi intact, when a QR pivot falls below 1e-4
// (a deflation the band algorithm must handle), for p > 16 and for p = 1; the
// caller then runs the band recurrence.
bool block_lanczos_qmatrix(const KrylovOp &H, Workspace &ws, std::vector<DevBuf<double>> &phi,
                           std::vector<double> &evals, std::vector<double> &Q, int &Mout) {
  const size_t D = H.D;
  const int p = (int)phi.size();
  if (p < 2 || p > 16) return false;  // one start vector: nothing to amortise
  cudaStream_t s = ws.stream;
  int M0 = (int)(14 * p * std::log(1.0 * D));
  if (!(M0 > 1)) fail(QED_ERR_INTERNAL, "Assertion failed: M>1 in build_Q_matrix");
  double accur_bl = opt_double("accur_band_lanczos");
  if (accur_bl < 0.0) accur_bl = 0.0;
  const long max_iter_BL = opt_int("max_iter_BL");
  const double min_gap = opt_double("band_lanczos_minimum_gap");
  const bool no_degenerate = opt_bool("no_degenerate_BL");
  if (M0 > max_iter_BL) M0 = (int)max_iter_BL;
  M0 = (M0 / p + 1) * p - p;  // bandLanczos: M0p - pc with pc = p
  if (M0 < p) return false;
  constexpr double kPivotMin = 1e-4;
  const int pp = p * p;
  const int max_blocks = 4096;
  DevBuf<double> part((size_t)max_blocks * pp), dsmall(2 * (size_t)pp);
  double *dG = dsmall.p, *dM = dsmall.p + pp;
  std::vector<double> hG(pp), R1, R1i, R2, R2i;
  auto gram_to_host = [&](int nb) {
    launch_finalize_ld(part.p, nb, pp, pp, dG, s);
    QED_CUDA(cudaMemcpyAsync(hG.data(), dG, pp * sizeof(double), cudaMemcpyDeviceToHost, s));
    ws.sync();
  };
  auto upload = [&](double *dst, const std::vector<double> &h) {
    QED_CUDA(cudaMemcpyAsync(dst, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  };
  // Blocks are p separate vectors (column-major D x p buffers, or the start
  // vectors themselves); their H.v is p single-vector H.v launches.
  const BlockIn none;
  auto block = [&](double *base) {
    BlockOut o;
    for (int c = 0; c < p; ++c) o.v[c] = base + (size_t)c * D;
    return o;
  };
  auto in = [&](const BlockOut &o) {
    BlockIn i;
    for (int c = 0; c < p; ++c) i.v[c] = o.v[c];
    return i;
  };
  // Cholesky QR, twice: X (its gram already in hG) -> tmp -> out; B = R2 R1
  auto cholqr2 = [&](const BlockIn &X, const BlockOut &tmp, const BlockOut &out, std::vector<double> &B) {
    if (!cholesky_upper(p, hG.data(), R1, R1i)) return false;
    for (int i = 0; i < p; ++i)
      if (R1[i * p + i] < kPivotMin) return false;
    upload(dM, R1i);
    int nb = launch_bl_update(D, p, 0.0, tmp, 1.0, X, dM, 1, none, part.p, max_blocks, s);
    gram_to_host(nb);
    if (!cholesky_upper(p, hG.data(), R2, R2i)) return false;
    upload(dM, R2i);
    launch_bl_update(D, p, 0.0, out, 1.0, in(tmp), dM, 0, none, part.p, max_blocks, s);
    B.assign(pp, 0.0);
    for (int i = 0; i < p; ++i)
      for (int j = i; j < p; ++j) {
        double t = 0.0;
        for (int k = i; k <= j; ++k) t += R2[i * p + k] * R1[k * p + j];
        B[i * p + j] = t;
      }
    return true;
  };
  const size_t bl = D * (size_t)p;
  DevBuf<double> b0(bl), b1(bl), b2(bl);
  BlockOut Vprev = block(b0.p), Vk = block(b1.p), W = block(b2.p);
  // V_0 = QR(phi) and P = phi^T V_0
  BlockOut X0;
  for (int i = 0; i < p; ++i) X0.v[i] = phi[i].p;
  std::vector<double> B;
  int nb = launch_bl_update(D, p, 1.0, X0, 0.0, none, nullptr, 1, none, part.p, max_blocks, s);  // phi^T phi
  gram_to_host(nb);
  if (!cholqr2(in(X0), Vprev, Vk, B)) return false;
  nb = launch_bl_update(D, p, 1.0, Vk, 0.0, none, nullptr, 2, in(X0), part.p, max_blocks, s);  // P(k, i) = <phi_k, v_i>
  gram_to_host(nb);
  const std::vector<double> P(hG);  // row-major [k][i]
  std::vector<double> t((size_t)M0 * M0, 0.0);
  auto T = [&](int r, int c) -> double & { return t[(size_t)r + (size_t)M0 * c]; };
  // The steps run on the device with their QR: the p x p Cholesky factors are
  // computed by k_block_chol, so a step needs no host value. Step k leaves
  // rec_k = [A_k | B_{k+1} | QR failed] in device memory; the host reads it
  // once, fills T and runs the convergence test while step k + 1, enqueued
  // beforehand, runs on the GPU. A step enqueued past the stopping point is
  // discarded.
  const int nsteps = M0 / p;  // the last step (jdim = M0) needs no QR
  const int ldr = 2 * pp + 1;
  DevBuf<double> drec((size_t)ldr * nsteps), dqr(5 * (size_t)pp);
  QED_CUDA(cudaMemsetAsync(drec.p, 0, drec.bytes(), s));
  double *dR1 = dqr.p, *dR1i = dqr.p + pp, *dR2 = dqr.p + 2 * pp, *dR2i = dqr.p + 3 * pp, *dBt = dqr.p + 4 * pp;
  double *hrec = ws.pinned(2 * (size_t)ldr);
  cudaEvent_t ev[2];
  QED_CUDA(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming));
  QED_CUDA(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming));
  struct Events {
    cudaEvent_t *e;
    ~Events() {
      cudaEventDestroy(e[0]);
      cudaEventDestroy(e[1]);
    }
  } ev_guard{ev};
  auto enqueue = [&](int k) {
    // W = H V_k - V_{k-1} B_k^T, then A_k = V_k^T W
    H.apply_block(p, in(Vk), W, ws.red, s);
    double *rk = drec.p + (size_t)ldr * k;
    int nbk;
    if (k > 0)
      nbk = launch_bl_update(D, p, 1.0, W, -1.0, in(Vprev), dBt, 2, in(Vk), part.p, max_blocks, s);
    else
      nbk = launch_bl_update(D, p, 1.0, W, 0.0, none, nullptr, 2, in(Vk), part.p, max_blocks, s);
    launch_finalize_ld(part.p, nbk, pp, pp, rk, s);
    // W -= V_k A_k (with the gram of the result for the QR)
    nbk = launch_bl_update(D, p, 1.0, W, -1.0, in(Vk), rk, 1, none, part.p, max_blocks, s);
    if ((k + 1) * p < M0) {
      // W = V_{k+1} B_{k+1}, Cholesky QR twice, through V_{k-1}'s buffer
      launch_finalize_ld(part.p, nbk, pp, pp, dG, s);
      launch_block_chol(p, dG, kPivotMin, dR1, dR1i, nullptr, nullptr, nullptr, rk + 2 * pp, s);
      nbk = launch_bl_update(D, p, 0.0, Vprev, 1.0, in(W), dR1i, 1, none, part.p, max_blocks, s);
      launch_finalize_ld(part.p, nbk, pp, pp, dG, s);
      launch_block_chol(p, dG, 0.0, dR2, dR2i, dR1, rk + pp, dBt, rk + 2 * pp, s);
      launch_bl_update(D, p, 0.0, W, 1.0, in(Vprev), dR2i, 0, none, part.p, max_blocks, s);
    }
    QED_CUDA(cudaMemcpyAsync(hrec + (size_t)ldr * (k & 1), rk, ldr * sizeof(double), cudaMemcpyDeviceToHost, s));
    QED_CUDA(cudaEventRecord(ev[k & 1], s));
    const BlockOut nv = W;  // V_{k+1}
    W = Vprev;
    Vprev = Vk;
    Vk = nv;
  };
  double ev_old = 1e12;
  int jdim = 0;
  BandLowest lowest;
  PhaseScope ps_loop(kPhBlockLoop);
  enqueue(0);
  for (int k = 0;; ++k) {
    if ((k + 1) * p < M0) enqueue(k + 1);  // runs while the host handles step k
    QED_CUDA(cudaEventSynchronize(ev[k & 1]));
    const double *A = hrec + (size_t)ldr * (k & 1);
    for (int i = 0; i < p; ++i)
      for (int c = 0; c < p; ++c) T(k * p + i, k * p + c) = 0.5 * (A[i * p + c] + A[c * p + i]);
    jdim = (k + 1) * p;
    if (jdim >= M0) {
      jdim = M0;
      break;
    }
    if (jdim >= 4 * p) {  // bandLanczos step (12) at j = jdim, on the leading jdim x jdim block
      PhaseScope ps_check(kPhBandCheck);
      double ev0 = 0.0;
      bool fast = false;
      if (!no_degenerate) {  // only the lowest eigenvalue is needed
        std::vector<double> Bb((size_t)jdim * (p + 1), 0.0);
        for (int i = 0; i < jdim; ++i)
          for (int kk = 0; kk <= std::min(i, p); ++kk) Bb[(size_t)i * (p + 1) + kk] = T(i, i - kk);
        fast = band_lowest(jdim, p, Bb, lowest, &ev0);
      }
      if (!fast) {
        std::vector<double> Hpr((size_t)jdim * jdim), evs;
        for (int c = 0; c < jdim; ++c)
          for (int r = 0; r < jdim; ++r) Hpr[(size_t)r + (size_t)jdim * c] = T(r, c);
        if (!band_eigenvalues(jdim, p, Hpr, evs)) fail(QED_ERR_INTERNAL, "projected eigensolver failed");
        if (jdim > 1 && evs[1] - evs[0] < min_gap && no_degenerate) {
          ws.sync();
          fail(QED_ERR_LANCZOS, "band Lanczos: the gap between the first two eigenvalues is smaller than " +
                                    std::to_string(min_gap));
        }
        ev0 = evs[0];
        lowest.valid = false;
      }
      const double test = std::fabs(ev0 - ev_old);
      ev_old = ev0;
      if (test < accur_bl) break;
    }
    if (A[2 * pp] != 0.0) {  // a QR pivot below kPivotMin: the band recurrence takes over
      ws.sync();
      return false;
    }
    const double *Bn = A + pp;
    for (int r = 0; r < p; ++r)
      for (int c = r; c < p; ++c) {
        T((k + 1) * p + r, k * p + c) = Bn[r * p + c];
        T(k * p + c, (k + 1) * p + r) = Bn[r * p + c];
      }
  }
  ws.sync();
  for (auto &f : phi) f.release();
  Mout = jdim;
  PhaseScope ps_eig(kPhBandEig);
  std::vector<double> Hpr((size_t)jdim * jdim), U;
  for (int c = 0; c < jdim; ++c)
    for (int r = 0; r < jdim; ++r) Hpr[(size_t)r + (size_t)jdim * c] = T(r, c);
  if (!band_eig_rows(jdim, p, Hpr, p, evals, U)) fail(QED_ERR_INTERNAL, "projected eigensolver failed");
  Q.assign((size_t)p * jdim, 0.0);
  for (int m = 0; m < jdim; ++m)
    for (int i = 0; i < p; ++i) {
      double acc = 0.0;
      for (int kk = 0; kk < p; ++kk) acc += P[(size_t)i * p + kk] * U[(size_t)kk + (size_t)p * m];
      Q[(size_t)i + (size_t)p * m] = acc;
    }
  return true;
}

}  // namespace

int mgs_qr(size_t D, int p, double *X, double tol, std::vector<double> &R, Workspace &ws) {
  R.assign((size_t)p * p, 0.0);
  cudaStream_t s = ws.stream;
  for (int l = 0; l < p; ++l) {
    double *xl = X + (size_t)l * D;
    for (int k = 0; k < l; ++k) {
      VecList one;
      one.n = 1;
      one.v[0] = X + (size_t)k * D;
      const int nb = launch_dots(D, xl, 1.0, 0, one, ws.red, s);
      const double z = ws.sums(nb, 1)[0];
      R[(size_t)k * p + l] = z;
      launch_axpby(D, 1.0, xl, -z, X + (size_t)k * D, 0, ws.red, s);
    }
    VecList self;
    self.n = 1;
    self.v[0] = xl;
    const int nb = launch_dots(D, xl, 1.0, 0, self, ws.red, s);
    const double nrm = std::sqrt(ws.sums(nb, 1)[0]);
    if (nrm < tol) return l;
    R[(size_t)l * p + l] = nrm;
    launch_scale(D, xl, 1.0 / nrm, s);
  }
  return p;
}

void block_lanczos_mcf(const KrylovOp &H, Workspace &ws, const double *Q0, int p, bool qr, McfFloors &out) {
  out = McfFloors();
  out.p = p;
  const size_t D = H.D;
  if (D == 0 || p < 1 || p > 16) fail(QED_ERR_ARGUMENT, "block Lanczos: block size outside [1, 16]");
  cudaStream_t s = ws.stream;
  const double accur_def = opt_double("accur_deflation");
  double accur_bl = opt_double("accur_band_lanczos");
  if (accur_bl < 0.0) accur_bl = 0.0;
  int M0 = (int)(14 * p * std::log(1.0 * D));
  if (M0 > opt_int("max_iter_BL")) M0 = (int)opt_int("max_iter_BL");
  constexpr double kPivotMin = 1e-4;
  const int pp = p * p;
  const int max_blocks = 4096;
  DevBuf<double> part((size_t)max_blocks * pp), dsmall(2 * (size_t)pp);
  double *dG = dsmall.p, *dM = dsmall.p + pp;
  std::vector<double> hG(pp);
  auto gram_to_host = [&](int nb) {
    launch_finalize_ld(part.p, nb, pp, pp, dG, s);
    QED_CUDA(cudaMemcpyAsync(hG.data(), dG, pp * sizeof(double), cudaMemcpyDeviceToHost, s));
    ws.sync();
  };
  auto upload = [&](const std::vector<double> &h) {
    QED_CUDA(cudaMemcpyAsync(dM, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  };
  const BlockIn none;
  auto block = [&](double *base) {
    BlockOut o;
    for (int c = 0; c < p; ++c) o.v[c] = base + (size_t)c * D;
    return o;
  };
  auto in = [&](double *base) {
    BlockIn i;
    for (int c = 0; c < p; ++c) i.v[c] = base + (size_t)c * D;
    return i;
  };
  const size_t bl = D * (size_t)p;
  DevBuf<double> b0(bl), b1(bl), b2(bl), b3(bl);
  double *Qprev = b0.p, *Qcur = b1.p, *Z = b2.p, *Tmp = b3.p;
  QED_CUDA(cudaMemcpyAsync(Qcur, Q0, bl * sizeof(double), cudaMemcpyDeviceToDevice, s));
  std::vector<double> Aj(pp), Bj(pp), Bt(pp), R1, R1i, R2, R2i;
  double ev_old = 1e12;
  BandLowest lowest;
  const int bw = qr ? p : 2 * p - 1;  // half-bandwidth of the projected matrix
  // convergence test on the (j + 1) p leading rows (blockLanczos step 6)
  auto converged = [&](int j) {
    if (!((j + 1) >= 2 * p && (j + 1) % p == 0)) return false;
    const int n = (j + 1) * p;
    auto T = [&](int r, int c) -> double {  // r >= c, r - c <= bw
      const int I = r / p, J = c / p;
      if (I == J) return out.A[(size_t)I * pp + (r % p) * p + (c % p)];
      if (I == J + 1) return out.B[(size_t)J * pp + (r % p) * p + (c % p)];
      return 0.0;
    };
    std::vector<double> Bb((size_t)n * (bw + 1), 0.0);
    for (int i = 0; i < n; ++i)
      for (int k = 0; k <= std::min(i, bw); ++k) Bb[(size_t)i * (bw + 1) + k] = T(i, i - k);
    double ev0 = 0.0;
    if (!band_lowest(n, bw, Bb, lowest, &ev0)) {
      std::vector<double> full((size_t)n * n, 0.0), evs;
      for (int i = 0; i < n; ++i)
        for (int k = 0; k <= std::min(i, bw); ++k) {
          full[(size_t)i + (size_t)n * (i - k)] = Bb[(size_t)i * (bw + 1) + k];
          full[(size_t)(i - k) + (size_t)n * i] = Bb[(size_t)i * (bw + 1) + k];
        }
      if (!band_eigenvalues(n, bw, full, evs)) fail(QED_ERR_INTERNAL, "projected eigensolver failed");
      ev0 = evs[0];
      lowest.valid = false;
    }
    const double delta = std::fabs(ev0 - ev_old);
    ev_old = ev0;
    return delta < accur_bl;
  };
  PhaseScope ps_loop(kPhBlockLoop);
  for (int j = 0; j < M0; ++j) {
    // Z = H Q_j - Q_{j-1} B_{j-1}^T, A_j = Q_j^T Z (upper triangle, mirrored)
    H.apply_block(p, in(Qcur), block(Z), ws.red, s);
    int nb;
    if (j > 0) {
      for (int r = 0; r < p; ++r)
        for (int c = 0; c < p; ++c) Bt[(size_t)r * p + c] = Bj[(size_t)c * p + r];
      upload(Bt);
      nb = launch_bl_update(D, p, 1.0, block(Z), -1.0, in(Qprev), dM, 2, in(Qcur), part.p, max_blocks, s);
    } else {
      nb = launch_bl_update(D, p, 1.0, block(Z), 0.0, none, nullptr, 2, in(Qcur), part.p, max_blocks, s);
    }
    gram_to_host(nb);
    for (int l = 0; l < p; ++l)
      for (int k = 0; k <= l; ++k) Aj[(size_t)k * p + l] = Aj[(size_t)l * p + k] = hG[(size_t)k * p + l];
    out.A.insert(out.A.end(), Aj.begin(), Aj.end());
    // Z -= Q_j A_j, with the Gram matrix of the result
    upload(Aj);
    nb = launch_bl_update(D, p, 1.0, block(Z), -1.0, in(Qcur), dM, 1, none, part.p, max_blocks, s);
    gram_to_host(nb);
    bool singular = false;
    double *Qnext = Qprev;  // Q_{j-1}'s buffer is free once Z has been formed
    if (qr) {
      bool chol = cholesky_upper(p, hG.data(), R1, R1i);
      for (int i = 0; i < p && chol; ++i) chol = R1[(size_t)i * p + i] >= kPivotMin;
      if (chol) {  // Cholesky QR twice: Z -> Tmp -> Q_{j+1}; B_j = R2 R1
        upload(R1i);
        nb = launch_bl_update(D, p, 0.0, block(Tmp), 1.0, in(Z), dM, 1, none, part.p, max_blocks, s);
        gram_to_host(nb);
        chol = cholesky_upper(p, hG.data(), R2, R2i);
        if (chol) {
          upload(R2i);
          launch_bl_update(D, p, 0.0, block(Qnext), 1.0, in(Tmp), dM, 0, none, part.p, max_blocks, s);
          std::fill(Bj.begin(), Bj.end(), 0.0);
          for (int i = 0; i < p; ++i)
            for (int c = i; c < p; ++c) {
              double t = 0.0;
              for (int k = i; k <= c; ++k) t += R2[(size_t)i * p + k] * R1[(size_t)k * p + c];
              Bj[(size_t)i * p + c] = t;
            }
        }
      }
      if (!chol) {  // the reference's column-by-column QR, which may deflate
        const int l = mgs_qr(D, p, Z, accur_def, Bj, ws);
        if (l < p) {
          singular = true;
          QED_CUDA(cudaMemsetAsync(Z + (size_t)l * D, 0, (size_t)(p - l) * D * sizeof(double), s));
        }
        Qnext = Z;
      }
      out.B.insert(out.B.end(), Bj.begin(), Bj.end());
      out.M = j + 1;
      if (converged(j) || singular) break;
    } else {
      // polar factor: G = V diag(d) V^T, B_j = V d^(1/2) V^T, Q_{j+1} = Z V d^(-1/2) V^T
      std::vector<double> d, V;
      if (!sym_eig(p, hG, d, &V)) fail(QED_ERR_INTERNAL, "block Lanczos: Gram eigensolver failed");
      for (int m = 0; m < p; ++m)
        if (d[m] < accur_def * accur_def) singular = true;
      std::vector<double> Binv(pp, 0.0);
      for (int r = 0; r < p; ++r)
        for (int c = 0; c < p; ++c) {
          double b = 0.0, bi = 0.0;
          for (int m = 0; m < p; ++m) {
            const double vv = V[(size_t)r + (size_t)p * m] * V[(size_t)c + (size_t)p * m];
            b += vv * std::sqrt(std::max(d[m], 0.0));
            if (!singular) bi += vv / std::sqrt(d[m]);
          }
          Bj[(size_t)r * p + c] = b;
          Binv[(size_t)r * p + c] = bi;
        }
      out.B.insert(out.B.end(), Bj.begin(), Bj.end());
      out.M = j + 1;
      if (singular) break;
      upload(Binv);
      launch_bl_update(D, p, 0.0, block(Qnext), 1.0, in(Z), dM, 0, none, part.p, max_blocks, s);
      if (converged(j)) break;
    }
    // Q_{j-1} <- Q_j, Q_j <- Q_{j+1}
    double *freed = Qprev;
    Qprev = Qcur;
    if (Qnext == Z) Z = freed;  // the MGS path left Q_{j+1} in Z's buffer
    Qcur = Qnext;
  }
  ws.sync();
}

bool band_lanczos_qmatrix(const KrylovOp &H, Workspace &ws, std::vector<DevBuf<double>> &phi,
                          std::vector<double> &evals, std::vector<double> &Q, int &Mout) {
  const size_t D = H.D;
  const int p = (int)phi.size();
  cudaStream_t s = ws.stream;
  if (D == 0 || p == 0) {
    Mout = 0;
    return false;
  }
  if ((long)D >= opt_int("block_lanczos_min_dim") && p >= opt_int("block_lanczos_min_p")) {
    if (block_lanczos_qmatrix(H, ws, phi, evals, Q, Mout)) return true;
    if (profiling()) profile_add(kPhBlockFallback, 0.0);
  }
  // number of iterations (Hamiltonian::build_Q_matrix, Hamiltonian_base.hpp:236-239)
  int M0 = (int)(14 * p * std::log(1.0 * D));
  if (!(M0 > 1)) fail(QED_ERR_INTERNAL, "Assertion failed: M>1 in build_Q_matrix");
  const double accur_deflation = opt_double("accur_deflation");
  double accur_bl = opt_double("accur_band_lanczos");
  if (accur_bl < 0.0) accur_bl = 0.0;
  const long max_iter_BL = opt_int("max_iter_BL");
  const double min_gap = opt_double("band_lanczos_minimum_gap");
  const bool no_degenerate = opt_bool("no_degenerate_BL");
  // bandLanczos (src_ed/Hamiltonian/Lanczos.hpp:214-395)
  int pc = p;
  if (M0 > max_iter_BL) M0 = (int)max_iter_BL;
  int M0p = (M0 / p + 1) * p;
  M0 = M0p - pc;
  VecPool pool(D);
  std::vector<int> v(M0p + 1, -1);  // slot of Lanczos vector j
  std::vector<double> t((size_t)M0 * M0, 0.0);
  auto T = [&](int r, int c) -> double & { return t[(size_t)r + (size_t)M0 * c]; };
  std::vector<double> P((size_t)p * std::max(M0, 1), 0.0);
  std::vector<int> def(M0 + 1, 0), I;
  for (int i = 0; i < p; ++i) {
    v[i] = pool.get();
    QED_CUDA(cudaMemcpyAsync(pool.p(v[i]), phi[i].p, D * sizeof(double), cudaMemcpyDeviceToDevice, s));
  }
  bool phi_alive = true;
  double ev_old = 1e12;
  int j = 0;
  int nd = 0;
  VecList ys;
  PhaseScope ps_loop(kPhBandLoop);
  // step (12): convergence test on the lowest eigenvalue of the projected matrix
  // Without deflation t is banded (half-bandwidth p) and only its lowest
  // eigenvalue is needed: band_lowest (warm-started inverse iteration, O(j p^2)
  // per test, certified to 1e-14) with band_eigenvalues (O(j^2 p)) where it
  // declines; after a deflation, the dense eigenvalues.
  BandLowest lowest;
  auto converged_at = [&](int jc) {
    PhaseScope ps_check(kPhBandCheck);
    double ev0 = 0.0;
    bool fast = false;
    if (nd == 0 && !no_degenerate) {
      std::vector<double> Bb((size_t)jc * (p + 1), 0.0);
      for (int i = 0; i < jc; ++i)
        for (int kk = 0; kk <= std::min(i, p); ++kk) Bb[(size_t)i * (p + 1) + kk] = T(i, i - kk);
      fast = band_lowest(jc, p, Bb, lowest, &ev0);
    }
    if (!fast) {
      std::vector<double> Hpr((size_t)jc * jc), ev;
      for (int c = 0; c < jc; ++c)
        for (int r = 0; r < jc; ++r) Hpr[(size_t)r + (size_t)jc * c] = T(r, c);
      const bool ok = (nd == 0) ? band_eigenvalues(jc, p, Hpr, ev) : sym_eig(jc, Hpr, ev, nullptr);
      if (!ok) fail(QED_ERR_INTERNAL, "projected eigensolver failed");
      if (jc > 1 && ev[1] - ev[0] < min_gap && no_degenerate)
        fail(QED_ERR_LANCZOS, "band Lanczos: the gap between the first two eigenvalues is smaller than " +
                                  std::to_string(min_gap));
      ev0 = ev[0];
      lowest.valid = false;
    }
    double test = std::fabs(ev0 - ev_old);
    ev_old = ev0;
    return test < accur_bl;
  };
  // Device-resident steps: while nothing has been deflated (nd == 0) and the
  // window is in steady state (j > pc: every step releases v_{j-pc-1} and
  // takes its slot for v_{j+pc}), a chunk of steps runs with all scalars in
  // device memory and no host round trip: z and 1/z (with the deflation test),
  // the window dots, T(j, j) and the subtraction coefficients of the row pass.
  // A step whose z falls below accur_deflation raises a device flag; it and
  // every later step of the chunk then do nothing, and the host redoes that
  // step on the host path (which deflates). The host reads the chunk's
  // T entries once and fills T exactly as the step-by-step path does.
  constexpr int kRec = 34;          // z, window dots (<= 31), T(j, j)
  constexpr int kBandChunk = 32;
  DevBuf<double> drec((size_t)kRec * (M0p + 1)), dinv(1);
  DevBuf<int> dflag(1);
  std::vector<double> hrec;
  int host_step = -1;
  for (j = 0; j < M0; ++j) {
    if (phi_alive && j >= p) {  // P(k, j) is only used for j < p (Q = P U over k < p)
      for (auto &f : phi) f.release();
      phi_alive = false;
    }
    if (nd == 0 && j >= p && j > pc && j != host_step) {
      int je = std::min(M0 - 1, j + kBandChunk - 1);
      int chk = std::max(j, 4 * p);
      chk = ((chk + p - 1) / p) * p;  // first convergence test at or after j
      if (chk <= je) je = chk;
      const std::vector<int> free0 = pool.free_list, v0 = v;
      QED_CUDA(cudaMemsetAsync(dflag.p, 0, sizeof(int), s));
      auto slots = [&](int jj) {  // steady-state window move of step jj
        pool.put(v[jj - pc - 1]);
        v[jj - pc - 1] = -1;
        v[jj + pc] = pool.get();
      };
      for (int jj = j; jj <= je; ++jj) {
        double *rec = drec.p + (size_t)kRec * jj;
        double *vj = pool.p(v[jj]);
        VecList one;  // (3)-(4): z = |v_j| and the deflation test
        one.n = 1;
        one.v[0] = vj;
        one.skip = dflag.p;
        int nb = launch_dots(D, vj, 1.0, 0, one, ws.red, s);
        launch_finalize_norm(ws.red.partials, nb, accur_deflation, rec, dinv.p, dflag.p, jj, s);
        VecList win;  // (5)-(6): v_j /= z; t_k = <v_j, v_k>; v_k -= t_k v_j
        win.skip = dflag.p;
        win.xsdev = dinv.p;
        for (int k = jj + 1; k < jj + pc; ++k) win.v[win.n++] = pool.p(v[k]);
        if (win.n) {
          nb = launch_dots(D, vj, 1.0, 1, win, ws.red, s);
          launch_finalize(ws.red.partials, nb, win.n, rec + 1, s);
          win.cdev = rec + 1;
          launch_multi_axpy(D, vj, 1.0, win, 0, ws.red, s);
        } else {
          launch_scale_dev(D, vj, dinv.p, dflag.p, s);
        }
        // (7)-(8): w = H v_j - sum_{k=j-pc}^{j-1} T(j, k) v_k, T(j, k) = rec[k - j + pc]
        slots(jj);
        double *w = pool.p(v[jj + pc]);
        SubList sub;
        sub.cdev = rec;
        for (int k = jj - pc; k < jj; ++k) sub.z[sub.n++] = pool.p(v[k]);
        nb = H.apply(vj, 1.0, w, sub, 1, ws.red, s, dflag.p);
        launch_finalize(ws.red.partials, nb, 1, rec + pc, s);  // (10): T(j, j) = <v_j, w>
        launch_axpy_dev(D, w, vj, rec + pc, ws.red, s, dflag.p);
      }
      const int n = je - j + 1;
      hrec.resize((size_t)kRec * n);
      QED_CUDA(cudaMemcpyAsync(hrec.data(), drec.p + (size_t)kRec * j, hrec.size() * sizeof(double),
                               cudaMemcpyDeviceToHost, s));
      int flag = 0;
      QED_CUDA(cudaMemcpyAsync(&flag, dflag.p, sizeof(int), cudaMemcpyDeviceToHost, s));
      ws.sync();
      const int jd = flag ? flag - 1 : je + 1;  // first step not done on the device
      if (jd <= je) {  // the window moves of the skipped steps are undone
        pool.free_list = free0;
        v = v0;
        for (int jj = j; jj < jd; ++jj) slots(jj);
      }
      for (int jj = j; jj < jd; ++jj) {
        const double *r = hrec.data() + (size_t)kRec * (jj - j);
        T(jj, jj - pc) = r[0];
        for (int k = jj + 1; k < jj + pc; ++k) T(jj, k - pc) = r[k - jj];
        for (int k = jj - pc; k < jj; ++k) T(k, jj) = T(jj, k);
        T(jj, jj) = r[pc];
      }
      if (jd <= je) {
        host_step = jd;
        j = jd - 1;
        continue;
      }
      j = je;
      if (j >= 4 * p && j % p == 0 && converged_at(j)) break;
      continue;
    }
    // step (3): z = |v_j|
    ys.n = 1;
    ys.v[0] = pool.p(v[j]);
    int nb = launch_dots(D, pool.p(v[j]), 1.0, 0, ys, ws.red, s);
    const double z = std::sqrt(ws.sums(nb, 1)[0]);
    if (z < accur_deflation) {  // step (4): deflation
      if (j >= pc) {
        I.push_back(j - pc);
        def[j - pc] = 1;
        nd++;
      }
      pc--;
      if (pc == 0) break;
      pool.put(v[j]);
      for (int k = j; k < j + pc; ++k) v[k] = v[k + 1];
      v[j + pc] = -1;
      j--;
      continue;
    }
    if (j >= pc) T(j, j - pc) = z;
    // normalise v_j; dots with phi (j < p) and with the window v_{j+1..j+pc-1}
    ys.n = 0;
    const bool need_P = (j < p) && phi_alive;
    if (need_P)
      for (int k = 0; k < p; ++k) { ys.v[ys.n] = phi[k].p; ys.c[ys.n++] = 0.0; }
    const int nP = ys.n;
    for (int k = j + 1; k < j + pc; ++k) { ys.v[ys.n] = pool.p(v[k]); ys.c[ys.n++] = 0.0; }
    nb = launch_dots(D, pool.p(v[j]), 1.0 / z, 1, ys, ws.red, s);
    std::vector<double> dots;
    if (ys.n) {
      const double *h = ws.sums(nb, ys.n);
      dots.assign(h, h + ys.n);
    }
    for (int k = 0; k < nP; ++k) P[(size_t)k + (size_t)p * j] = dots[k];
    // step (6): v_k -= <v_j, v_k> v_j
    VecList ax;
    for (int k = j + 1; k < j + pc; ++k) {
      double zz = dots[nP + (k - j - 1)];
      ax.v[ax.n] = pool.p(v[k]);
      ax.c[ax.n++] = zz;
      if (k >= pc) T(j, k - pc) = zz;
    }
    if (ax.n) launch_multi_axpy(D, pool.p(v[j]), 1.0, ax, 0, ws.red, s);
    // step (7): v_{j+pc} = H v_j, fused with step (8): - sum_{k0<=k<j} t(k,j) v_k
    int k0 = 0;
    if (j > pc) {
      k0 = j - pc;
      if (def[k0 - 1] == 0) {
        pool.put(v[k0 - 1]);
        v[k0 - 1] = -1;
      }
    }
    v[j + pc] = pool.get();
    double *w = pool.p(v[j + pc]);
    SubList sub;
    for (int k = k0; k < j; ++k) {
      T(k, j) = T(j, k);
      if (sub.n == 32) fail(QED_ERR_UNSUPPORTED, "band width above 32");
      sub.c[sub.n] = T(k, j);
      sub.z[sub.n++] = pool.p(v[k]);
    }
    nb = H.apply(pool.p(v[j]), 1.0, w, sub, nd == 0 ? 1 : 0, ws.red, s);
    double wjj;
    if (nd == 0) {
      wjj = ws.sums(nb, 1)[0];
    } else {
      // step (9): orthogonalise against the deflated vectors, one at a time
      for (int k = 0; k < nd; ++k) {
        VecList one;
        one.n = 1;
        one.v[0] = w;
        int nb2 = launch_dots(D, pool.p(v[I[k]]), 1.0, 0, one, ws.red, s);
        double ww = ws.sums(nb2, 1)[0];
        launch_axpby(D, 1.0, w, -ww, pool.p(v[I[k]]), 0, ws.red, s);
        T(I[k], j) = ww;
      }
      VecList one;
      one.n = 1;
      one.v[0] = w;
      int nb2 = launch_dots(D, pool.p(v[j]), 1.0, 0, one, ws.red, s);
      wjj = ws.sums(nb2, 1)[0];
    }
    launch_axpby(D, 1.0, w, -wjj, pool.p(v[j]), 0, ws.red, s);
    T(j, j) = wjj;
    for (int k = 0; k < nd; ++k) T(j, I[k]) = T(I[k], j);
    if (j >= 4 * p && j % p == 0 && converged_at(j)) break;
  }
  ws.sync();
  Mout = j;
  if (j == 0) return false;
  PhaseScope ps_eig(kPhBandEig);
  // projected eigensystem and Q = P U, summed over the first p Lanczos vectors
  std::vector<double> Hpr((size_t)j * j), U;
  for (int c = 0; c < j; ++c)
    for (int r = 0; r < j; ++r) Hpr[(size_t)r + (size_t)j * c] = T(r, c);
  const int kmax = std::min(p, j);
  // only rows k < p of the eigenvectors enter Q; without deflation the
  // projected matrix is banded (half-bandwidth p)
  int ldu = j;
  if (nd == 0) {
    if (!band_eig_rows(j, p, Hpr, kmax, evals, U)) fail(QED_ERR_INTERNAL, "projected eigensolver failed");
    ldu = kmax;
  } else if (!sym_eig(j, Hpr, evals, &U)) {
    fail(QED_ERR_INTERNAL, "projected eigensolver failed");
  }
  Q.assign((size_t)p * j, 0.0);
  for (int m = 0; m < j; ++m)
    for (int i = 0; i < p; ++i) {
      double acc = 0.0;
      for (int k = 0; k < kmax; ++k) acc += P[(size_t)i + (size_t)p * k] * U[(size_t)k + (size_t)ldu * m];
      Q[(size_t)i + (size_t)p * m] = acc;
    }
  return true;
}

}  // namespace qed
