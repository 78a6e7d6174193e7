// The C ABI of include/qed_b200.h: registries of models / instances / sector
// Hamiltonians, and the error convention (status code + per-thread message).
#include <algorithm>
#include <chrono>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <thread>
#include <map>
#include <memory>
#include <mutex>
#include <string>

#include "common.hpp"
#include "instance.hpp"
#include "options.hpp"
#include "symmetry.hpp"
#include "mixed.hpp"
#include "qed_b200.h"
#if defined(__SSE2__)
#include <emmintrin.h>
#endif
#include "worker_pool.hpp"

using namespace qed;

// mult_add pipeline: x goes up in kMultAddChunks row blocks, each block's row
// pass starting as soon as its copy lands; H x comes back in the same blocks and
// the host adds each block into y while the next one is in flight. Only the
// last block's add runs after the transfers end, so blocks are small (41 MB of
// H x each on the 4x4 sector).
constexpr int kMultAddChunks = 32;

// y[i] += s[i]. The sums are not read again soon, so where y is 16-byte aligned
// they are written with non-temporal stores: no read-for-ownership of y's lines,
// 24 instead of 32 bytes of host memory traffic per element. Same sums as the
// scalar loop (plain IEEE additions).
static void add_streaming(double *y, const double *s, size_t n) {
  size_t i = 0;
#if defined(__SSE2__)
  for (; i < n && ((uintptr_t)(y + i) & 15u); ++i) y[i] += s[i];
  for (; i + 4 <= n; i += 4) {
    const __m128d a = _mm_add_pd(_mm_load_pd(y + i), _mm_loadu_pd(s + i));
    const __m128d b = _mm_add_pd(_mm_load_pd(y + i + 2), _mm_loadu_pd(s + i + 2));
    _mm_stream_pd(y + i, a);
    _mm_stream_pd(y + i + 2, b);
  }
  _mm_sfence();
#endif
  for (; i < n; ++i) y[i] += s[i];
}

struct qed_mixed_hamiltonian {
  std::unique_ptr<MixedHamiltonian> H;
  std::mutex m;
};

struct qed_hamiltonian {
  std::unique_ptr<SectorOp> H;
  DevBuf<double> x, y;
  DevBuf<double> partials;  // per-block partial sums of apply_dots_device
  std::mutex m;             // calls on one handle are serialised
  // mult_add staging: device H x, pinned host copy of it, copy stream, events
  DevBuf<double> z;
  double *hz = nullptr;
  size_t hz_n = 0;
  cudaStream_t copy = nullptr;
  cudaEvent_t ev_in[kMultAddChunks] = {}, ev_out[kMultAddChunks] = {};
  ~qed_hamiltonian() {
    if (copy) cudaStreamSynchronize(copy);
    for (int k = 0; k < kMultAddChunks; ++k) {
      if (ev_in[k]) cudaEventDestroy(ev_in[k]);
      if (ev_out[k]) cudaEventDestroy(ev_out[k]);
    }
    if (copy) cudaStreamDestroy(copy);
    if (hz) cudaFreeHost(hz);
  }
};

namespace {

thread_local std::string t_err;

// Models and instances live in process-global maps, as the reference's
// (src_ed/qcm_ED.cpp:25-26). GPU work runs on a Workspace (stream + reduction
// buffers) owned by the calling host thread, so threads driving different
// instances overlap on the GPU; calls on one instance are serialised by its mutex.
std::mutex g_reg;
std::map<std::string, std::shared_ptr<Model>> g_models;
std::map<int, std::shared_ptr<Instance>> g_instances;
std::atomic<int> g_device{0};
std::atomic<bool> g_device_fixed{false};

Workspace &ws() {
  thread_local std::unique_ptr<Workspace> tws;
  if (!tws) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0)
      fail(QED_ERR_NO_DEVICE, std::string("no CUDA device available: ") + cudaGetErrorString(e));
    const int dev = g_device.load();
    QED_CUDA(cudaSetDevice(dev));
    static std::once_flag pool_once;
    std::call_once(pool_once, [dev] {
      // keep freed blocks in the device's pool: repeated solves reuse them
      cudaMemPool_t pool;
      if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
      }
    });
    g_device_fixed = true;
    tws.reset(new Workspace());
  }
  return *tws;
}

template <class F> int guarded(F &&f) {
  try {
    f();
    return QED_OK;
  } catch (const Error &e) {
    t_err = e.what();
    return e.code;
  } catch (const std::out_of_range &e) {
    t_err = std::string("unknown name or label: ") + e.what();
    return QED_ERR_ARGUMENT;
  } catch (const std::exception &e) {
    t_err = e.what();
    return QED_ERR_INTERNAL;
  }
}

std::shared_ptr<Instance> instance(int label) {
  std::lock_guard<std::mutex> l(g_reg);
  auto it = g_instances.find(label);
  if (it == g_instances.end())
    fail(QED_ERR_ARGUMENT, "The cluster instance label " + std::to_string(label) + " is out of range.");
  return it->second;
}

// Runs fn(i) for i in [0, n) on `threads` host threads (each with its own
// Workspace / CUDA stream). Returns the status of the first failure.
WorkerPool &pool() {
  static WorkerPool *p = new WorkerPool;  // never destroyed: its threads live until exit
  return *p;
}

template <class F> int run_batch(int n, int threads, F &&fn) {
  if (n <= 0) return QED_OK;
  int hw = (int)std::thread::hardware_concurrency();
  if (threads <= 0) threads = hw > 0 ? hw : 8;
  threads = std::max(1, std::min({threads, n, 64}));
  std::atomic<int> next{0};
  std::atomic<int> first_code{QED_OK};
  std::mutex emtx;
  std::string first_msg;
  auto work = [&] {
    for (int i = next++; i < n; i = next++) {
      int rc = guarded([&] { fn(i); });
      if (rc != QED_OK) {
        int expected = QED_OK;
        if (first_code.compare_exchange_strong(expected, rc)) {
          std::lock_guard<std::mutex> l(emtx);
          first_msg = t_err;
        }
      }
    }
  };
  pool().run(threads - 1, work);
  if (first_code != QED_OK) t_err = first_msg;
  return first_code;
}
// The batched eigenvalue pass spreads its per-sector Ritz tests over the pool.
// Those tests run inside a batch call whose own work loop may hold the pool,
// so they take a second, smaller pool of their own.
WorkerPool &ritz_pool() {
  static WorkerPool *p = new WorkerPool;
  return *p;
}

const bool g_parallel_for_set = [] {
  set_parallel_for([](int n, const std::function<void(int)> &fn) {
    int hw = (int)std::thread::hardware_concurrency();
    const int threads = std::max(1, std::min({hw > 0 ? hw : 8, n, 64}));
    std::atomic<int> next{0};
    auto work = [&] {
      for (int i = next++; i < n; i = next++) fn(i);
    };
    ritz_pool().run(threads - 1, work);
  });
  return true;
}();

// Weighted tasks run longest-first (LPT) on the batch thread pool.
struct Task {
  double cost;
  std::function<void()> fn;
};

int run_tasks(std::vector<Task> &tasks, int threads) {
  std::stable_sort(tasks.begin(), tasks.end(), [](const Task &a, const Task &b) { return a.cost > b.cost; });
  return run_batch((int)tasks.size(), threads, [&](int i) { tasks[i].fn(); });
}

// The instances of a batch call, each once, locked in label order for the
// whole call (single-instance entries lock one instance at a time, so the
// order cannot deadlock).
struct BatchSet {
  std::vector<std::shared_ptr<Instance>> inst;  // unique, by label
  std::vector<std::unique_lock<std::mutex>> locks;
  explicit BatchSet(const int *labels, int n) {
    std::map<int, std::shared_ptr<Instance>> u;
    for (int i = 0; i < n; ++i) u[labels[i]] = instance(labels[i]);
    for (auto &x : u) inst.push_back(x.second);
    for (auto &I : inst) locks.emplace_back(I->mtx);
  }
};

// Ground states of a batch: every target sector of every unsolved instance as
// one task (eigenvalue pass), the selection per instance, then the eigenvector
// of every kept state as one task.
int batch_ground_states(BatchSet &b, int threads) {
  std::vector<Instance *> todo;
  int rc = guarded([&] {
    for (auto &I : b.inst) {
      if (I->gs_solved) continue;
      if (!I->is_correlated) {  // the one-body problem: nothing to spread over threads
        I->low_energy_states(ws());
        continue;
      }
      todo.push_back(I.get());
    }
  });
  if (rc != QED_OK || todo.empty()) return rc;
  std::vector<std::vector<SectorSolve>> res(todo.size());
  std::vector<Task> tasks;
  DeferredSectors defer;  // small Lanczos sectors: one batched eigenvalue pass below
  for (size_t k = 0; k < todo.size(); ++k) {
    Instance *I = todo[k];
    res[k].resize(I->target_sectors.size());
    size_t i = 0;
    for (auto &sec : I->target_sectors) {
      SectorSolve *out = &res[k][i++];
      Sector s = sec;
      tasks.push_back({(double)I->sector_dim(s), [I, s, out, &defer] { I->solve_sector(s, *out, ws(), &defer); }});
    }
  }
  if ((rc = run_tasks(tasks, threads)) != QED_OK) return rc;
  // eigenvalue passes: every large sector as one task, all small sectors as one
  // batched task, so that the batched launches overlap the large sectors' work
  tasks.clear();
  double small_cost = 0.0;
  for (auto &it : defer.items) small_cost += (double)it.H->D;
  if (!defer.items.empty())
    tasks.push_back({small_cost, [&defer] { lanczos_energy_batch(defer.items, ws()); }});
  for (auto &it : defer.large) {
    LanczosBatchItem *p = &it;
    tasks.push_back({(double)it.H->D, [p] {
                       try {
                         *p->out = lanczos_energy(*p->H, ws(), p->seed);
                       } catch (const Error &e) {
                         fail(e.code, std::string(e.what()) + p->where);
                       }
                     }});
  }
  if ((rc = run_tasks(tasks, threads)) != QED_OK) return rc;
  rc = guarded([&] {
    defer.items.clear();
    defer.large.clear();
    defer.ops.clear();
    for (size_t k = 0; k < todo.size(); ++k) todo[k]->select_states(res[k]);
  });
  if (rc != QED_OK) return rc;
  res.clear();
  tasks.clear();
  for (Instance *I : todo)
    for (auto &st : I->states) {
      State *sp = st.get();
      tasks.push_back({(double)I->sector_dim(sp->sec), [I, sp] { I->state_vector(*sp, ws()); }});
    }
  if ((rc = run_tasks(tasks, threads)) != QED_OK) return rc;
  tasks.clear();
  for (Instance *I : todo) {  // operator averages, one task per instance
    double cost = 0.0;
    for (auto &st : I->states) cost += (double)I->sector_dim(st->sec);
    tasks.push_back({cost * (double)I->value.size(), [I] { I->finish_gs(ws()); }});
  }
  return run_tasks(tasks, threads);
}

// Green functions of a batch: each Q-matrix half (state, spin, hole/electron)
// or continued-fraction set (state, spin) as one task, then the per-state
// combination and the per-instance averages.
int batch_green_functions(BatchSet &b, int threads) {
  int rc = batch_ground_states(b, threads);
  if (rc != QED_OK) return rc;
  struct Job {
    Instance *I;
    State *st;
    bool sd;
    QPart parts[2];
  };
  std::vector<Instance *> todo;
  rc = guarded([&] {
    for (auto &I : b.inst)
      if (!I->gf_solved) {
        I->check_gf_solvable();
        todo.push_back(I.get());
      }
  });
  if (rc != QED_OK || todo.empty()) return rc;
  std::vector<std::unique_ptr<Job>> jobs;
  std::vector<Task> tasks;
  for (Instance *I : todo) {
    const int p = I->model->n_sites;
    for (auto &st : I->states)
      for (int sd = 0; sd < ((I->mix & mixing::up_down) ? 2 : 1); ++sd) {
        State *sp = st.get();
        const double cost = (double)I->sector_dim(sp->sec) * p;
        if (I->use_cf) {
          tasks.push_back({cost * p, [I, sp, sd] { I->build_cf(*sp, sd != 0, ws()); }});
          continue;
        }
        if (I->use_mcf) {
          tasks.push_back({cost * p, [I, sp, sd] { I->build_mcf(*sp, sd != 0, ws()); }});
          continue;
        }
        jobs.emplace_back(new Job{I, sp, sd != 0, {}});
        Job *j = jobs.back().get();
        for (int s = 0; s < 2; ++s)
          tasks.push_back({cost, [j, s] { j->I->qmatrix_part(*j->st, j->sd, s, j->parts[s], ws()); }});
      }
  }
  if ((rc = run_tasks(tasks, threads)) != QED_OK) return rc;
  return guarded([&] {
    for (auto &j : jobs) j->I->qmatrix_combine(*j->st, j->sd, j->parts, ws());
    for (Instance *I : todo) I->finish_gf();
  });
}

}  // namespace

extern "C" {

int qed_last_error(char *buf, int len) {
  if (buf && len > 0) {
    std::strncpy(buf, t_err.c_str(), (size_t)len - 1);
    buf[len - 1] = 0;
  }
  return (int)t_err.size();
}

int qed_hv_tuning_report(char *buf, int len) {
  const std::string r = hv_tuning_report();
  if (buf && len > 0) {
    std::strncpy(buf, r.c_str(), (size_t)len - 1);
    buf[len - 1] = 0;
  }
  return (int)r.size();
}

namespace {
std::vector<uint32_t> all_strings(int L, int N) {
  if (L < 1 || L > 24 || N < 0 || N > L) fail(QED_ERR_ARGUMENT, "window diagnostics: L in [1, 24], N in [0, L]");
  std::vector<uint32_t> b;
  for (uint32_t s = 0; s < (1u << L); ++s)
    if (__builtin_popcount(s) == N) b.push_back(s);
  return b;
}
}  // namespace

int qed_window_plan(int L, int N, int npairs, const int *pd, const int *ps, const double *amp, const double *x,
                    double *y, int *nwindows) {
  return guarded([&] {
    if (npairs < 0 || !nwindows) fail(QED_ERR_ARGUMENT, "qed_window_plan: bad arguments");
    const std::vector<uint32_t> bits = all_strings(L, N);
    WindowPlan P;
    *nwindows = 0;
    if (!plan_windows(L, N, bits, std::vector<int>(pd, pd + npairs), std::vector<int>(ps, ps + npairs), P)) return;
    *nwindows = (int)P.win.size();
    window_apply_host(P, std::vector<double>(amp, amp + npairs), x, y);
  });
}

int qed_window_compile(int L, int n_up, int n_dn, int npairs, const int *pd, const int *ps, char *buf, int len,
                       int *ok) {
  return guarded([&] {
    if (npairs < 0 || !ok) fail(QED_ERR_ARGUMENT, "qed_window_compile: bad arguments");
    const std::vector<int> vd(pd, pd + npairs), vs(ps, ps + npairs);
    WindowPlan pu, pdn;
    if (!plan_windows(L, n_up, all_strings(L, n_up), vd, vs, pu) ||
        !plan_windows(L, n_dn, all_strings(L, n_dn), vd, vs, pdn))
      fail(QED_ERR_UNSUPPORTED, "qed_window_compile: the pairs do not fit windows");
    bool good = false;
    const std::string log = window_compile_log(pu, pdn, &good);
    *ok = good ? 1 : 0;
    if (buf && len > 0) {
      std::strncpy(buf, log.c_str(), (size_t)len - 1);
      buf[len - 1] = 0;
    }
  });
}

int qed_window_launches(long long *n) {
  return guarded([&] {
    if (!n) fail(QED_ERR_ARGUMENT, "qed_window_launches: null pointer");
    *n = window_launches();
  });
}

int qed_spin_table_host(int L, int N, const double *t, const double *vsame, int bank_order, unsigned *bits,
                        unsigned char *cnt, double *diag, unsigned *ell, long ell_capacity, int *width,
                        double *vals, int *nvals) {
  return guarded([&] {
    if (L < 1 || L > 24 || N < 0 || N > L || !t || !vsame || !width || !nvals)
      fail(QED_ERR_ARGUMENT, "qed_spin_table_host: L in [1, 24], N in [0, L], non-null t, vsame, width, nvals");
    const std::vector<double> tv(t, t + (size_t)L * L), vs(vsame, vsame + (size_t)L * L);
    std::vector<int> pd, ps, pslot;
    std::vector<double> vl;
    hop_pairs(L, tv, pd, ps, pslot, vl);
    if (vl.size() > 256) fail(QED_ERR_UNSUPPORTED, "more than 128 distinct hopping amplitudes per spin");
    const int w = std::min<int>((int)pd.size(), N * (L - N));
    std::vector<double> tdiag(L);
    for (int r = 0; r < L; ++r) tdiag[r] = tv[(size_t)r * L + r];
    const uint32_t dim = (uint32_t)binom(L, N);
    const HostHalf T = host_half_tables(L, N, dim, tdiag, vs, pd, ps, pslot, vl, w, bank_order != 0);
    if ((long)T.ell.size() > ell_capacity) fail(QED_ERR_ARGUMENT, "qed_spin_table_host: ell_capacity too small");
    std::copy(T.bits.begin(), T.bits.end(), bits);
    std::copy(T.cnt.begin(), T.cnt.end(), cnt);
    std::copy(T.diag.begin(), T.diag.end(), diag);
    std::copy(T.ell.begin(), T.ell.end(), ell);
    std::copy(T.vals.begin(), T.vals.end(), vals);
    *width = T.width;
    *nvals = (int)T.vals.size();
  });
}

int qed_init(int device) {
  return guarded([&] {
    if (g_device_fixed && device != g_device) fail(QED_ERR_ARGUMENT, "qed_init: device already selected");
    g_device = device;
    ws();
  });
}

int qed_set_global_int(const char *name, long v) { return guarded([&] { set_opt_int(name, v); }); }
int qed_set_global_double(const char *name, double v) { return guarded([&] { set_opt_double(name, v); }); }
int qed_set_global_char(const char *name, char v) { return guarded([&] { set_opt_char(name, v); }); }
int qed_set_global_bool(const char *name, int v) { return guarded([&] { set_opt_bool(name, v != 0); }); }
int qed_get_global_double(const char *name, double *v) { return guarded([&] { *v = opt_double(name); }); }

int qed_new_model(const char *name, int n_sites, int n_bath) {
  return guarded([&] {
    // ED::new_model (src_ed/qcm_ED.cpp:46-60)
    if (n_bath > 32 || n_bath < 0) fail(QED_ERR_ARGUMENT, "number of bath orbitals exceeds limits or negative!");
    if (n_sites > 1024 || n_sites < 1) fail(QED_ERR_ARGUMENT, "number of cluster sites  exceeds limits or negative!");
    std::lock_guard<std::mutex> l(g_reg);
    if (g_models.count(name)) return;  // reused, as the reference does (with a warning)
    auto m = std::make_shared<Model>();
    m->name = name;
    m->n_sites = n_sites;
    m->n_bath = n_bath;
    m->n_orb = n_sites + n_bath;
    if (m->n_orb > 32) fail(QED_ERR_UNSUPPORTED, "more than 32 orbitals per spin");
    m->in_bath.assign(2 * m->n_orb, false);
    for (int i = n_sites; i < m->n_orb; ++i) m->in_bath[i] = m->in_bath[i + m->n_orb] = true;
    g_models[name] = m;
  });
}

int qed_new_model_generators(const char *name, int n_sites, int n_bath, int n_gen, const int *gen, int bath_irrep) {
  return guarded([&] {
    // ED::new_model with generators (src_ed/qcm_ED.cpp:46-60, symmetry_group ctor)
    std::vector<std::vector<int>> g(n_gen < 0 ? 0 : n_gen, std::vector<int>(n_sites + n_bath));
    if (n_gen > 0 && !gen) fail(QED_ERR_ARGUMENT, "bad generators");
    for (int j = 0; j < n_gen; ++j)
      for (int i = 0; i < n_sites + n_bath; ++i) g[j][i] = gen[(size_t)j * (n_sites + n_bath) + i];
    auto grp = std::make_shared<const SymmetryGroup>(build_symmetry_group(n_sites, n_bath, g, bath_irrep != 0));
    const int rc = qed_new_model(name, n_sites, n_bath);
    if (rc != QED_OK) fail(rc, t_err);
    std::lock_guard<std::mutex> l(g_reg);
    auto &m = g_models.at(name);
    std::lock_guard<std::mutex> lm(m->mtx);
    if (!m->group && m->term.empty() && grp->g() > 1) m->group = grp;
  });
}

int qed_new_operator(const char *model, const char *name, const char *type, int n, const int *r,
                     const int *c, const double *v) {
  return guarded([&] {
    if (n <= 0) return;  // ED::new_operator ignores empty element lists
    std::shared_ptr<Model> m;
    {
      std::lock_guard<std::mutex> l(g_reg);
      auto it = g_models.find(model);
      if (it == g_models.end())
        fail(QED_ERR_ARGUMENT, std::string("The model ") + model + " is not defined. Check spelling.");
      m = it->second;
    }
    std::vector<Element> el(n);
    for (int k = 0; k < n; ++k) el[k] = {r[k], c[k], v[k]};
    auto op = make_operator(*m, name, type, el);
    std::lock_guard<std::mutex> l(m->mtx);
    if (m->is_closed) return;  // closed for modifications (warning in the reference)
    m->term[name] = op;
  });
}

int qed_new_model_instance(const char *model, int n, const char **names, const double *values,
                           const char *sectors, int label) {
  return guarded([&] {
    std::shared_ptr<Model> m;
    {
      std::lock_guard<std::mutex> l(g_reg);
      auto it = g_models.find(model);
      if (it == g_models.end())
        fail(QED_ERR_ARGUMENT, std::string("The model ") + model +
                                   " is not defined and so no model instance based on it is allowed.");
      m = it->second;
      g_instances.erase(label);
    }
    std::map<std::string, double> param;
    {
      std::lock_guard<std::mutex> l(m->mtx);
      m->is_closed = true;
      for (int k = 0; k < n; ++k)  // values of undefined operators are dropped (src_ed/qcm_ED.cpp:137-145)
        if (m->term.count(names[k])) param[names[k]] = values[k];
    }
    auto inst = std::make_shared<Instance>(label, m, param, sectors);
    std::lock_guard<std::mutex> l(g_reg);
    g_instances[label] = inst;
  });
}

int qed_erase_model_instance(int label) {
  return guarded([&] {
    std::shared_ptr<Instance> keep;
    {
      std::lock_guard<std::mutex> l(g_reg);
      auto it = g_instances.find(label);
      if (it == g_instances.end()) return;
      keep = it->second;
      g_instances.erase(it);
    }
    ws();
    keep.reset();
  });
}

int qed_mixing(int label, int *mixing) {
  return guarded([&] { *mixing = instance(label)->mix; });
}

int qed_ground_state_solve(int label, double *energy, char *sectors, int len) {
  return guarded([&] {
    auto I = instance(label);
    I->require_supported_group();
    std::lock_guard<std::mutex> li(I->mtx);
    auto r = I->low_energy_states(ws());
    *energy = r.first;
    if (sectors && len > 0) {
      std::strncpy(sectors, r.second.c_str(), (size_t)len - 1);
      sectors[len - 1] = 0;
    }
  });
}


int qed_ground_state_solve_batch(const int *labels, int n, int threads, double *energies) {
  if (n > 0 && (!labels || !energies)) {
    t_err = "null argument";
    return QED_ERR_ARGUMENT;
  }
  std::unique_ptr<BatchSet> b;
  int rc = guarded([&] { b.reset(new BatchSet(labels, n)); });
  if (rc != QED_OK) return rc;
  if ((rc = batch_ground_states(*b, threads)) != QED_OK) return rc;
  return guarded([&] {
    for (int i = 0; i < n; ++i) energies[i] = instance(labels[i])->GS_energy;
  });
}

int qed_Green_function_solve_batch(const int *labels, int n, int threads) {
  if (n > 0 && !labels) {
    t_err = "null argument";
    return QED_ERR_ARGUMENT;
  }
  std::unique_ptr<BatchSet> b;
  int rc = guarded([&] { b.reset(new BatchSet(labels, n)); });
  if (rc != QED_OK) return rc;
  return batch_green_functions(*b, threads);
}

}  // extern "C"

namespace {

// The asynchronous batch queue: one background thread per submitted batch.
struct AsyncBatch {
  std::thread th;
  std::mutex m;
  std::condition_variable cv;
  bool done = false;
  int status = QED_OK;
  std::string msg;
};

struct AsyncBatches {
  std::mutex m;
  long long next = 1;
  std::map<long long, std::shared_ptr<AsyncBatch>> jobs;
  ~AsyncBatches() {  // batches still running at exit finish first
    for (auto &j : jobs)
      if (j.second->th.joinable()) j.second->th.join();
  }
};

AsyncBatches &async_batches() {
  static AsyncBatches b;
  return b;
}

// *done and the batch's status once it has finished (the ticket is then released)
int async_result(long long ticket, int timeout_ms, int *done) {
  if (!done) {
    t_err = "null argument";
    return QED_ERR_ARGUMENT;
  }
  std::shared_ptr<AsyncBatch> job;
  {
    std::lock_guard<std::mutex> l(async_batches().m);
    auto it = async_batches().jobs.find(ticket);
    if (it == async_batches().jobs.end()) {
      t_err = "unknown batch ticket " + std::to_string(ticket);
      return QED_ERR_ARGUMENT;
    }
    job = it->second;
  }
  {
    std::unique_lock<std::mutex> l(job->m);
    if (timeout_ms < 0) job->cv.wait(l, [&] { return job->done; });
    else if (timeout_ms > 0) job->cv.wait_for(l, std::chrono::milliseconds(timeout_ms), [&] { return job->done; });
    *done = job->done ? 1 : 0;
    if (!job->done) return QED_OK;
  }
  job->th.join();
  {
    std::lock_guard<std::mutex> l(async_batches().m);
    async_batches().jobs.erase(ticket);
  }
  if (job->status != QED_OK) t_err = job->msg;
  return job->status;
}

}  // namespace

extern "C" {

int qed_batch_submit(const int *labels, int n, int what, int threads, long long *ticket) {
  if ((n > 0 && !labels) || !ticket) {
    t_err = "null argument";
    return QED_ERR_ARGUMENT;
  }
  if (what != QED_BATCH_GROUND_STATE && what != QED_BATCH_GREEN_FUNCTION) {
    t_err = "qed_batch_submit: what must be QED_BATCH_GROUND_STATE or QED_BATCH_GREEN_FUNCTION";
    return QED_ERR_ARGUMENT;
  }
  std::vector<int> lab(labels, labels + std::max(n, 0));
  for (int x : lab)  // unknown labels fail here, before anything runs
    if (int rc = guarded([&] { instance(x); }); rc != QED_OK) return rc;
  auto job = std::make_shared<AsyncBatch>();
  std::lock_guard<std::mutex> l(async_batches().m);
  const long long t = async_batches().next++;
  job->th = std::thread([job, lab, what, threads] {
    int rc;
    if (what == QED_BATCH_GROUND_STATE) {
      std::vector<double> e(lab.size());
      rc = qed_ground_state_solve_batch(lab.data(), (int)lab.size(), threads, e.data());
    } else {
      rc = qed_Green_function_solve_batch(lab.data(), (int)lab.size(), threads);
    }
    std::lock_guard<std::mutex> lj(job->m);
    job->status = rc;
    if (rc != QED_OK) job->msg = t_err;
    job->done = true;
    job->cv.notify_all();
  });
  async_batches().jobs[t] = job;
  *ticket = t;
  return QED_OK;
}

int qed_batch_poll(long long ticket, int *done) { return async_result(ticket, 0, done); }

int qed_batch_wait(long long ticket, int timeout_ms, int *done) { return async_result(ticket, timeout_ms, done); }

int qed_Green_function_solve(int label) {
  return guarded([&] {
    auto I = instance(label);
    I->require_supported_group();
    std::lock_guard<std::mutex> li(I->mtx);
    I->green_solve(ws());
  });
}

int qed_Green_function_dimension(int label, int *dim) {
  return guarded([&] { *dim = instance(label)->dim_GF; });
}

int qed_Green_function(int label, int spin_down, int nz, const double *z, double *G) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    I->green_function(reinterpret_cast<const cplx *>(z), nz, spin_down != 0, reinterpret_cast<cplx *>(G), ws());
  });
}

int qed_sef_integrand_grid(int label, int spin_down, int dim, const double *V0, int nel, const int *r, const int *c,
                           const int *R, const double *v, int nw, const double *w, int nkx, int nky, int nkz,
                           double *I_w) {
  return guarded([&] {
    if (nw < 0 || nel < 0 || nkx < 1 || nky < 1 || nkz < 1) fail(QED_ERR_ARGUMENT, "qed_sef_integrand_grid: bad sizes");
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    if (dim != I->model->n_sites)
      fail(QED_ERR_ARGUMENT, "qed_sef_integrand_grid: dim differs from the cluster's Green function dimension");
    for (int e = 0; e < nel; ++e)
      if (r[e] < 0 || r[e] >= dim || c[e] < 0 || c[e] >= dim)
        fail(QED_ERR_ARGUMENT, "qed_sef_integrand_grid: element index outside the Green function");
    if (nw == 0) return;
    Workspace &W = ws();
    std::vector<cplx> z(nw);
    for (int i = 0; i < nw; ++i) z[i] = cplx(0.0, w[i]);
    const size_t nn = (size_t)dim * dim;
    DevBuf<double> dG(2 * nn * nw), dV0(2 * nn), dR(3 * (size_t)std::max(nel, 1)), dv(2 * (size_t)std::max(nel, 1));
    DevBuf<int> dr(std::max(nel, 1)), dc(std::max(nel, 1));
    I->green_function_device(z.data(), nw, spin_down != 0, dG.p, W);
    dV0.upload(V0, 2 * nn, W.stream);
    if (nel) {
      std::vector<double> Rd(3 * (size_t)nel);
      for (size_t i = 0; i < Rd.size(); ++i) Rd[i] = (double)R[i];
      dR.upload(Rd, W.stream);
      dv.upload(v, 2 * (size_t)nel, W.stream);
      dr.upload(r, nel, W.stream);
      dc.upload(c, nel, W.stream);
    }
    const long nk = (long)nkx * nky * nkz;
    const int nblk = (int)((nk + 127) / 128);
    DevBuf<double> part((size_t)nblk * nw);
    const int nb = launch_sef_logdet(dim, nw, dG.p, dV0.p, nel, dr.p, dc.p, dR.p, dv.p, nkx, nky, nkz, part.p, W.stream);
    if (nb != nblk) fail(QED_ERR_INTERNAL, "qed_sef_integrand_grid: block count mismatch");
    std::vector<double> h((size_t)nblk * nw);
    part.download(h.data(), h.size(), W.stream);
    W.sync();
    for (int i = 0; i < nw; ++i) {
      double s = 0.0;
      for (int b = 0; b < nblk; ++b) s += h[(size_t)i * nblk + b];
      I_w[i] = s / (double)nk;
    }
  });
}

int qed_cpt_projected_green_function(int label, int spin_down, int dim, const double *V0, int nel, const int *r,
                                     const int *c, const int *R, const double *v, int nw, const double *w,
                                     int nkx, int nky, int nkz, double offset, double *Gproj) {
  return guarded([&] {
    if (nw < 0 || nel < 0 || nkx < 1 || nky < 1 || nkz < 1)
      fail(QED_ERR_ARGUMENT, "qed_cpt_projected_green_function: bad sizes");
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    if (dim != I->model->n_sites)
      fail(QED_ERR_ARGUMENT, "qed_cpt_projected_green_function: dim differs from the cluster's Green function dimension");
    for (int e = 0; e < nel; ++e)
      if (r[e] < 0 || r[e] >= dim || c[e] < 0 || c[e] >= dim)
        fail(QED_ERR_ARGUMENT, "qed_cpt_projected_green_function: element index outside the Green function");
    if (nw == 0) return;
    Workspace &W = ws();
    std::vector<cplx> z(nw);
    for (int i = 0; i < nw; ++i) z[i] = cplx(0.0, w[i]);
    const size_t nn = (size_t)dim * dim;
    DevBuf<double> dG(2 * nn * nw), dV0(2 * nn * nw), dR(3 * (size_t)std::max(nel, 1)),
        dv(2 * (size_t)std::max(nel, 1)), part((size_t)cpt_partials_size(dim, nw)), dP(2 * nn * nw);
    DevBuf<int> dr(std::max(nel, 1)), dc(std::max(nel, 1));
    I->green_function_device(z.data(), nw, spin_down != 0, dG.p, W);
    dV0.upload(V0, 2 * nn * nw, W.stream);
    if (nel) {
      std::vector<double> Rd(3 * (size_t)nel);
      for (size_t i = 0; i < Rd.size(); ++i) Rd[i] = (double)R[i];
      dR.upload(Rd, W.stream);
      dv.upload(v, 2 * (size_t)nel, W.stream);
      dr.upload(r, nel, W.stream);
      dc.upload(c, nel, W.stream);
    }
    launch_cpt_projected(dim, nw, dG.p, dV0.p, nel, dr.p, dc.p, dR.p, dv.p, nkx, nky, nkz, offset, part.p, dP.p,
                         W.stream);
    dP.download(Gproj, 2 * nn * nw, W.stream);
    W.sync();
  });
}

int qed_self_energy(int label, int spin_down, int nz, const double *z, double *S) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    I->self_energy(reinterpret_cast<const cplx *>(z), nz, spin_down != 0, reinterpret_cast<cplx *>(S), ws());
  });
}

int qed_hybridization_function(int label, int spin_down, int nz, const double *z, double *H) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    I->hybridization(reinterpret_cast<const cplx *>(z), nz, spin_down != 0, reinterpret_cast<cplx *>(H));
  });
}

int qed_Green_function_average(int label, int spin_down, double *M) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    I->green_solve(ws());
    const int sd = (spin_down && (I->mix & mixing::up_down)) ? 1 : 0;
    const auto &src = I->is_correlated ? I->Mave[sd] : I->Mfull[sd];
    std::memcpy(M, src.data(), src.size() * sizeof(cplx));
  });
}

int qed_Green_function_average_dimension(int label, int *d) {
  return guarded([&] {
    auto I = instance(label);
    *d = I->is_correlated ? I->dim_GF : I->model->n_orb;
  });
}

int qed_cluster_averages(int label, int cap, int *n, double *ave, double *var, char *names, int names_size) {
  return guarded([&] {
    if (!n || !ave || !var || !names) fail(QED_ERR_ARGUMENT, "null argument");
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    I->low_energy_states(ws());
    const auto &a = I->averages;
    if ((int)a.size() > cap) fail(QED_ERR_ARGUMENT, "qed_cluster_averages: capacity too small");
    std::string all;
    for (size_t i = 0; i < a.size(); ++i) {
      ave[i] = std::get<1>(a[i]);
      var[i] = std::get<2>(a[i]);
      all += std::get<0>(a[i]);
      all += '\n';
    }
    if ((int)all.size() + 1 > names_size) fail(QED_ERR_ARGUMENT, "qed_cluster_averages: name buffer too small");
    std::memcpy(names, all.c_str(), all.size() + 1);
    *n = (int)a.size();
  });
}

int qed_model_size(const char *model, int *n_sites, int *n_bath, int *n_elements) {
  return guarded([&] {
    std::shared_ptr<Model> m;
    {
      std::lock_guard<std::mutex> l(g_reg);
      auto it = g_models.find(model ? model : "");
      if (it == g_models.end()) fail(QED_ERR_ARGUMENT, "model " + std::string(model ? model : "") + " does not exist!");
      m = it->second;
    }
    *n_sites = m->n_sites;
    *n_bath = m->n_bath;
    *n_elements = 1;
  });
}

int qed_operator_exists(const char *model, const char *op, int *found) {
  return guarded([&] {
    std::lock_guard<std::mutex> l(g_reg);
    auto it = g_models.find(model ? model : "");
    if (it == g_models.end()) fail(QED_ERR_ARGUMENT, "model " + std::string(model ? model : "") + " does not exist!");
    *found = it->second->term.count(op ? op : "") ? 1 : 0;
  });
}

int qed_matrix_elements(const char *model, const char *op, char *type, int type_size, int cap, int *n, int *r,
                        int *c, double *v) {
  return guarded([&] {
    std::shared_ptr<Operator> o;
    {
      std::lock_guard<std::mutex> l(g_reg);
      auto it = g_models.find(model ? model : "");
      if (it == g_models.end())
        fail(QED_ERR_ARGUMENT, "The model " + std::string(model ? model : "") + " is not defined. Check spelling.");
      auto jt = it->second->term.find(op ? op : "");
      if (jt == it->second->term.end())
        fail(QED_ERR_ARGUMENT, "operator " + std::string(op ? op : "") + " is not defined in model . Check spelling.");
      o = jt->second;
    }
    const std::string t = o->is_interaction ? "interaction" : "one_body";
    if ((int)t.size() + 1 > type_size || (int)o->elements.size() > cap)
      fail(QED_ERR_ARGUMENT, "qed_matrix_elements: buffer too small");
    std::memcpy(type, t.c_str(), t.size() + 1);
    for (size_t i = 0; i < o->elements.size(); ++i) {
      r[i] = o->elements[i].r;
      c[i] = o->elements[i].c;
      v[i] = o->elements[i].v;
    }
    *n = (int)o->elements.size();
  });
}

int qed_complex_HS(int label, int *flag) {
  return guarded([&] {
    instance(label);
    *flag = 0;
  });
}

int qed_Green_function_density(int label, double *density) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    *density = I->GF_density;
  });
}

namespace {
void put_real_as_complex(const std::vector<double> &h, double *out) {
  for (size_t i = 0; i < h.size(); ++i) {
    out[2 * i] = h[i];
    out[2 * i + 1] = 0.0;
  }
}
}  // namespace

int qed_hopping_matrix(int label, int spin_down, double *H) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    put_real_as_complex(I->hopping_matrix(spin_down != 0), H);
  });
}

int qed_hopping_matrix_full(int label, int spin_down, int diag, int *d, double *H) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    *d = I->model->n_orb;
    if (H) put_real_as_complex(I->hopping_matrix_full(spin_down != 0, diag != 0), H);
  });
}

int qed_interactions(int label, int cap, int *n, int *r, int *c, double *v) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    const auto V = I->interactions();
    if ((int)V.size() > cap) fail(QED_ERR_ARGUMENT, "qed_interactions: capacity too small");
    for (size_t i = 0; i < V.size(); ++i) {
      r[i] = V[i].r;
      c[i] = V[i].c;
      v[i] = V[i].v;
    }
    *n = (int)V.size();
  });
}

int qed_tr_sigma_inf(int label, double *value) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    *value = I->tr_sigma_inf(ws());
  });
}

int qed_susceptibility(int label, const char *op, int nw, const double *w, double *chi) {
  return guarded([&] {
    if (!op || (nw > 0 && (!w || !chi))) fail(QED_ERR_ARGUMENT, "null argument");
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    I->susceptibility(op, reinterpret_cast<const cplx *>(w), nw, reinterpret_cast<cplx *>(chi), ws());
  });
}

int qed_susceptibility_poles(int label, const char *op, int cap, int *n, double *e, double *r) {
  return guarded([&] {
    if (!op || !n || !e || !r) fail(QED_ERR_ARGUMENT, "null argument");
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    const auto p = I->susceptibility_poles(op, ws());
    if ((int)p.size() > cap) fail(QED_ERR_ARGUMENT, "qed_susceptibility_poles: capacity too small");
    for (size_t i = 0; i < p.size(); ++i) {
      e[i] = p[i].first;
      r[i] = p[i].second;
    }
    *n = (int)p.size();
  });
}

int qed_fidelity(int label1, int label2, double *fidelity) {
  return guarded([&] {
    if (!fidelity) fail(QED_ERR_ARGUMENT, "null argument");
    auto I1 = instance(label1), I2 = instance(label2);
    // both instances locked, in label order
    std::unique_lock<std::mutex> la, lb;
    if (I1 == I2) {
      la = std::unique_lock<std::mutex>(I1->mtx);
    } else {
      Instance *first = label1 < label2 ? I1.get() : I2.get(), *second = label1 < label2 ? I2.get() : I1.get();
      la = std::unique_lock<std::mutex>(first->mtx);
      lb = std::unique_lock<std::mutex>(second->mtx);
    }
    Workspace &w = ws();
    I1->low_energy_states(w);
    I2->low_energy_states(w);
    double z = 0.0;
    for (auto &s1 : I1->states)
      for (auto &s2 : I2->states) {
        if (!(s1->sec == s2->sec) || s1->psi.n != s2->psi.n || s1->psi.n == 0) continue;
        VecList one;
        one.n = 1;
        one.v[0] = s2->psi.p;
        const int nb = launch_dots(s1->psi.n, s1->psi.p, 1.0, 0, one, w.red, w.stream);
        const double zz = w.sums(nb, 1)[0];
        z += zz * zz * s1->weight * s2->weight;
      }
    *fidelity = z;
  });
}

int qed_Potthoff_functional(int label, double *omega) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    *omega = I->potthoff(ws());
  });
}

int qed_qmatrix(int label, int spin_down, int *M, int *L, double *e, double *v) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    if (I->use_cf || I->use_mcf)
      fail(QED_ERR_ARGUMENT, "Green function format is not Lehmann! Cannot output the Q matrix.");
    {
      I->green_solve(ws());
    }
    // model_instance::qmatrix (src_ed/model_instance.hpp:1425-1451): one state
    // as is; several states appended, each scaled by sqrt(weight) once more.
    const int sd = spin_down ? 1 : 0;
    std::vector<double> ee, vv;
    int l = I->dim_GF;
    for (auto &st : I->states) {
      const QMat &q = st->q[sd];
      double sc = I->states.size() > 1 ? std::sqrt(st->weight) : 1.0;
      ee.insert(ee.end(), q.e.begin(), q.e.end());
      for (double x : q.V) vv.push_back(x * sc);
    }
    int m = (int)ee.size();
    if (m > *M) fail(QED_ERR_ARGUMENT, "qed_qmatrix: capacity too small (" + std::to_string(m) + " poles)");
    *M = m;
    *L = l;
    for (int i = 0; i < m; ++i) e[i] = ee[i];
    for (size_t i = 0; i < vv.size(); ++i) {
      v[2 * i] = vv[i];
      v[2 * i + 1] = 0.0;
    }
  });
}

int qed_cf_coefficients(int label, int spin_down, int o1, int o2, int pm, int *n, double *a, double *b) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    if (!I->use_cf) fail(QED_ERR_ARGUMENT, "not a continued-fraction instance");
    {
      I->green_solve(ws());
    }
    const CFSet &cf = I->states.front()->cf[spin_down ? 1 : 0];
    if (o1 < 0 || o2 < 0 || o2 > o1 || o1 >= cf.n) fail(QED_ERR_ARGUMENT, "bad orbital pair");
    size_t idx = (size_t)o1 * cf.n + o2;
    const auto &A = pm > 0 ? cf.ea[idx] : cf.ha[idx];
    const auto &B = pm > 0 ? cf.eb[idx] : cf.hb[idx];
    if ((int)A.size() > *n) fail(QED_ERR_ARGUMENT, "capacity too small");
    *n = (int)A.size();
    for (size_t i = 0; i < A.size(); ++i) a[i] = A[i];
    for (size_t i = 0; i < A.size() && i < B.size(); ++i) b[i] = B[i];
  });
}

// ---- instance checkpoints (model_instance::write_hdf5 / read_hdf5,
// src_ed/model_instance.hpp:1339-1421; the file itself is written by the caller)

int qed_instance_states(int label, int *n_states, double *gs_energy, char *gs_sectors, int len, int *gf_format,
                        int *mixing) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    if (I->has_group()) fail(QED_ERR_UNSUPPORTED, "checkpoints of models with a point group are not supported");
    I->green_solve(ws());  // write_hdf5 solves the Green function first
    *n_states = (int)I->states.size();
    *gs_energy = I->GS_energy;
    const std::string g = I->gs_string();
    if (gs_sectors && len > 0) {
      std::strncpy(gs_sectors, g.c_str(), (size_t)len - 1);
      gs_sectors[len - 1] = 0;
    }
    *gf_format = I->use_cf ? 1 : I->use_mcf ? 2 : 0;
    *mixing = I->mix;
  });
}

int qed_instance_parameters(int label, int cap, int *n, char *names, int names_size, double *values) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    *n = (int)I->value.size();
    if (*n > cap) fail(QED_ERR_ARGUMENT, "qed_instance_parameters: capacity too small");
    std::string all;
    int k = 0;
    for (auto &kv : I->value) {
      all += kv.first + '\n';
      values[k++] = kv.second;
    }
    if ((int)all.size() + 1 > names_size) fail(QED_ERR_ARGUMENT, "qed_instance_parameters: name buffer too small");
    std::memcpy(names, all.c_str(), all.size() + 1);
  });
}

int qed_instance_state(int label, int i, char *sector, int len, double *energy, double *weight) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    if (i < 0 || i >= (int)I->states.size()) fail(QED_ERR_ARGUMENT, "state index out of range");
    const State &st = *I->states[i];
    std::strncpy(sector, st.sec.name().c_str(), (size_t)len - 1);
    sector[len - 1] = 0;
    *energy = st.energy;
    *weight = st.weight;
  });
}

int qed_instance_state_qmatrix(int label, int i, int spin_down, int cap, int *L, int *M, double *e, double *v) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    if (i < 0 || i >= (int)I->states.size()) fail(QED_ERR_ARGUMENT, "state index out of range");
    if (I->use_cf || I->use_mcf) fail(QED_ERR_ARGUMENT, "the instance's Green function is not a Q-matrix");
    const QMat &q = I->states[i]->q[spin_down ? 1 : 0];
    *L = q.L;
    *M = q.M;
    if (!e) return;  // sizes only
    if (q.M > cap) fail(QED_ERR_ARGUMENT, "qed_instance_state_qmatrix: capacity too small");
    std::copy(q.e.begin(), q.e.end(), e);
    std::copy(q.V.begin(), q.V.end(), v);
  });
}

int qed_instance_state_cf(int label, int i, int spin_down, int o1, int o2, int pm, int cap, int *n, double *a,
                          double *b) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    if (i < 0 || i >= (int)I->states.size()) fail(QED_ERR_ARGUMENT, "state index out of range");
    if (!I->use_cf) fail(QED_ERR_ARGUMENT, "not a continued-fraction instance");
    const CFSet &cf = I->states[i]->cf[spin_down ? 1 : 0];
    if (o1 < 0 || o2 < 0 || o2 > o1 || o1 >= cf.n) fail(QED_ERR_ARGUMENT, "bad orbital pair");
    const size_t idx = (size_t)o1 * cf.n + o2;
    const auto &A = pm > 0 ? cf.ea[idx] : cf.ha[idx];
    const auto &B = pm > 0 ? cf.eb[idx] : cf.hb[idx];
    *n = (int)A.size();
    if (!a) return;
    if ((int)A.size() > cap) fail(QED_ERR_ARGUMENT, "qed_instance_state_cf: capacity too small");
    std::copy(A.begin(), A.end(), a);
    for (size_t k = 0; k < A.size(); ++k) b[k] = k < B.size() ? B[k] : 0.0;
  });
}

int qed_instance_load_begin(int label, double gs_energy, int gf_format, int mixing) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    if (I->has_group()) fail(QED_ERR_UNSUPPORTED, "checkpoints of models with a point group are not supported");
    if (gf_format == 2) fail(QED_ERR_UNSUPPORTED, "matrix continued-fraction checkpoints are not supported");
    if (gf_format != 0 && gf_format != 1) fail(QED_ERR_ARGUMENT, "unknown Green-function format");
    I->states.clear();
    I->use_cf = gf_format == 1;
    I->use_mcf = false;
    I->mix = mixing;
    I->GS_energy = gs_energy;
    I->gs_solved = false;
    I->gf_solved = false;
  });
}

int qed_instance_load_state(int label, const char *sector, double energy, double weight, int *index) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    auto st = std::make_shared<State>();
    st->sec = Sector(sector);
    st->energy = energy;
    st->weight = weight;
    const int n = I->model->n_sites;
    for (auto &c : st->cf) {
      c.n = n;
      c.ea.assign((size_t)n * n, {});
      c.eb.assign((size_t)n * n, {});
      c.ha.assign((size_t)n * n, {});
      c.hb.assign((size_t)n * n, {});
    }
    I->states.push_back(st);
    *index = (int)I->states.size() - 1;
  });
}

int qed_instance_load_qmatrix(int label, int i, int spin_down, int L, int M, const double *e, const double *v) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    if (i < 0 || i >= (int)I->states.size()) fail(QED_ERR_ARGUMENT, "state index out of range");
    if (L != I->model->n_sites) fail(QED_ERR_ARGUMENT, "Q-matrix with " + std::to_string(L) + " rows for " +
                                                          std::to_string(I->model->n_sites) + " cluster sites");
    QMat &q = I->states[i]->q[spin_down ? 1 : 0];
    q.L = L;
    q.M = M;
    q.e.assign(e, e + M);
    q.V.assign(v, v + (size_t)L * M);
  });
}

int qed_instance_load_cf(int label, int i, int spin_down, int o1, int o2, int pm, int n, const double *a,
                         const double *b) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    if (i < 0 || i >= (int)I->states.size()) fail(QED_ERR_ARGUMENT, "state index out of range");
    CFSet &cf = I->states[i]->cf[spin_down ? 1 : 0];
    if (o1 < 0 || o2 < 0 || o2 > o1 || o1 >= cf.n) fail(QED_ERR_ARGUMENT, "bad orbital pair");
    const size_t idx = (size_t)o1 * cf.n + o2;
    (pm > 0 ? cf.ea : cf.ha)[idx].assign(a, a + n);
    (pm > 0 ? cf.eb : cf.hb)[idx].assign(b, b + n);
  });
}

int qed_instance_load_end(int label) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    if (I->states.empty()) fail(QED_ERR_ARGUMENT, "a checkpoint without states");
    I->E0 = 0.0;
    for (auto &st : I->states) {
      I->E0 += st->weight * st->energy;
      for (int sd = 0; sd < 2; ++sd) {
        QMat &q = st->q[sd];
        if (q.M > 0) {
          q.de.upload(q.e, ws().stream);
          q.dV.upload(q.V, ws().stream);
        }
      }
    }
    ws().sync();
    I->is_correlated = true;
    I->gs_solved = true;
    I->finish_gf();  // gf_solved, Green_function_average, Green_function_density
  });
}

int qed_ground_state_vector(int label, long *dim, double *psi) {
  return guarded([&] {
    auto I = instance(label);
    std::lock_guard<std::mutex> li(I->mtx);
    I->low_energy_states(ws());
    const State &st = *I->states.front();
    *dim = (long)st.psi.n;
    if (psi) {
      st.psi.download(psi, st.psi.n, ws().stream);
      ws().sync();
    }
  });
}

int qed_hamiltonian_create(int label, const char *sector, qed_hamiltonian **h, long *dim) {
  return guarded([&] {
    auto I = instance(label);
    auto *hh = new qed_hamiltonian;
    try {
      hh->H.reset(new SectorOp(I->terms, Sector(sector), ws()));
    } catch (...) {
      delete hh;
      throw;
    }
    *dim = (long)hh->H->D;
    *h = hh;
  });
}

// y += H x with host vectors (Hamiltonian::mult_add). Only x crosses to the
// device and only H x comes back: x in row blocks on a copy stream, each
// block's row pass (diagonal + up-spin hops, on a view of the down-spin tables
// shifted to the block) waiting for its own copy; the column pass once all of x
// is there; H x back in row blocks, and host threads adding each block into y
// as soon as it has landed.
int qed_hamiltonian_mult_add(qed_hamiltonian *h, const double *x, double *y) {
  return guarded([&] {
    if (!h) fail(QED_ERR_ARGUMENT, "null Hamiltonian");
    std::lock_guard<std::mutex> hl(h->m);
    const size_t D = h->H->D;
    if (!D) return;
    Workspace &w = ws();
    if (!h->copy) {
      QED_CUDA(cudaStreamCreateWithFlags(&h->copy, cudaStreamNonBlocking));
      for (int k = 0; k < kMultAddChunks; ++k) {
        QED_CUDA(cudaEventCreateWithFlags(&h->ev_in[k], cudaEventDisableTiming));
        QED_CUDA(cudaEventCreateWithFlags(&h->ev_out[k], cudaEventDisableTiming));
      }
    }
    if (h->x.n < D) h->x.alloc(D);
    if (h->z.n < D) h->z.alloc(D);
    if (h->hz_n < D) {
      if (h->hz) QED_CUDA(cudaFreeHost(h->hz));
      h->hz = nullptr;
      QED_CUDA(cudaMallocHost(&h->hz, D * sizeof(double)));
      h->hz_n = D;
    }
    w.sync();  // buffers allocated on w.stream are ready for the copy stream
    const HvOperator &op = h->H->op;
    const uint32_t du = op.up.dim, dd = op.dn.dim;
    size_t off[kMultAddChunks + 1];
    for (int k = 0; k <= kMultAddChunks; ++k) off[k] = (size_t)du * (size_t)((uint64_t)dd * k / kMultAddChunks);
    SubList none;
    for (int k = 0; k < kMultAddChunks; ++k) {
      const size_t n = off[k + 1] - off[k];
      if (n) QED_CUDA(cudaMemcpyAsync(h->x.p + off[k], x + off[k], n * sizeof(double), cudaMemcpyHostToDevice, h->copy));
      QED_CUDA(cudaEventRecord(h->ev_in[k], h->copy));
      QED_CUDA(cudaStreamWaitEvent(w.stream, h->ev_in[k], 0));
      if (!n) continue;
      HvOperator blk = op;  // rows [r0, r1) of the sector
      const uint32_t r0 = (uint32_t)(off[k] / du), r1 = (uint32_t)(off[k + 1] / du);
      blk.dn.bits += r0;
      blk.dn.diag += r0;
      blk.dn.dim = r1 - r0;
      launch_hv_rows(blk, h->x.p + off[k], 1.0, h->z.p + off[k], none, w.stream);
    }
    // the down-spin pass needs all of x; it runs by row blocks so that each
    // block's download (copy stream) overlaps the next blocks' work
    for (int k = 0; k < kMultAddChunks; ++k) {
      const size_t n = off[k + 1] - off[k];
      if (n) launch_hv_cols_rows(op, h->x.p, 1.0, h->z.p, (uint32_t)(off[k] / du), (uint32_t)(off[k + 1] / du),
                                 w.stream);
      QED_CUDA(cudaEventRecord(h->ev_in[k], w.stream));
      QED_CUDA(cudaStreamWaitEvent(h->copy, h->ev_in[k], 0));
      if (n) QED_CUDA(cudaMemcpyAsync(h->hz + off[k], h->z.p + off[k], n * sizeof(double), cudaMemcpyDeviceToHost, h->copy));
      QED_CUDA(cudaEventRecord(h->ev_out[k], h->copy));
    }
    int nt = (int)std::thread::hardware_concurrency();
    nt = std::max(1, std::min(nt, 16));
    std::atomic<int> bad{0};
    auto add = [&](int t) {
      for (int k = 0; k < kMultAddChunks; ++k) {
        if (cudaEventSynchronize(h->ev_out[k]) != cudaSuccess) {
          bad = 1;
          return;
        }
        const size_t n = off[k + 1] - off[k], a = off[k] + n * t / nt, b = off[k] + n * (t + 1) / nt;
        add_streaming(y + a, h->hz + a, b - a);
      }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; ++t) pool.emplace_back(add, t);
    add(0);
    for (auto &th : pool) th.join();
    if (bad) fail(QED_ERR_CUDA, "qed_hamiltonian_mult_add: device work failed");
    QED_CUDA(cudaStreamSynchronize(h->copy));
    w.sync();
  });
}

int qed_hamiltonian_apply_device(qed_hamiltonian *h, const double *x, double *y, void *stream) {
  return guarded([&] {
    if (!h) fail(QED_ERR_ARGUMENT, "null Hamiltonian");
    std::lock_guard<std::mutex> hl(h->m);
    Workspace &w = ws();
    cudaStream_t s = (cudaStream_t)stream;
    if (!h->H->D) return;
    SubList none;
    launch_hv(h->H->op, x, 1.0, y, none, 0, w.red, s);
  });
}

int qed_hamiltonian_apply_dots_device(qed_hamiltonian *h, const double *x, double *y, double *dots,
                                      void *stream) {
  return guarded([&] {
    if (!h) fail(QED_ERR_ARGUMENT, "null Hamiltonian");
    if (!dots) fail(QED_ERR_ARGUMENT, "null output array");
    std::lock_guard<std::mutex> hl(h->m);
    ws();
    cudaStream_t s = (cudaStream_t)stream;
    if (!h->H->D) {
      QED_CUDA(cudaMemsetAsync(dots, 0, 3 * sizeof(double), s));
      return;
    }
    if (!h->partials.n) {
      h->partials.alloc((size_t)kHvColsMaxBlocks * Reducer::kMaxRed);
      ws().sync();  // allocated in this thread's stream order, used on `stream`
    }
    Reducer r;
    r.partials = h->partials.p;
    r.max_blocks = kHvColsMaxBlocks;
    SubList none;
    int nb = launch_hv(h->H->op, x, 1.0, y, none, 7, r, s);
    launch_finalize(r.partials, nb, 3, dots, s);
  });
}

// No-allocation variant of qed_hamiltonian_apply_dots_device (see the header):
// no workspace lookup, no buffer growth; the scratch is the fixed device array
// behind launch_hv_dots_noalloc.
int qed_hamiltonian_apply_dots_device_noalloc(qed_hamiltonian *h, const double *x, double *y,
                                              double *dots, void *stream) {
  return guarded([&] {
    if (!h || !x || !y || !dots) fail(QED_ERR_ARGUMENT, "null argument");
    std::lock_guard<std::mutex> hl(h->m);
    // The Hamiltonian's tables live on the library's device: make it current in
    // this thread (cudaSetDevice allocates nothing), so that the scratch address
    // is looked up, and the kernels run, on that device.
    QED_CUDA(cudaSetDevice(g_device.load()));
    cudaStream_t s = (cudaStream_t)stream;
    if (!h->H->D) {
      QED_CUDA(cudaMemsetAsync(dots, 0, 3 * sizeof(double), s));
      return;
    }
    launch_hv_dots_noalloc(h->H->op, x, y, dots, s);
  });
}

int qed_hamiltonian_diag(qed_hamiltonian *h, double *d) {
  return guarded([&] {
    if (!h) fail(QED_ERR_ARGUMENT, "null Hamiltonian");
    std::lock_guard<std::mutex> hl(h->m);
    // diagonal = H applied to unit vectors is wasteful; rebuild it from the tables on the host
    const SectorOp &H = *h->H;
    std::vector<double> du(H.up->dim), dd(H.dn->dim);
    Workspace &w = ws();
    H.up->diag.download(du.data(), du.size(), w.stream);
    H.dn->diag.download(dd.data(), dd.size(), w.stream);
    std::vector<double> vin;
    if (H.op.inter.mode >= 2) {
      vin.resize(H.vinter.n);
      H.vinter.download(vin.data(), vin.size(), w.stream);
    }
    w.sync();
    const int n = H.L;
    for (uint32_t b = 0; b < H.dn->dim; ++b)
      for (uint32_t a = 0; a < H.up->dim; ++a) {
        uint32_t up = H.up->hbits[a], dn = H.dn->hbits[b];
        double s = du[a] + dd[b];
        const auto &it = H.op.inter;
        if (it.mode == 1) s += it.u * __builtin_popcount(up & dn);
        else if (it.mode == 2) { for (int r = 0; r < n; ++r) if ((up & dn) >> r & 1u) s += vin[r]; }
        else if (it.mode == 3) {
          for (int r = 0; r < n; ++r)
            if (dn >> r & 1u)
              for (int c = 0; c < n; ++c)
                if (up >> c & 1u) s += vin[(size_t)r * n + c];
        }
        d[a + (size_t)H.up->dim * b] = s;
      }
  });
}

int qed_hamiltonian_destroy(qed_hamiltonian *h) {
  return guarded([&] {
    delete h;
  });
}

int qed_halfbasis(int L, int N, unsigned *strings, long *dim) {
  return guarded([&] {
    if (L < 1 || L > 32 || N < 0 || N > L) fail(QED_ERR_ARGUMENT, "bad (L, N)");
    uint64_t d = binom(L, N);
    *dim = (long)d;
    if (!strings || !d) return;
    Workspace &w = ws();
    DevBuf<uint32_t> b(d);
    launch_unrank(L, N, (uint32_t)d, b.p, w.stream);
    b.download(strings, d, w.stream);
    w.sync();
  });
}

int qed_halfbasis_rank(int L, int N, long n, const unsigned *strings, unsigned *ranks) {
  return guarded([&] {
    if (L < 1 || L > 32 || N < 0 || N > L) fail(QED_ERR_ARGUMENT, "bad (L, N)");
    if (n <= 0) return;
    Workspace &w = ws();
    DevBuf<uint32_t> s(n), r(n);
    s.upload(strings, n, w.stream);
    launch_rank(L, N, n, s.p, r.p, w.stream);
    r.download(ranks, n, w.stream);
    w.sync();
  });
}

int qed_destroy_table(int L, int n_up, int n_dn, int a, long *target, int *phase) {
  return guarded([&] {
    if (L < 1 || L > 32 || a < 0 || a >= 2 * L) fail(QED_ERR_ARGUMENT, "bad orbital");
    Workspace &w = ws();
    // Evaluate c_a on every source state with the device gather: the source
    // state index is encoded as its value, so the gathered value identifies it.
    const int spin = a >= L ? 1 : 0, orb = a % L;
    const int tnu = n_up - (spin ? 0 : 1), tnd = n_dn - (spin ? 1 : 0);
    const uint64_t sdu = binom(L, n_up), sdd = binom(L, n_dn);
    const uint64_t tdu = (tnu < 0) ? 0 : binom(L, tnu), tdd = (tnd < 0) ? 0 : binom(L, tnd);
    const size_t Ds = sdu * sdd, Dt = tdu * tdd;
    for (size_t i = 0; i < Ds; ++i) { target[i] = -1; phase[i] = 0; }
    if (!Dt) return;
    DevBuf<uint32_t> tub(tdu), tdb(tdd);
    launch_unrank(L, tnu, (uint32_t)tdu, tub.p, w.stream);
    launch_unrank(L, tnd, (uint32_t)tdd, tdb.p, w.stream);
    std::vector<double> code(Ds);
    for (size_t i = 0; i < Ds; ++i) code[i] = (double)(i + 1);
    DevBuf<double> src(Ds), y(Dt);
    src.upload(code, w.stream);
    launch_cdag_gather(L, spin, orb, -1, tub.p, (uint32_t)tdu, tdb.p, (uint32_t)tdd, n_up, n_dn,
                       (uint32_t)sdu, src.p, y.p, 1.0, 0, w.stream);
    std::vector<double> hy(Dt);
    y.download(hy.data(), Dt, w.stream);
    w.sync();
    for (size_t I = 0; I < Dt; ++I) {
      if (hy[I] == 0.0) continue;
      long s = (long)std::llround(std::fabs(hy[I])) - 1;
      target[s] = (long)I;
      phase[s] = hy[I] < 0 ? 1 : 0;
    }
  });
}


// ---- point group (symmetry.hpp / symmetry.cuh) ------------------------------

static SymmetryGroup group_from_abi(int n_sites, int n_bath, int n_gen, const int *gen, int bath_irrep) {
  if (n_gen < 0 || (n_gen > 0 && !gen)) fail(QED_ERR_ARGUMENT, "bad generators");
  const int N = n_sites + n_bath;
  std::vector<std::vector<int>> g(n_gen, std::vector<int>(N));
  for (int j = 0; j < n_gen; ++j)
    for (int i = 0; i < N; ++i) g[j][i] = gen[(size_t)j * N + i];
  return build_symmetry_group(n_sites, n_bath, g, bath_irrep != 0);
}

int qed_symmetry_group(int n_sites, int n_bath, int n_gen, const int *gen, int bath_irrep, int *g, int *phi,
                       double *S_re, double *S_im, int *site_irrep_dim) {
  return guarded([&] {
    const SymmetryGroup G = group_from_abi(n_sites, n_bath, n_gen, gen, bath_irrep);
    const int n = G.g();
    if (g) *g = n;
    if (phi)
      for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) phi[a * n + b] = G.tab.phi[a][b];
    for (size_t k = 0; k < G.S.size(); ++k) {
      if (S_re) S_re[k] = G.S[k].real();
      if (S_im) S_im[k] = G.S[k].imag();
    }
    if (site_irrep_dim)
      for (int r = 0; r < n; ++r) site_irrep_dim[r] = G.site_irrep_dim[r];
  });
}

int qed_symmetry_representatives(int n_sites, int n_bath, int n_gen, const int *gen, int bath_irrep, int irrep,
                                 long n, const uint64_t *states, uint64_t *rep, int *phase, int *length) {
  return guarded([&] {
    const SymmetryGroup G = group_from_abi(n_sites, n_bath, n_gen, gen, bath_irrep);
    if (irrep < 0 || irrep >= G.g()) fail(QED_ERR_ARGUMENT, "irrep out of range");
    for (long i = 0; i < n; ++i) {
      const RepMap m = sym_representative(G.tab, states[i], irrep);
      rep[i] = m.rep;
      phase[i] = m.phase;
      length[i] = m.length;
    }
  });
}

// ---- Hamiltonian in the symmetry-adapted basis (mixed.hpp) -------------------

int qed_mixed_hamiltonian_create(int label, const char *sector, qed_mixed_hamiltonian **h, long *dim) {
  return guarded([&] {
    auto I = instance(label);
    if (!I->model->group) fail(QED_ERR_ARGUMENT, "model " + I->model->name + " has no point-group generators");
    // A generator of order above 2 gives the group complex characters; the
    // reference then works in a complex Hilbert space (src_ed/qcm_ED.cpp:153)
    // with phases such as i in the matrix elements. This product is real only.
    if (I->model->group->has_complex_irrep)
      fail(QED_ERR_UNSUPPORTED, "model " + I->model->name +
                                    ": point group with complex characters (a generator of order above 2) needs "
                                    "a complex Hilbert space, which this solver does not provide");
    const Sector S(sector);
    if (!sector_is_valid(S, I->model->n_orb, I->model->group->g()) || S.N >= Sector::odd || S.S >= Sector::odd)
      fail(QED_ERR_ARGUMENT, std::string("sector ") + sector + " is not valid");
    const MixedTerms t = mixed_terms(*I->model, I->value);
    Workspace &w = ws();
    auto *hh = new qed_mixed_hamiltonian;
    try {
      hh->H.reset(new MixedHamiltonian(*I->model->group, t, S.irrep, S.Nup(), S.Ndw(), w.stream));
    } catch (...) {
      delete hh;
      throw;
    }
    *dim = (long)hh->H->D;
    *h = hh;
  });
}

int qed_mixed_hamiltonian_states(qed_mixed_hamiltonian *h, uint64_t *states) {
  return guarded([&] {
    if (!h) fail(QED_ERR_ARGUMENT, "null Hamiltonian");
    std::lock_guard<std::mutex> hl(h->m);
    Workspace &w = ws();
    h->H->states.download(states, h->H->D, w.stream);
    w.sync();
  });
}

int qed_mixed_hamiltonian_mult_add(qed_mixed_hamiltonian *h, const double *x, double *y) {
  return guarded([&] {
    if (!h) fail(QED_ERR_ARGUMENT, "null Hamiltonian");
    std::lock_guard<std::mutex> hl(h->m);
    const size_t D = h->H->D;
    if (!D) return;
    Workspace &w = ws();
    DevBuf<double> dx(D), dy(D);
    dx.upload(x, D, w.stream);
    h->H->apply(dx.p, dy.p, w.stream);
    std::vector<double> hy(D);
    dy.download(hy.data(), D, w.stream);
    w.sync();
    for (size_t i = 0; i < D; ++i) y[i] += hy[i];
  });
}

int qed_mixed_hamiltonian_apply_device(qed_mixed_hamiltonian *h, const double *x, double *y, void *stream) {
  return guarded([&] {
    if (!h) fail(QED_ERR_ARGUMENT, "null Hamiltonian");
    h->H->apply(x, y, (cudaStream_t)stream);
  });
}

int qed_mixed_hamiltonian_ground_state(qed_mixed_hamiltonian *h, double *energy, int *iterations) {
  return guarded([&] {
    if (!h) fail(QED_ERR_ARGUMENT, "null Hamiltonian");
    std::lock_guard<std::mutex> hl(h->m);
    const LanczosResult r = lanczos_energy_mixed(*h->H, ws(), (uint64_t)opt_int("seed"));
    *energy = r.energy;
    if (iterations) *iterations = r.iterations;
  });
}

int qed_mixed_hamiltonian_ground_state_vector(qed_mixed_hamiltonian *h, double *energy, double *psi) {
  return guarded([&] {
    if (!h) fail(QED_ERR_ARGUMENT, "null Hamiltonian");
    std::lock_guard<std::mutex> hl(h->m);
    Workspace &w = ws();
    const uint64_t seed = (uint64_t)opt_int("seed");
    const LanczosResult r = lanczos_energy_mixed(*h->H, w, seed);
    DevBuf<double> v;
    lanczos_eigenvector_mixed(*h->H, w, r, seed, v);
    v.download(psi, h->H->D, w.stream);
    w.sync();
    *energy = r.energy;
  });
}

int qed_mixed_hamiltonian_nnz(qed_mixed_hamiltonian *h, long *nnz) {
  return guarded([&] {
    if (!h) fail(QED_ERR_ARGUMENT, "null Hamiltonian");
    *nnz = (long)h->H->nnz;
  });
}

int qed_mixed_hamiltonian_destroy(qed_mixed_hamiltonian *h) {
  return guarded([&] {
    if (!h) return;
    {
      std::lock_guard<std::mutex> hl(h->m);
      if (h->H && h->H->D) ws().sync();
    }
    delete h;
  });
}

}  // extern "C"
