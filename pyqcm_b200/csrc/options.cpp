// Global options (see options.hpp). Defaults follow src_util/global_parameter.cpp:10-92.
#include "options.hpp"

#include <atomic>
#include <map>
#include <mutex>

#include "common.hpp"

namespace qed {

namespace {

struct Table {
  std::map<std::string, bool> b;
  std::map<std::string, long> i;
  std::map<std::string, double> d;
  std::map<std::string, char> c;
  std::mutex m;
  Table() {
    // ED options that drive this solver
    b["check_lanczos_residual"] = false;
    b["no_degenerate_BL"] = false;
    b["continued_fraction"] = false;
    b["verb_ED"] = false;
    b["verb_Hilbert"] = false;
    b["verb_warning"] = false;
    b["parallel_sectors"] = false;
    b["merge_states"] = false;
    b["combine_mcf"] = false;
    b["block_Lanczos_QR"] = false;
    b["nosym"] = false;
    b["print_Hamiltonian"] = false;
    b["strip_anomalous_self"] = false;
    b["print_variances"] = false;
    d["accur_band_lanczos"] = 1e-12;
    d["accur_continued_fraction"] = 0.01;
    d["accur_Davidson"] = 1.0e-5;
    d["accur_deflation"] = 1e-7;
    d["accur_lanczos"] = 1e-12;
    d["accur_Q_matrix"] = 1.0e-5;
    d["band_lanczos_minimum_gap"] = 1e-5;
    d["minimum_weight"] = 0.01;
    d["Qmatrix_wtol"] = 1.0e-5;
    d["Qmatrix_vtol"] = 1.0e-10;
    d["temperature"] = 0.0;
    i["n_states"] = 1;
    i["max_dim_print"] = 64;
    i["max_dim_full"] = 256;
    i["max_iter_BL"] = 600;
    i["max_iter_CF"] = 400;
    i["max_iter_lanczos"] = 1000;
    // solver options (not in the reference): band-Lanczos sectors with at least
    // block_lanczos_min_dim states and at least block_lanczos_min_p start
    // vectors run the block form of the recurrence (p vectors per H.v). Measured
    // on a B200 (Green function of one instance, band against block form): p = 8,
    // 4900 states 83 / 57 ms; p = 10, 63504 states 107 / 68 ms; p = 12, 853776
    // states 588 / 432 ms; p = 4, 16 concurrent 853776-state instances, 32.8 / 32.7
    // solves/s; 1024 random clusters (bench batch): 112 solves/s with the block form
    // from 1000 states, 142 from 200 states (also 142 from 50 states and p = 2; G
    // equal to 2e-13 between the three).
    // solver option: the 16-step chunks of the ground-state Lanczos of sectors of
    // at least lanczos_graphs_min_dim states are captured once per solve into
    // CUDA graphs (one per rotation of the three Krylov buffers) and replayed.
    // Measured on a B200 (default bench batches): 256 points of the 2x2 + 8-bath
    // model (853776 states) 43.3 solves/s with graphs, 40.6 without; 1024 random
    // clusters (sectors up to 63504 states) 49-61 with graphs for every sector
    // above the job table, 72 without: the three captures per solve cost more than
    // the replays save on sectors of tens of thousands of states.
    b["lanczos_graphs"] = true;
    // solver option: sectors of at most this many states run the ground-state
    // Lanczos in the one-CTA-per-sector job table (see lanczos_energy_batch).
    // Measured on a B200 (1024 random clusters, default bench batch): 73 solves/s
    // at 8192 (sectors above it step by step on whole-GPU kernels, 16 host
    // threads), 125-128 at 65536 (every sector of those clusters in the table;
    // energies equal to 1e-15, G to 5e-12). 256 bath points (853776-state
    // sectors): 44.7 solves/s at 65536, 24.8 at 2^20 (one CTA is too little there).
    i["lanczos_job_max_dim"] = 65536;
    // solver options: the symmetry-adapted (mixed-basis) Hamiltonian of a sector
    // is stored as CSR unless that takes more than mixed_csr_max_gb gigabytes;
    // then (or always, with mixed_on_the_fly) every product recomputes its entries.
    b["mixed_on_the_fly"] = false;
    d["mixed_csr_max_gb"] = 32.0;
    i["lanczos_graphs_min_dim"] = 131072;
    // solver option: launch variant of the H.v kernels of sectors without the
    // staged kernels (bits: 1 L2-only column gathers, 2 row pass with four
    // gathers in flight, 4 staged kernels off); see hv_variant (kernels.cu).
    i["hv_variant"] = 2;
    // solver option: spin tables of at most this many strings are built on the
    // host (the same tables as the device build, uploaded at once).
    i["host_table_max_dim"] = 4096;
    // solver options: with hv_windows, sectors of at least hv_windows_min_dim
    // states whose hops fit windows of eight consecutive sites run their H.v
    // through the window kernels (winhv.hpp), compiled at run time for the
    // lattice. Off by default: measured on a B200 (4x4 sector, 12870^2 states)
    // 10.9 ms per H.v against 4.6 ms for the staged kernels (same H x to 2e-16).
    b["hv_windows"] = false;
    i["hv_windows_min_dim"] = 1 << 22;
    i["block_lanczos_min_dim"] = 200;
    i["block_lanczos_min_p"] = 4;
    i["seed"] = 0;
    i["GF_lookup_depth"] = 64;
    c["Hamiltonian_format"] = 'E';
    c["Ground_state_method"] = 'L';
    c["GF_method"] = 'L';
    // lattice-layer options: accepted, unused here
    for (auto s : {"dual_basis", "periodic", "periodized_averages", "zero_dim", "print_all",
                   "compact_tiling_per_site", "use_pcubature", "verb_integrals"})
      b[s] = false;
    d["eta"] = 0.0001;
    d["small_scale"] = 0.5;
    d["cutoff_scale"] = 1.0e12;
    d["accur_OP"] = 1e-4;
    d["large_scale"] = 20;
    d["accur_SEF"] = 5e-8;
    d["cdmft_jacobian_delta"] = 1.0e-5;
    i["kgrid_side"] = 32;
    i["max_iter_QN"] = 60;
    i["print_precision"] = 9;
    c["periodization"] = 'G';
  }
};

Table &T() {
  static Table t;
  return t;
}

std::atomic<unsigned long long> g_generation{0};

template <class M> typename M::mapped_type get(M &m, const std::string &name) {
  auto it = m.find(name);
  if (it == m.end()) fail(QED_ERR_ARGUMENT, "global parameter " + name + " does not exist.");
  return it->second;
}
template <class M, class V> void put(M &m, const std::string &name, V v) {
  auto it = m.find(name);
  if (it == m.end()) fail(QED_ERR_ARGUMENT, "global parameter " + name + " does not exist.");
  it->second = v;
}

}  // namespace

bool opt_bool(const std::string &n) { std::lock_guard<std::mutex> l(T().m); return get(T().b, n); }
long opt_int(const std::string &n) { std::lock_guard<std::mutex> l(T().m); return get(T().i, n); }
double opt_double(const std::string &n) { std::lock_guard<std::mutex> l(T().m); return get(T().d, n); }
char opt_char(const std::string &n) { std::lock_guard<std::mutex> l(T().m); return get(T().c, n); }

void set_opt_bool(const std::string &n, bool v) {
  std::lock_guard<std::mutex> l(T().m);
  put(T().b, n, v);
  ++g_generation;
}
void set_opt_int(const std::string &n, long v) {
  std::lock_guard<std::mutex> l(T().m);
  put(T().i, n, v);
  ++g_generation;
}
void set_opt_double(const std::string &n, double v) {
  std::lock_guard<std::mutex> l(T().m);
  put(T().d, n, v);
  ++g_generation;
}
void set_opt_char(const std::string &n, char v) {
  std::lock_guard<std::mutex> l(T().m);
  put(T().c, n, v);
  ++g_generation;
}

unsigned long long options_generation() { return g_generation.load(std::memory_order_acquire); }

}  // namespace qed
