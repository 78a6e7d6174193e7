// Model instance: ground-state search over sectors, Green-function
// representations and their evaluation. Follows model_instance<double>
// (src_ed/model_instance.hpp) and model_instance_base (src_ed/model_instance_base.cpp)
// for the spin-conserving, trivial-group case.
#pragma once
#include <complex>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "model.hpp"
#include "mixed.hpp"
#include "solver.hpp"

namespace qed {

using cplx = std::complex<double>;

// Lehmann representation of one state (Q_matrix, src_ed/Q_matrix.hpp:20-40):
// poles e[M], residues V (L x M, column-major), plus a device copy for G(z).
struct QMat {
  int L = 0, M = 0;
  std::vector<double> e, V;
  DevBuf<double> de, dV;
};

// Continued fractions of one state (continued_fraction_set, src_ed/continued_fraction_set.cpp):
// electron (e) and hole (h) fractions for pairs o2 <= o1 of the n cluster sites.
struct CFSet {
  int n = 0;
  std::vector<std::vector<double>> ea, eb, ha, hb;  // index o1*n + o2
};

// One matrix continued fraction of a state and spin (the hole or the electron
// part of mcf_set, src_ed/mcf_set.hpp:51-60): M floors of p x p blocks, A
// shifted by the state's energy as matrix_continued_fraction's constructor
// does (src_ed/matrix_continued_fraction.hpp:84-100), B the off-diagonal blocks,
// W the p x q weight (row-major; sqrt(weight) folded in).
struct McfPart {
  int M = 0, p = 0, q = 0;
  std::vector<double> A, B, W;
};
struct McfSet {
  McfPart e, h;
};

struct State {
  Sector sec;
  double energy = 0.0, weight = 0.0;
  DevBuf<double> psi;
  LanczosResult lanczos;     // tridiagonal of the eigenvalue pass (replayed for psi)
  bool dense = false;        // psi from full diagonalisation (small sector, non-factorized model)
  std::vector<double> hpsi;  // dense: the eigenvector on the host until it is uploaded
  QMat q[2];   // [spin_down]
  CFSet cf[2];
  McfSet mcf[2];
};

// Eigenvalue pass of one target sector: the unit of work that batched drivers
// spread over host threads (the selection of states needs all of them).
struct SectorSolve {
  Sector sec;
  size_t dim = 0;
  bool dense = false;
  std::vector<double> w, U;  // dense: all eigenvalues (ascending) and eigenvectors
  LanczosResult lanczos;     // Lanczos: tridiagonal and lowest energy
};

// Small Lanczos sectors set aside by Instance::solve_sector for one
// lanczos_energy_batch over a whole batch call.
struct DeferredSectors {
  std::mutex m;
  std::vector<std::unique_ptr<SectorOp>> ops;
  std::vector<LanczosBatchItem> items;  // at most lanczos_job_max_dim() states: one batched pass
  std::vector<LanczosBatchItem> large;  // the others: one task each
};


// Hole (s = 0) or electron (s = 1) part of the Q-matrix of one state and spin.
struct QPart {
  std::vector<double> e, V;
  // models with a point group: one segment per irrep of the symmetric orbitals,
  // V in that irrep's orbital basis (n_r rows), in irrep order
  struct Seg {
    int r = 0;
    std::vector<double> e, V;
  };
  std::vector<Seg> segs;
};

struct Instance {
  int label = 0;
  std::shared_ptr<Model> model;
  std::map<std::string, double> value;
  SectorSet target_sectors;
  int mix = 0;
  bool is_correlated = false;
  bool use_cf = false;
  bool use_mcf = false;  // GF_method 'M': matrix continued fractions (block Lanczos)
  bool mcf_qr = false;   // block_Lanczos_QR: QR (true) or polar (false) off-diagonal blocks
  int dim_GF = 0;
  bool gs_solved = false, gf_solved = false, hopping_solved = false;
  double GS_energy = 0.0, E0 = 0.0, SEF_bath = 0.0, GF_density = 0.0;
  std::vector<std::shared_ptr<State>> states;
  SpinData terms;
  HalfCache tables;  // spin tables shared by the sectors of this instance
  std::map<std::string, HalfCache> op_tables;  // the same for each operator alone (averages, susceptibility)
  std::vector<double> tc[2], tb[2], tcb[2];  // cluster, bath (diagonalised), cluster-bath
  std::vector<double> tb_nd[2], tcb_nd[2];   // bath and cluster-bath before the bath diagonalisation
  std::vector<cplx> Mave[2];
  // uncorrelated instances: <c+_b c_a> over cluster and bath orbitals, which is
  // what the reference's Green_function_average returns for them
  std::vector<cplx> Mfull[2];
  // cluster_averages: (operator, average, variance) for every operator of the
  // instance, in name order (model_instance::averages, src_ed/model_instance.hpp:340-345)
  std::vector<std::tuple<std::string, double, double>> averages;
  std::mutex mtx;

  Instance(int label, std::shared_ptr<Model> m, std::map<std::string, double> value,
           const std::string &sectors);

  // fails (unsupported) for what the symmetry-adapted path does not cover:
  // complex characters, continued-fraction Green functions, susceptibilities
  void require_supported_group() const;
  bool has_group() const { return model->group && model->group->g() > 1; }
  std::pair<double, std::string> low_energy_states(Workspace &ws);
  void green_solve(Workspace &ws);

  // The steps of low_energy_states and green_solve, for drivers that run the
  // sectors, states and Q-matrix halves of many instances concurrently. A
  // single instance runs them in this order on one thread.
  // uncorrelated instances (no interaction operator): one_body_solve
  // (src_ed/model_instance.hpp:1164-1256), the one-body problem in full
  void one_body_solve(Workspace &ws);
  size_t sector_dim(const Sector &s) const;
  // defer: if given, a Lanczos sector is only prepared (its operator and result
  // slot go to defer, with the small sectors apart)
  void solve_sector(const Sector &s, SectorSolve &out, Workspace &ws, DeferredSectors *defer = nullptr);
  void select_states(std::vector<SectorSolve> &r);  // every sector, in target order
  void state_vector(State &st, Workspace &ws);
  // the operator averages of the selected states, then gs_solved
  void finish_gs(Workspace &ws);
  void check_gf_solvable() const;
  void qmatrix_part(State &st, bool spin_down, int s, QPart &out, Workspace &ws);
  void qmatrix_combine(State &st, bool spin_down, QPart (&parts)[2], Workspace &ws);
  void build_cf(State &st, bool spin_down, Workspace &ws);
  // build_mcf (src_ed/model_instance.hpp:847-946): per hole / electron part, the
  // start block c_i^{-+}|state>, its QR (weight W), block Lanczos, the shifted floors
  void build_mcf(State &st, bool spin_down, Workspace &ws);
  void finish_gf();
  // G(z) for nz frequencies: out[k*n*n + b + a*n] (column-major blocks)
  void green_function(const cplx *z, int nz, bool spin_down, cplx *out, Workspace &ws);
  // the same into device memory (n_sites^2 * nz complex, column-major per z)
  void green_function_device(const cplx *z, int nz, bool spin_down, double *dG, Workspace &ws);
  void self_energy(const cplx *z, int nz, bool spin_down, cplx *out, Workspace &ws);
  void hybridization(const cplx *z, int nz, bool spin_down, cplx *out);
  double potthoff(Workspace &ws);
  // model_instance::hopping_matrix / hopping_matrix_full (src_ed/model_instance.cpp:13-16,
  // src_ed/model_instance.hpp:1491-1523): column-major, real parts (real Hilbert space)
  std::vector<double> hopping_matrix(bool spin_down) const;
  std::vector<double> hopping_matrix_full(bool spin_down, bool diag) const;
  // model_instance::interactions (src_ed/model_instance.hpp:1528-1541)
  std::vector<Element> interactions() const;
  // model_instance::tr_sigma_inf (src_ed/model_instance.hpp:1279-1312)
  double tr_sigma_inf(Workspace &ws);
  // model_instance::susceptibility / susceptibility_poles (src_ed/model_instance.hpp:1027-1115):
  // chi(w) = sum over states of weight * sum_i |<i|O|psi>|^2 / (w - (E_i - E0)),
  // from the Lehmann representation of O|psi> in the state's own sector
  void susceptibility(const std::string &op, const cplx *w, int nw, cplx *chi, Workspace &ws);
  std::vector<std::pair<double, double>> susceptibility_poles(const std::string &op, Workspace &ws);
  std::string gs_string() const;
  void set_hopping_matrix();

 private:
  // Q-matrix (p = 1) of O|psi> for every state: poles shifted by the state energy
  struct SusQ {
    const State *st;
    std::vector<double> e, V;
  };
  std::vector<SusQ> susceptibility_qmatrices(const std::string &op, Workspace &ws);
  void build_qmatrix(State &st, bool spin_down, Workspace &ws);
  void compute_weights();
  std::string where(const Sector &s) const;
  void green_average();
  // fills phi = c^{pm}_{orb, spin} |psi> on the target sector of H
  void apply_cdag(const State &st, int pm, int spin, int orb, const SectorOp &H, double *y,
                  double coef, bool accumulate, Workspace &ws);
  // the symmetry-adapted Hamiltonian of a sector (models with a point group)
  std::unique_ptr<MixedHamiltonian> mixed_sector(const Sector &s, Workspace &ws) const;
  void qmatrix_part_mixed(State &st, bool spin_down, int s, QPart &out, Workspace &ws);
  void qmatrix_combine_mixed(State &st, bool spin_down, QPart (&parts)[2], Workspace &ws);
};

bool sector_is_valid(const Sector &s, int n_orb, int g = 1);
Sector shift_sector(const Sector &s, int pm, int spin);

}  // namespace qed
