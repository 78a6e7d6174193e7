// Host-side model description: sectors, operators, models and the one-body /
// interaction data a sector Hamiltonian is built from.
//
// Mirrors the reference's definitions for the spin-factorized case:
//   sector               src_ed/sector.hpp:23-147
//   one-body operator    src_ed/Operators/one_body_operator.hpp:53-190
//   interaction operator src_ed/Operators/interaction_operator.hpp:32-120
//   model                src_ed/model.hpp:24-55
#pragma once
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <string>
#include <vector>

namespace qed {

// Hilbert-space mixing states (src_ed/sector.hpp:11-17). This solver handles
// the spin-conserving cases: normal and up_down.
namespace mixing {
constexpr int normal = 0, anomalous = 1, spin_flip = 2, full = 3, up_down = 4;
}

struct Sector {
  static constexpr int odd = 9999, even = 10000;
  int N = 0, S = 0, irrep = 0;
  Sector() = default;
  Sector(int n, int s, int r) : N(n), S(s), irrep(r) {}
  explicit Sector(const std::string &str);  // "R0:N8:S0" (src_ed/sector.hpp:55-96)
  int Nup() const { return (N + S) / 2; }
  int Ndw() const { return (N - S) / 2; }
  std::string name() const;  // "R0:N8:S0" (src_ed/sector.hpp:101-107)
  bool operator==(const Sector &o) const { return N == o.N && S == o.S && irrep == o.irrep; }
  bool operator!=(const Sector &o) const { return !(*this == o); }
};

// Ordering of std::less<sector> (src_ed/sector.hpp:155-166): by S, then N, then irrep.
struct SectorLess {
  bool operator()(const Sector &x, const Sector &y) const {
    if (x.S != y.S) return x.S < y.S;
    if (x.N != y.N) return x.N < y.N;
    return x.irrep < y.irrep;
  }
};
using SectorSet = std::set<Sector, SectorLess>;

struct Element {
  int r, c;
  double v;
};

struct Operator {
  std::string name;
  bool is_interaction = false;
  int target = 1;   // 1 cluster, 2 bath, 3 cluster-bath (set_target)
  int mix = 0;      // mixing contribution of this operator
  std::vector<Element> elements;  // after the reference's normalisation
};

struct SymmetryGroup;

struct Model {
  std::string name;
  // point group of the generators given at creation; null for none (g = 1)
  std::shared_ptr<const SymmetryGroup> group;
  int n_sites = 0, n_bath = 0, n_orb = 0;
  bool is_closed = false;
  int mix = -1;  // mixing fixed by the first instance (src_ed/model_instance_base.cpp:71-78)
  // Hamiltonian_format latched at the model's first instance
  // (src_ed/model_instance_base.cpp:45-54) and the factorized flag derived from
  // it (:86-97). Non-factorized models diagonalise sectors smaller than
  // max_dim_full densely (src_ed/model_instance.hpp:200-205).
  char format = 0;
  bool factorized = false;
  std::map<std::string, std::shared_ptr<Operator>> term;
  std::vector<bool> in_bath;  // 2*n_orb entries
  mutable std::mutex mtx;
};

// Builds the Operator from raw elements with the reference's normalisation and
// checks (Hermiticity, target, spin symmetry). Throws Error on invalid input.
std::shared_ptr<Operator> make_operator(const Model &m, const std::string &name,
                                        const std::string &type, const std::vector<Element> &raw);

// Total one-body matrix of one spin species (n_orb x n_orb, row-major t[r*n+c],
// meaning sum t[r][c] c^+_r c_c) and the density-density interaction data of a
// parameter set, in the conventions of the factorized Hamiltonian
// (src_ed/Operators/HS_half_operator.hpp:17-45, HS_interaction_operator.hpp:32-54).
struct SpinData {
  int n = 0;
  std::vector<double> t_up, t_dn;    // one-body, per spin
  // interaction, expressed on the factorized bit strings b = dn | (up << 32)
  // exactly as the reference tests masks (src_ed/binary_state.hpp:60-63):
  std::vector<double> v_dd;   // n x n: v_dd[r*n+c] * [dn_r][dn_c], r<=c
  std::vector<double> v_uu;   // n x n on the up string
  std::vector<double> v_du;   // n x n: v_du[r*n+s] * [dn_r][up_s]
  bool correlated = false;
};
SpinData collect_terms(const Model &m, const std::map<std::string, double> &value);

}  // namespace qed
