// Host construction of a cluster's Abelian point group from its generators:
// validation, the group elements, the character phases and the symmetric
// orbitals, filling the SymGroup tables that the per-state maps and kernels
// read (symmetry.cuh).
#pragma once

#include <complex>
#include <vector>

#include "symmetry.cuh"

namespace qed {

struct SymmetryGroup {
  int n_sites = 0, n_bath = 0;
  bool bath_irrep = false;
  bool has_complex_irrep = false;
  std::vector<int> orders;                    // order of each generator
  std::vector<std::vector<int>> elements;     // g elements, N entries each
  SymGroup tab{};                             // the tables for symmetry.cuh
  // Symmetric orbitals: row k of S (n_sites x n_sites, row-major) is the k-th
  // orbital, irreps in order; site_irrep_dim[r] of them belong to irrep r.
  std::vector<std::complex<double>> S;
  std::vector<int> site_irrep_dim;

  int g() const { return tab.g; }
};

// Builds the group of generators `gen` (0-based, as ED::new_model takes them:
// n_sites + n_bath entries each, site entries a permutation of the first L
// orbitals, bath entries orbital labels or, with bath_irrep, phases in units of
// 2 pi / g). Errors (QED_ERR_ARGUMENT) carry the reference's messages. With no
// generator the group is trivial (g = 1).
SymmetryGroup build_symmetry_group(int n_sites, int n_bath, const std::vector<std::vector<int>> &gen,
                                   bool bath_irrep);

// Irrep labels are mixed-radix numbers over the generators' orders: the product
// of two irreps adds the digits, the conjugate negates them, each modulo its
// order (symmetry_group::tensor and conjugate, src_ed/symmetry_group.cpp:343-356).
int sym_tensor(const SymmetryGroup &G, int r1, int r2);
int sym_conjugate(const SymmetryGroup &G, int r);

}  // namespace qed
