// Hamiltonian of one sector in the symmetry-adapted (mixed) basis of a cluster
// with point-group generators: the reference's CSR format
// (src_ed/Hamiltonian/Hamiltonian_CSR.hpp over ED_mixed_basis) built on the
// device and kept resident in HBM.
//
// Build, all on the device: every state of the factorized (N_up, N_dn) sector
// is marked when it is its orbit's representative with a nonzero projection
// (sym_representative); a scan over the marks, in the factorized order (down
// string major), gives the sorted representative list and a dense map from
// factorized index to basis index. Each basis row J then applies every
// off-diagonal one-body element to its state, finds the representative K of the
// image and its basis index through the map (combinatorial ranks of the two
// strings), and stores (K, phase x coefficient x fermion sign x
// sqrt(len_J / len_K)): the reference's element of
// src_ed/Operators/HS_one_body_operator.hpp:17-37 read along the row, as H is
// symmetric. Rows are counted first, then filled. The diagonal (one-body
// diagonal and interaction elements, mask rule of
// src_ed/Operators/HS_interaction_operator.hpp:44-53) is its own vector.
//
// H x is then a CSR product: eight lanes per row, HBM-bound on the column and
// value arrays (12 bytes per entry), x gathered through L2. Sectors whose CSR
// would exceed mixed_csr_max_gb (or every sector of at least max_dim_full
// states, with mixed_on_the_fly) store no matrix: each product recomputes the
// entries from the states, eight lanes per row over the one-body elements
// (on_the_fly), with the same epilogues.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "common.hpp"
#include "kernels.cuh"
#include "model.hpp"
#include "symmetry.hpp"

namespace qed {

// Elements of H = sum over operators of value x operator, split as the mixed
// basis uses them: off-diagonal one-body (r != c, both orders, merged by (r, c))
// and diagonal masks (a one-body diagonal is one bit; an interaction element
// (r, c) is mask(r) + mask(c)).
struct MixedTerms {
  std::vector<int> r, c;
  std::vector<double> v;
  std::vector<uint64_t> dmask;
  std::vector<double> dval;
};
MixedTerms mixed_terms(const Model &m, const std::map<std::string, double> &value);

struct MixedHamiltonian {
  size_t D = 0;          // basis dimension
  size_t nnz = 0;        // off-diagonal entries
  int irrep = 0, n_up = 0, n_dn = 0;
  uint32_t du = 0, dd = 0;   // strings per spin of the (n_up, n_dn) sector
  SymGroup group{};          // the group tables the basis was built with
  DevBuf<uint64_t> states;   // sorted representatives (spin up in the low word)
  DevBuf<uint8_t> len;       // orbit lengths
  DevBuf<int32_t> fmap;      // factorized index (up rank + du * dn rank) -> basis index, -1 if none
  DevBuf<uint64_t> row_ptr;  // D + 1
  DevBuf<uint32_t> col;
  DevBuf<double> val;
  DevBuf<double> dg;         // diagonal
  bool on_the_fly = false;   // no stored matrix: entries recomputed by every product
  int n_terms = 0;           // off-diagonal one-body elements (kept for the on-the-fly products)
  DevBuf<int> term_r, term_c;
  DevBuf<double> term_v;

  MixedHamiltonian(const SymmetryGroup &G, const MixedTerms &t, int irrep, int n_up, int n_dn, cudaStream_t s);
  // y = H x on device vectors of D doubles, on stream s
  void apply(const double *x, double *y, cudaStream_t s) const;
  // y = xs H x - sum_k sub.c[k] sub.z[k], with the column pass's reductions of
  // the result (red_mask bit 0: <xs x, y>, bit 1: <y, y>, bit 2: <xs x, xs x>)
  // as per-block partials (stride Reducer::kMaxRed); nothing at all when
  // *skip != 0. Returns the block count.
  int apply_full(const double *x, double xs, double *y, const SubList &sub, int red_mask, Reducer &r,
                 cudaStream_t s, const int *skip = nullptr) const;
  // the matrix as D x D dense (column-major), for full diagonalisation of small sectors
  std::vector<double> dense(cudaStream_t s) const;
  // w = H v - (*beta_dev) vprev, with per-block partials of <v, w> at
  // partials[block * ld]; returns the number of blocks (at most max_blocks)
  int lanczos_w(const double *v, const double *vprev, const double *beta_dev, double *w, double *partials, int ld,
                int max_blocks, cudaStream_t s) const;
};

// c or c+ of one symmetric orbital (site coefficients coef[a], a < n_sites,
// spin 0 up / 1 down) on a mixed-basis state: phi = c^{pm} psi with psi in the
// basis of `src` and phi in the basis of `tgt` (pm = +1: tgt has one more
// particle of that spin; -1: one fewer). One thread per target state, no
// atomics: creation gathers, per occupied orbital of the target state, the
// representative of the state with that orbital emptied; destruction walks the
// target state's orbit (each distinct image once) and, per orbital the image
// leaves empty, the representative of the image with it filled. The matrix
// elements are those of the reference's destruction operator
// (src_ed/ED_basis.cpp:62-78, src_ed/Operators/destruction_operator.cpp:12-32).
void mixed_cdag(const MixedHamiltonian &src, const MixedHamiltonian &tgt, int pm, int spin, int n_sites,
                const double *coef, const double *psi, double *phi, cudaStream_t s);

}  // namespace qed
