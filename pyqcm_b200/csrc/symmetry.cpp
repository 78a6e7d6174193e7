// Host construction of the cluster point group (see symmetry.hpp). Follows the
// steps of symmetry_group::symmetry_group and ::build
// (src_ed/symmetry_group.cpp:17-34, 184-345): check the generators, their
// commutation and orders, enumerate the elements in mixed-radix order (the
// first generator's power varying fastest), the character phases
// phi(a, b) = sum_k a_k b_k g / n_k mod g, and the symmetric site orbitals
// sum_e chi(r, e) |e(site)> normalised, one per orbit that survives.
#include "symmetry.hpp"

#include <cmath>
#include <string>

#include "common.hpp"
#include "qed_b200.h"

namespace qed {

namespace {

using Elem = std::vector<int>;

struct Builder {
  int N, L, g = 1;

  Elem identity() const {
    Elem v(N, 0);
    for (int i = 0; i < L; ++i) v[i] = i;
    return v;
  }
  // x after y on the sites; bath phases add mod g
  Elem product(const Elem &x, const Elem &y) const {
    Elem v(N);
    for (int i = 0; i < L; ++i) v[i] = x[y[i]];
    for (int i = L; i < N; ++i) v[i] = (x[i] + y[i]) % g;
    return v;
  }
  bool sites_identity(const Elem &v) const {
    for (int i = 0; i < L; ++i)
      if (v[i] != i) return false;
    return true;
  }
  bool is_identity(const Elem &v) const {
    if (!sites_identity(v)) return false;
    for (int i = L; i < N; ++i)
      if (v[i] != 0) return false;
    return true;
  }
  bool valid_sites(const Elem &v) const {
    for (int i = 0; i < L; ++i) {
      if (v[i] < 0 || v[i] >= L) return false;
      for (int j = 0; j < i; ++j)
        if (v[i] == v[j]) return false;
    }
    return true;
  }
  bool differ(const Elem &x, const Elem &y, bool with_bath) const {
    const int n = with_bath ? N : L;
    for (int i = 0; i < n; ++i)
      if (x[i] != y[i]) return true;
    return false;
  }
};

std::vector<int> digits(int label, const std::vector<int> &radix) {
  std::vector<int> d(radix.size());
  for (size_t k = 0; k < radix.size(); ++k) {
    d[k] = label % radix[k];
    label /= radix[k];
  }
  return d;
}

}  // namespace

SymmetryGroup build_symmetry_group(int n_sites, int n_bath, const std::vector<std::vector<int>> &gen_in,
                                   bool bath_irrep) {
  const int N = n_sites + n_bath;
  if (n_sites < 1 || n_bath < 0 || N > kMaxSymOrb) fail(QED_ERR_ARGUMENT, "bad (n_sites, n_bath)");
  SymmetryGroup G;
  G.n_sites = n_sites;
  G.n_bath = n_bath;
  G.bath_irrep = bath_irrep && !gen_in.empty();
  Builder B{N, G.bath_irrep ? n_sites : N};
  std::vector<std::vector<int>> gen = gen_in;
  if (gen.empty()) gen.push_back(B.identity());
  if (gen.size() > 4) fail(QED_ERR_ARGUMENT, "Number of group generators exceeds the limit of 4");
  for (size_t i = 0; i < gen.size(); ++i) {
    if ((int)gen[i].size() != N)
      fail(QED_ERR_ARGUMENT, "generator " + std::to_string(i + 1) + " should have " + std::to_string(N) +
                                 " elements");
    if (!B.valid_sites(gen[i])) fail(QED_ERR_ARGUMENT, "generator " + std::to_string(i + 1) + " is not valid!");
  }
  auto check_commute = [&](bool with_bath) {
    for (size_t i = 0; i < gen.size(); ++i)
      for (size_t j = 0; j < i; ++j)
        if (B.differ(B.product(gen[i], gen[j]), B.product(gen[j], gen[i]), with_bath))
          fail(QED_ERR_ARGUMENT, "generators " + std::to_string(i + 1) + " and " + std::to_string(j + 1) +
                                     " do not commute!");
  };
  check_commute(false);

  // Orders from the site permutation alone; the bath phases are reduced mod the
  // partial group order while the orders are found, as in the reference.
  B.g = 1;
  for (const Elem &x : gen) {
    Elem p = B.identity();
    int n = 1;
    for (;;) {
      p = B.product(p, x);
      if (B.sites_identity(p)) break;
      ++n;
      if (n > kMaxGroup) fail(QED_ERR_UNSUPPORTED, "group order above " + std::to_string(kMaxGroup));
    }
    G.orders.push_back(n);
    B.g *= n;
    if (n > 2) G.has_complex_irrep = true;
  }
  if (B.g > kMaxGroup) fail(QED_ERR_UNSUPPORTED, "group order above " + std::to_string(kMaxGroup));
  check_commute(true);

  const int g = B.g;
  for (int i = 0; i < g; ++i) {
    const std::vector<int> d = digits(i, G.orders);
    Elem p = B.identity();
    for (size_t j = 0; j < gen.size(); ++j)
      for (int l = 0; l < d[j]; ++l) p = B.product(p, gen[j]);
    if (i != 0 && B.is_identity(p))
      fail(QED_ERR_ARGUMENT, "The identity is generated as a non trivial element (element " + std::to_string(i) + ")");
    for (int k = B.L; k < N; ++k)
      if (p[k] < 0 || p[k] >= g) fail(QED_ERR_ARGUMENT, "element " + std::to_string(i + 1) + " is not valid!");
    G.elements.push_back(p);
  }

  SymGroup &T = G.tab;
  T.N = N;
  T.L = B.L;
  T.g = g;
  for (int e = 0; e < g; ++e)
    for (int i = 0; i < N; ++i) T.perm[e][i] = (uint8_t)G.elements[e][i];
  for (int a = 0; a < g; ++a) {
    const std::vector<int> da = digits(a, G.orders);
    for (int b = 0; b < g; ++b) {
      const std::vector<int> db = digits(b, G.orders);
      int s = 0;
      for (size_t k = 0; k < G.orders.size(); ++k) s += da[k] * db[k] * g / G.orders[k];
      T.phi[a][b] = (int8_t)(s % g);
    }
  }

  // Symmetric site orbitals, irrep by irrep.
  using C = std::complex<double>;
  G.S.assign((size_t)n_sites * n_sites, C(0, 0));
  G.site_irrep_dim.assign(g, 0);
  int n_orb = 0;
  for (int r = 0; r < g; ++r) {
    std::vector<char> covered(n_sites, 0);
    for (int s = 0; s < n_sites; ++s) {
      if (covered[s]) continue;
      covered[s] = 1;
      std::vector<C> orb(n_sites, C(0, 0));
      for (int e = 0; e < g; ++e) {
        const int t = G.elements[e][s];
        if (t >= n_sites) fail(QED_ERR_ARGUMENT, "a generator maps a cluster site onto a bath orbital");
        covered[t] = 1;
        const double ang = 2.0 * M_PI * T.phi[r][e] / g;
        double c = std::cos(ang), si = std::sin(ang);
        if (std::fabs(c) < 1e-12) c = 0;   // characters are chopped as the reference does
        if (std::fabs(si) < 1e-12) si = 0;
        orb[t] += C(c, si);
      }
      double nrm = 0;
      for (const C &z : orb) nrm += std::norm(z);
      nrm = std::sqrt(nrm);
      if (nrm < 1e-12) continue;
      if (n_orb >= n_sites) fail(QED_ERR_ARGUMENT, "Problem with construction of symmetric orbitals");
      for (int i = 0; i < n_sites; ++i) G.S[(size_t)n_orb * n_sites + i] = orb[i] / nrm;
      ++n_orb;
      ++G.site_irrep_dim[r];
    }
  }
  if (n_orb != n_sites)
    fail(QED_ERR_ARGUMENT, "Problem with construction of symmetric orbitals: " + std::to_string(n_orb) +
                               " found instead of " + std::to_string(n_sites));
  return G;
}

int sym_tensor(const SymmetryGroup &G, int r1, int r2) {
  int out = 0, mult = 1;
  for (int n : G.orders) {
    out += ((r1 % n + r2 % n) % n) * mult;
    r1 /= n;
    r2 /= n;
    mult *= n;
  }
  return out;
}

int sym_conjugate(const SymmetryGroup &G, int r) {
  int out = 0, mult = 1;
  for (int n : G.orders) {
    out += ((n - r % n) % n) * mult;
    r /= n;
    mult *= n;
  }
  return out;
}

}  // namespace qed
