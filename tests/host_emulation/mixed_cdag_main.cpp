// Host driver for the mixed-basis c / c+ gathers of pyqcm_b200/csrc/mixed.cu
// (k_mixed_create, k_mixed_destroy) compiled for the CPU with one-thread launch
// shims (tests/test_mixed_kernels_host.py extracts the kernel source into
// kernels_host.hpp). stdin: the group, the source sector (irrep, N_up, N_dn),
// the target irrep, pm, spin, the orbital's site coefficients and the source
// vector; stdout: the target basis and phi = c^{pm} psi.
#include "kernels_host.hpp"
#include "symmetry.hpp"
#include "common.hpp"
#include <iostream>
using namespace qed;

struct Basis {
  std::vector<uint64_t> st;
  std::vector<uint8_t> ln;
  std::vector<int32_t> fmap;
  uint32_t du = 0;
};

static Basis build(const SymmetryGroup &G, int irrep, int nu, int nd) {
  const int N = G.tab.N;
  std::vector<uint32_t> us, ds;
  for (uint32_t s = 0; s < (1u << N); ++s) {
    if (__builtin_popcount(s) == nu) us.push_back(s);
    if (__builtin_popcount(s) == nd) ds.push_back(s);
  }
  Basis b;
  b.du = (uint32_t)us.size();
  const uint64_t nf = (uint64_t)us.size() * ds.size();
  std::vector<uint8_t> lenf(nf);
  if (nf) k_mixed_mark(G.tab, irrep, us.data(), b.du, ds.data(), nf, lenf.data());
  b.fmap.assign(nf, -1);
  for (uint64_t f = 0; f < nf; ++f)
    if (lenf[f]) {
      b.fmap[f] = (int32_t)b.st.size();
      b.st.push_back((uint64_t)us[f % b.du] | ((uint64_t)ds[f / b.du] << 32));
      b.ln.push_back(lenf[f]);
    }
  return b;
}

int main() {
  int ns, nb, bi, ng;
  std::cin >> ns >> nb >> bi >> ng;
  std::vector<std::vector<int>> gen(ng, std::vector<int>(ns + nb));
  for (auto &g : gen)
    for (auto &v : g) std::cin >> v;
  int r_src, nu, nd, r_tgt, pm, spin;
  std::cin >> r_src >> nu >> nd >> r_tgt >> pm >> spin;
  OrbCoef cf{};
  for (int a = 0; a < ns; ++a) std::cin >> cf.c[a];
  SymmetryGroup G = build_symmetry_group(ns, nb, gen, bi != 0);
  for (int n = 0; n <= 32; ++n)
    for (int k = 0; k <= n; ++k) c_mbinom[n][k] = (uint32_t)qed::binom(n, k);
  const Basis src = build(G, r_src, nu, nd);
  std::vector<double> psi(src.st.size());
  for (auto &x : psi) std::cin >> x;
  const int tu = nu + (spin == 0 ? pm : 0), td = nd + (spin == 1 ? pm : 0);
  const Basis tgt = build(G, r_tgt, tu, td);
  std::vector<double> phi(tgt.st.size(), 0.0);
  if (!tgt.st.empty()) {
    if (pm == 1)
      k_mixed_create(G.tab, r_src, r_tgt, spin, ns, cf, tgt.st.data(), tgt.ln.data(), tgt.st.size(), src.fmap.data(),
                     src.du, src.ln.data(), psi.data(), phi.data());
    else
      k_mixed_destroy(G.tab, r_src, r_tgt, spin, ns, cf, tgt.st.data(), tgt.st.size(), src.fmap.data(), src.du,
                      src.ln.data(), psi.data(), phi.data());
  }
  printf("%zu %zu\n", src.st.size(), tgt.st.size());
  for (size_t J = 0; J < tgt.st.size(); ++J) printf("%llu %.17g\n", (unsigned long long)tgt.st[J], phi[J]);
}
