// Host driver for the mixed-basis kernels of pyqcm_b200/csrc/mixed.cu compiled
// for the CPU with one-thread launch shims (tests/test_mixed_kernels_host.py
// extracts the kernel source into kernels_host.hpp): builds the basis and the
// CSR rows of one sector from a model read on stdin and prints them.
#include "kernels_host.hpp"
#include "symmetry.hpp"
#include "common.hpp"
#include <iostream>
using namespace qed;
int main() {
  int ns, nb, bi, ng; std::cin >> ns >> nb >> bi >> ng;
  std::vector<std::vector<int>> gen(ng, std::vector<int>(ns + nb));
  for (auto &g : gen) for (auto &v : g) std::cin >> v;
  int irrep, nu, nd; std::cin >> irrep >> nu >> nd;
  int no; std::cin >> no; std::vector<int> r(no), c(no); std::vector<double> v(no);
  for (int k = 0; k < no; ++k) std::cin >> r[k] >> c[k] >> v[k];
  int ndg; std::cin >> ndg; std::vector<uint64_t> dm(ndg); std::vector<double> dv(ndg);
  for (int k = 0; k < ndg; ++k) std::cin >> dm[k] >> dv[k];
  SymmetryGroup G = build_symmetry_group(ns, nb, gen, bi != 0);
  for (int n = 0; n <= 32; ++n) for (int k = 0; k <= n; ++k) c_mbinom[n][k] = (uint32_t)qed::binom(n, k);
  const int N = G.tab.N;
  std::vector<uint32_t> us, ds;
  for (uint32_t s = 0; s < (1u << N); ++s) { if (__builtin_popcount(s) == nu) us.push_back(s); if (__builtin_popcount(s) == nd) ds.push_back(s); }
  uint64_t du = us.size(), nf = du * ds.size();
  std::vector<uint8_t> lenf(nf);
  k_mixed_mark(G.tab, irrep, us.data(), (uint32_t)du, ds.data(), nf, lenf.data());
  std::vector<int32_t> fmap(nf, -1); std::vector<uint64_t> st; std::vector<uint8_t> ln;
  for (uint64_t f = 0; f < nf; ++f) if (lenf[f]) { fmap[f] = (int32_t)st.size(); st.push_back((uint64_t)us[f % du] | ((uint64_t)ds[f / du] << 32)); ln.push_back(lenf[f]); }
  uint64_t D = st.size();
  OffTerms ot{no, r.data(), c.data(), v.data()};
  std::vector<uint32_t> cnt(D);
  k_mixed_rows<false>(G.tab, irrep, ot, st.data(), ln.data(), D, fmap.data(), (uint32_t)du, cnt.data(), nullptr, nullptr, nullptr);
  std::vector<uint64_t> rp(D + 1, 0);
  for (uint64_t J = 0; J < D; ++J) rp[J + 1] = rp[J] + cnt[J];
  std::vector<uint32_t> col(rp[D]); std::vector<double> val(rp[D]);
  k_mixed_rows<true>(G.tab, irrep, ot, st.data(), ln.data(), D, fmap.data(), (uint32_t)du, nullptr, rp.data(), col.data(), val.data());
  std::vector<double> dg(D);
  k_mixed_diag(st.data(), D, dm.data(), dv.data(), ndg, dg.data());
  printf("%llu\n", (unsigned long long)D);
  for (uint64_t J = 0; J < D; ++J) printf("%llu %.17g\n", (unsigned long long)st[J], dg[J]);
  for (uint64_t J = 0; J < D; ++J) for (uint64_t k = rp[J]; k < rp[J + 1]; ++k) printf("%llu %u %.17g\n", (unsigned long long)J, col[k], val[k]);
}
