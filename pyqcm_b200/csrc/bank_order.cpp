// Hop-list ordering for bank-conflict-free shared-memory gathers (see bank_order.hpp).
#include "bank_order.hpp"

#include <algorithm>
#include <functional>

namespace qed {

bool order_for_banks(std::vector<uint32_t> &ell, std::vector<uint8_t> &cnt, uint32_t dim, int &width, int zero_slot) {
  constexpr int G = 8;
  const uint32_t ngroups = (dim + G - 1) / G;
  std::vector<std::vector<uint32_t>> out(ngroups);  // per group: steps x G entries
  std::vector<int> steps(ngroups, 0);
  int wmax = 0;
  for (uint32_t g = 0; g < ngroups; ++g) {
    const uint32_t u0 = g * G;
    const int nl = (int)std::min<uint32_t>(G, dim - u0);
    std::vector<std::vector<uint32_t>> left(nl);
    for (int l = 0; l < nl; ++l)
      for (int k = 0; k < cnt[u0 + l]; ++k) left[l].push_back(ell[(size_t)k * dim + u0 + l]);
    auto &o = out[g];
    for (;;) {
      int remaining = 0;
      for (int l = 0; l < nl; ++l) remaining += (int)left[l].size();
      if (!remaining) break;
      int owner[G];  // lane holding each bank group this step, -1 free
      int pick[G];   // index into left[l] of the lane's hop, -1 none
      for (int s = 0; s < G; ++s) owner[s] = -1;
      for (int l = 0; l < G; ++l) pick[l] = -1;
      std::vector<int> order(nl);
      for (int l = 0; l < nl; ++l) order[l] = l;
      std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return left[a].size() > left[b].size(); });
      for (int l : order) {
        if (left[l].empty()) continue;
        bool seen[G] = {};
        std::function<bool(int)> augment = [&](int lane) -> bool {
          for (size_t i = 0; i < left[lane].size(); ++i) {
            const int s = (int)((left[lane][i] >> 8) % G);
            if (seen[s]) continue;
            seen[s] = true;
            if (owner[s] < 0 || augment(owner[s])) {
              owner[s] = lane;
              pick[lane] = (int)i;
              return true;
            }
          }
          return false;
        };
        augment(l);
      }
      std::vector<uint32_t> row(G, 0u);
      for (int l = 0; l < nl; ++l) {
        if (pick[l] >= 0) {
          row[l] = left[l][pick[l]];
          continue;
        }
        int s = 0;  // a free bank group for the padding entry
        while (s < G && owner[s] >= 0) ++s;
        uint32_t target = u0 + (uint32_t)(s % G);
        if (s == G || target >= dim) target = u0 + (uint32_t)l;
        if (s < G) owner[s] = l;
        row[l] = (target << 8) | (uint32_t)zero_slot;
      }
      for (int l = 0; l < nl; ++l)
        if (pick[l] >= 0) left[l].erase(left[l].begin() + pick[l]);
      o.insert(o.end(), row.begin(), row.end());
      ++steps[g];
    }
    wmax = std::max(wmax, steps[g]);
  }
  if (wmax > 255) return false;
  width = wmax;
  ell.assign((size_t)width * dim, 0u);
  for (uint32_t g = 0; g < ngroups; ++g) {
    const uint32_t u0 = g * G;
    const int nl = (int)std::min<uint32_t>(G, dim - u0);
    for (int k = 0; k < steps[g]; ++k)
      for (int l = 0; l < nl; ++l) ell[(size_t)k * dim + u0 + l] = out[g][(size_t)k * G + l];
    for (int l = 0; l < nl; ++l) cnt[u0 + l] = (uint8_t)steps[g];
  }
  return true;
}

}  // namespace qed
