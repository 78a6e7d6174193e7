// Hop-list ordering for bank-conflict-free shared-memory gathers (see bank_order.hpp).
#include "bank_order.hpp"

#include <algorithm>
#include <cmath>
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

namespace qed {

bool pack_hops16(const std::vector<uint32_t> &ell, const std::vector<uint8_t> &cnt, uint32_t dim,
                 const std::vector<double> &vals, int zero_slot, PackedHops &out) {
  constexpr int G = 8;
  if (dim == 0 || dim + G > (1u << 14)) return false;
  std::vector<double> mags;  // magnitude classes of the value slots in use
  for (uint32_t i = 0; i < dim; ++i)
    for (int k = 0; k < cnt[i]; ++k) {
      const int slot = (int)(ell[(size_t)k * dim + i] & 255u);
      if (slot == zero_slot) continue;
      const double m = std::fabs(vals[slot]);
      if (m != 0.0 && std::find(mags.begin(), mags.end(), m) == mags.end()) mags.push_back(m);
    }
  if (mags.size() > 2) return false;
  std::sort(mags.begin(), mags.end(), [](double a, double b) { return a > b; });
  while (mags.size() < 2) mags.push_back(0.0);
  // per class: an ELL sub-table (target << 8 | sign) ordered for banks
  const uint32_t zbase = dim % G;  // bank group of zero slot dim + j is (zbase + j) % G
  auto zero_entry = [&](uint32_t group) -> uint16_t { return (uint16_t)(dim + (group + G - zbase) % G); };
  std::vector<uint8_t> words[2];
  for (int c = 0; c < 2; ++c) {
    std::vector<std::vector<uint32_t>> lists(dim);
    int w = 0;
    for (uint32_t i = 0; i < dim; ++i) {
      for (int k = 0; k < cnt[i]; ++k) {
        const uint32_t e = ell[(size_t)k * dim + i];
        const int slot = (int)(e & 255u);
        if (slot == zero_slot) continue;
        const double v = vals[slot];
        if (v == 0.0 || std::fabs(v) != mags[c]) continue;
        lists[i].push_back(((e >> 8) << 8) | (v < 0 ? 1u : 0u));
      }
      w = std::max<int>(w, (int)lists[i].size());
    }
    std::vector<uint32_t> sub((size_t)std::max(w, 1) * dim, 0u);
    std::vector<uint8_t> sc(dim);
    for (uint32_t i = 0; i < dim; ++i) {
      sc[i] = (uint8_t)lists[i].size();
      for (size_t k = 0; k < lists[i].size(); ++k) sub[k * dim + i] = lists[i][k];
    }
    // bank ordering; its padding entries carry "slot" 2 (neither sign)
    int w2 = w;
    if (w > 0 && !order_for_banks(sub, sc, dim, w2, 2)) return false;
    if (w == 0) w2 = 0;
    words[c].assign(dim, 0);
    int wmax = 0;
    for (uint32_t i = 0; i < dim; ++i) {
      const int nw = (sc[i] + 3) / 4;
      if (nw > 15) return false;
      words[c][i] = (uint8_t)nw;
      wmax = std::max(wmax, nw);
    }
    out.width[c] = wmax;
    out.pk[c].assign((size_t)4 * wmax * dim, 0);
    for (uint32_t i = 0; i < dim; ++i) {
      const uint32_t lane = i % G;
      for (int k = 0; k < 4 * words[c][i]; ++k) {
        uint16_t e;
        if (k < sc[i]) {
          const uint32_t v = sub[(size_t)k * dim + i];
          const uint32_t tgt = v >> 8, tag = v & 255u;
          if (tag == 2) e = zero_entry(tgt % G);  // bank padding keeps its bank group
          else e = (uint16_t)(tgt | (tag ? 0x8000u : 0u));
        } else {
          e = zero_entry(lane);  // rounding to whole words: the lane's own bank group
        }
        out.pk[c][((size_t)(k / 4) * dim + i) * 4 + (k % 4)] = e;
      }
    }
  }
  out.cnt.assign(dim, 0);
  for (uint32_t i = 0; i < dim; ++i) out.cnt[i] = (uint8_t)(words[0][i] | (words[1][i] << 4));
  out.mag[0] = mags[0];
  out.mag[1] = mags[1];
  return true;
}

}  // namespace qed
