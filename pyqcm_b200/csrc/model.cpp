// Host-side model description (see model.hpp).
#include "model.hpp"

#include <cstdio>
#include <sstream>

#include "common.hpp"

namespace qed {

Sector::Sector(const std::string &str) {
  bool valid = true;
  auto grab = [&](char key, const char *fmt, int &dst, int dflt) {
    auto loc = str.find(key);
    if (loc == std::string::npos) {
      dst = dflt;
      return;
    }
    if (std::sscanf(str.c_str() + loc, fmt, &dst) != 1) valid = false;
  };
  grab('N', "N%d", N, even);
  grab('S', "S%d", S, even);
  grab('R', "R%d", irrep, 0);
  if (!valid) fail(QED_ERR_ARGUMENT, "sector string " + str + " does not conform to standard!");
  if (str.find('O') != std::string::npos) N = S = odd;
  if (S == even && N != even && N % 2) S = odd;
  if (N == even && S != even && S % 2) N = odd;
}

std::string Sector::name() const {
  std::ostringstream s;
  if (S == odd && N == odd) s << "O";
  s << "R" << irrep;
  if (N != even && N != odd) s << ":N" << N;
  if (S != even && S != odd) s << ":S" << S;
  return s.str();
}

std::shared_ptr<Operator> make_operator(const Model &m, const std::string &name,
                                        const std::string &type, const std::vector<Element> &raw) {
  auto op = std::make_shared<Operator>();
  op->name = name;
  const int no = m.n_orb;
  for (auto &x : raw)
    if (x.r < 0 || x.c < 0 || x.r >= 2 * no || x.c >= 2 * no)
      fail(QED_ERR_ARGUMENT, "operator " + name + ": orbital index out of range");
  std::map<std::pair<int, int>, double> emap;
  if (type == "one-body") {
    // Hermitian completion (src_ed/Operators/one_body_operator.hpp:63-71)
    for (auto &x : raw) {
      if (x.r < x.c) {
        op->elements.push_back({x.r, x.c, x.v});
        op->elements.push_back({x.c, x.r, x.v});
      } else if (x.r == x.c) {
        op->elements.push_back(x);
      }
    }
    if (op->elements.empty()) fail(QED_ERR_ARGUMENT, "operator " + name + " has no elements");
    for (auto &x : op->elements) emap[{x.r, x.c}] = x.v;
    // spin flip (check_spin_flip, :96-105)
    for (auto &x : op->elements)
      if ((x.r < no) != (x.c < no)) { op->mix |= mixing::spin_flip; break; }
    // spin symmetry (check_spin_symmetry, :112-128)
    if (!(op->mix & mixing::spin_flip)) {
      for (auto &kv : emap) {
        int r = kv.first.first, c = kv.first.second;
        r = r < no ? r + no : r - no;
        c = c < no ? c + no : c - no;
        auto y = emap.find({r, c});
        if (y == emap.end() || y->second != kv.second) { op->mix |= mixing::up_down; break; }
      }
    }
    // target (set_target, :141-176)
    const auto &e0 = op->elements[0];
    if (m.in_bath[e0.r]) op->target = m.in_bath[e0.c] ? 2 : 3;
    else op->target = m.in_bath[e0.c] ? 3 : 1;
    for (auto &x : op->elements) {
      bool br = m.in_bath[x.r], bc = m.in_bath[x.c];
      bool ok = (op->target == 1) ? (!br && !bc) : (op->target == 2) ? (br && bc) : (br != bc);
      if (!ok) fail(QED_ERR_ARGUMENT, "operator " + name + " has no unique target");
    }
  } else if (type == "interaction") {
    op->is_interaction = true;
    for (auto &x : raw) {
      if (x.r <= x.c) op->elements.push_back(x);
      else op->elements.push_back({x.c, x.r, x.v});
    }
    if (op->elements.empty()) fail(QED_ERR_ARGUMENT, "operator " + name + " has no elements");
    for (auto &x : op->elements) emap[{x.r, x.c}] = x.v;
    // spin symmetry (src_ed/Operators/interaction_operator.hpp:72-89)
    for (auto &kv : emap) {
      int r = kv.first.first, c = kv.first.second;
      r = r < no ? r + no : r - no;
      c = c < no ? c + no : c - no;
      auto y = emap.find({r, c}), y2 = emap.find({c, r});
      bool a = (y == emap.end() || y->second != kv.second);
      bool b = (y2 == emap.end() || y2->second != kv.second);
      if (a && b) { op->mix |= mixing::up_down; break; }
    }
    for (auto &x : op->elements)
      if (m.in_bath[x.r] || m.in_bath[x.c])
        fail(QED_ERR_ARGUMENT, "interaction operator " + name + " must be defined on the cluster only");
  } else {
    fail(QED_ERR_UNSUPPORTED, "operator type '" + type + "' of " + name +
                                  " is outside the spin-factorized solver (one-body, interaction)");
  }
  return op;
}

SpinData collect_terms(const Model &m, const std::map<std::string, double> &value) {
  SpinData s;
  const int n = m.n_orb;
  s.n = n;
  s.t_up.assign((size_t)n * n, 0.0);
  s.t_dn.assign((size_t)n * n, 0.0);
  s.v_dd.assign((size_t)n * n, 0.0);
  s.v_uu.assign((size_t)n * n, 0.0);
  s.v_du.assign((size_t)n * n, 0.0);
  for (auto &kv : value) {
    const Operator &op = *m.term.at(kv.first);
    const double z = kv.second;
    if (!op.is_interaction) {
      for (auto &x : op.elements) {
        if (x.r < n && x.c < n) s.t_up[(size_t)x.r * n + x.c] += z * x.v;
        else if (x.r >= n && x.c >= n) s.t_dn[(size_t)(x.r - n) * n + (x.c - n)] += z * x.v;
        else fail(QED_ERR_UNSUPPORTED, "spin-flip term in " + op.name);
      }
    } else {
      s.correlated = true;
      for (auto &x : op.elements) {
        // The reference tests mask(r) + mask(c) on b = dn | (up << 32), where
        // mask(i) = bit i for i < n and bit (i - n + 32) otherwise
        // (src_ed/Operators/HS_interaction_operator.hpp:44-53, binary_state.hpp:60-63).
        // The sum is taken literally, so r == c tests the next bit up.
        auto mask = [&](int i) -> unsigned long long {
          return i >= n ? (1ull << (i - n + 32)) : (1ull << i);
        };
        unsigned long long mk = mask(x.r) + mask(x.c);
        unsigned mdn = (unsigned)(mk & 0xffffffffull), mup = (unsigned)(mk >> 32);
        int cd = __builtin_popcount(mdn), cu = __builtin_popcount(mup);
        auto low = [](unsigned w) { return __builtin_ctz(w); };
        auto high = [](unsigned w) { return 31 - __builtin_clz(w); };
        if (cu == 0) {  // dn-string only
          int a = low(mdn), b = high(mdn);
          if (b >= n) fail(QED_ERR_UNSUPPORTED, "interaction bit outside the orbital range");
          s.v_dd[(size_t)a * n + b] += z * x.v;
        } else if (cd == 0) {
          int a = low(mup), b = high(mup);
          if (b >= n) fail(QED_ERR_UNSUPPORTED, "interaction bit outside the orbital range");
          s.v_uu[(size_t)a * n + b] += z * x.v;
        } else {
          int a = low(mdn), b = low(mup);
          if (a >= n || b >= n) fail(QED_ERR_UNSUPPORTED, "interaction bit outside the orbital range");
          s.v_du[(size_t)a * n + b] += z * x.v;
        }
      }
    }
  }
  return s;
}

}  // namespace qed
