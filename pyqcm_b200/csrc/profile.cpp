// Phase timers (see profile.hpp).
#include "profile.hpp"

#include <atomic>
#include <cstdio>
#include <cstdlib>

namespace qed {

namespace {
const char *kNames[kPhCount] = {"sector setup",       "GS Lanczos (eigenvalue)", "GS Lanczos (eigenvector)",
                                "dense sectors",      "c/c+ start vectors",      "band Lanczos recurrence",
                                "band Lanczos checks", "band projected eigensystem", "continued fractions",
                                "GS Ritz tests (in GS eigenvalue)", "block Lanczos recurrence",
                                "block Lanczos fallbacks", "ground-state operator averages",
                                "GS batched small sectors"};

struct Totals {
  std::atomic<long long> ns[kPhCount];
  std::atomic<long long> calls[kPhCount];
  bool on;
  Totals() : on(std::getenv("QED_PROFILE") != nullptr) {
    for (int i = 0; i < kPhCount; ++i) {
      ns[i] = 0;
      calls[i] = 0;
    }
  }
  ~Totals() {
    if (!on) return;
    std::fprintf(stderr, "qed profile (host wall time summed over threads):\n");
    for (int i = 0; i < kPhCount; ++i)
      if (calls[i])
        std::fprintf(stderr, "  %-28s %10.3f s  %8lld calls\n", kNames[i], ns[i] * 1e-9, (long long)calls[i]);
  }
};

Totals &totals() {
  static Totals t;
  return t;
}
}  // namespace

bool profiling() { return totals().on; }

void profile_add(Phase p, double seconds) {
  totals().ns[p] += (long long)(seconds * 1e9);
  totals().calls[p] += 1;
}

}  // namespace qed
