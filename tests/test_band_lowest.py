"""The warm-started lowest eigenvalue of the band-Lanczos convergence test
(band_lowest, pyqcm_b200/csrc/eigen.cpp) against numpy on growing sequences of
band matrices, each the leading block of the next: host code, compiled here
into a small driver."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "pyqcm_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include <vector>
#include "eigen.hpp"
using namespace qed;
// stdin: n_max b nchecks, then the full n_max x n_max band matrix (row-major);
// checks at n = 4b, 5b, ...: prints n, the eigenvalue, and 1 if band_lowest answered
int main() {
  int N, b, nc;
  if (scanf("%d %d %d", &N, &b, &nc) != 3) return 1;
  std::vector<double> A((size_t)N * N);
  for (auto &v : A) if (scanf("%lf", &v) != 1) return 1;
  BandLowest st;
  for (int c = 0; c < nc; ++c) {
    const int n = (4 + c) * b;
    std::vector<double> B((size_t)n * (b + 1), 0.0);
    for (int i = 0; i < n; ++i)
      for (int k = 0; k <= (i < b ? i : b); ++k) B[(size_t)i * (b + 1) + k] = A[(size_t)i * N + (i - k)];
    double lam = 0.0;
    const bool ok = band_lowest(n, b, B, st, &lam);
    if (!ok) {  // the caller's fallback: all eigenvalues, cold start next time
      std::vector<double> F((size_t)n * n, 0.0), ev;
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) F[(size_t)i + (size_t)n * j] = A[(size_t)i * N + j];
      band_eigenvalues(n, b, F, ev);
      lam = ev[0];
      st.valid = false;
    }
    printf("%d %.17g %d\n", n, lam, ok ? 1 : 0);
  }
  return 0;
}
"""


@pytest.fixture(scope="module")
def driver():
    d = tempfile.mkdtemp(prefix="band_lowest_")
    src = os.path.join(d, "drv.cpp")
    exe = os.path.join(d, "drv")
    with open(src, "w") as f:
        f.write(DRIVER)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, src, os.path.join(CSRC, "eigen.cpp"), "-o", exe],
                   check=True)
    return exe


def _band(N, b, rng, degenerate=False):
    A = np.zeros((N, N))
    for k in range(b + 1):
        v = rng.standard_normal(N - k)
        A += np.diag(v, -k) + (np.diag(v, k) if k else 0)
    if degenerate:  # two decoupled copies: every eigenvalue of the leading blocks at least doubled
        h = N // 2
        A[:h, h:] = 0
        A[h:, :h] = 0
        A[h:, h:] = A[:h, :h]
    return A


@pytest.mark.parametrize("b,seed,deg", [(2, 0, False), (4, 1, False), (10, 2, False), (16, 3, False), (4, 4, True)])
def test_band_lowest_matches_numpy(driver, b, seed, deg):
    rng = np.random.default_rng(seed)
    nc = 30
    N = (4 + nc) * b
    A = _band(N, b, rng, deg)
    inp = f"{N} {b} {nc}\n" + " ".join(f"{v:.17g}" for v in A.ravel())
    out = subprocess.run([driver], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    fast = 0
    for line in out:
        if not line.strip():
            continue
        n, lam, ok = line.split()
        n = int(n)
        want = np.linalg.eigvalsh(A[:n, :n])[0]
        assert abs(float(lam) - want) < 2e-14 * (1 + abs(want)) * max(1.0, np.abs(A[:n, :n]).sum(1).max()), (n, lam, want)
        fast += int(ok)
    assert fast >= nc // 2, fast  # most checks answered by the warm start
