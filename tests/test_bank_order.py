"""The hop-list ordering of the up-spin tables (order_for_banks,
pyqcm_b200/csrc/bank_order.cpp) on random tables: every string keeps its hops,
padding entries carry the zero value slot, and at every step the eight strings
of a group gather from eight distinct 16-byte bank groups. Host code, compiled
here into a small driver."""
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
#include "bank_order.hpp"
// stdin: dim width zero_slot, cnt[dim], ell[width * dim]; stdout: ok width cnt[dim] ell[width' * dim]
int main() {
  unsigned dim; int width, zero;
  if (scanf("%u %d %d", &dim, &width, &zero) != 3) return 1;
  std::vector<uint8_t> cnt(dim);
  std::vector<uint32_t> ell((size_t)width * dim);
  for (auto &c : cnt) { unsigned v; if (scanf("%u", &v) != 1) return 1; c = (uint8_t)v; }
  for (auto &e : ell) if (scanf("%u", &e) != 1) return 1;
  const bool ok = qed::order_for_banks(ell, cnt, dim, width, zero);
  printf("%d %d\n", ok ? 1 : 0, width);
  for (auto c : cnt) printf("%u ", (unsigned)c);
  printf("\n");
  for (auto e : ell) printf("%u ", e);
  printf("\n");
  return 0;
}
"""


@pytest.fixture(scope="module")
def driver():
    d = tempfile.mkdtemp(prefix="bank_order_")
    src = os.path.join(d, "drv.cpp")
    exe = os.path.join(d, "drv")
    with open(src, "w") as f:
        f.write(DRIVER)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, src, os.path.join(CSRC, "bank_order.cpp"), "-o", exe],
                   check=True)
    return exe


@pytest.mark.parametrize("dim,seed", [(924, 0), (1001, 1), (64, 2), (3432, 3)])
def test_order_for_banks_invariants(driver, dim, seed):
    rng = np.random.default_rng(seed)
    width = 36
    zero = 4
    cnt = rng.integers(0, width + 1, dim)
    hops = [sorted(rng.choice(dim, size=c, replace=False)) for c in cnt]
    slots = [rng.integers(0, 4, c) for c in cnt]
    ell = np.zeros((width, dim), dtype=np.uint64)
    for u in range(dim):
        for k in range(cnt[u]):
            ell[k, u] = (int(hops[u][k]) << 8) | int(slots[u][k])
    inp = f"{dim} {width} {zero}\n" + " ".join(map(str, cnt)) + "\n" + " ".join(map(str, ell.ravel()))
    out = subprocess.run([driver], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    ok, w2 = map(int, out[0].split())
    assert ok == 1
    c2 = np.array(out[1].split(), dtype=np.int64)
    e2 = np.array(out[2].split(), dtype=np.uint64).reshape(w2, dim)
    assert w2 == c2.max()
    for u in range(dim):
        entries = [int(e2[k, u]) for k in range(c2[u])]
        real = sorted((e >> 8, e & 255) for e in entries if (e & 255) != zero)
        assert real == sorted(zip(map(int, hops[u]), map(int, slots[u]))), u
        assert all((e >> 8) < dim for e in entries)
    for g0 in range(0, dim, 8):
        lanes = range(g0, min(g0 + 8, dim))
        assert len({c2[u] for u in lanes}) == 1  # one step count per group
        for k in range(c2[g0]):
            banks = [int(e2[k, u]) >> 8 for u in lanes]
            assert len({b % 8 for b in banks}) == len(banks), (g0, k, banks)
