"""The packed hop tables of the staged-row H.v kernels (pack_hops16 after
order_for_banks, pyqcm_b200/csrc/bank_order.cpp), on the hop tables of real
lattices: decoding every 16-bit entry as the kernels do (target = low 14 bits,
sign = bit 14, magnitude class = bit 15, padding aimed at the zero slots
dim .. dim + 7) gives back the one-spin hopping operator of the numpy
restatement exactly; at every step the eight strings of a group gather from
eight distinct 16-byte bank groups; tables with a third magnitude or too many
strings are refused. Host code, compiled here into a small driver."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import port
from pyqcm_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "pyqcm_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include <vector>
#include "bank_order.hpp"
// stdin: dim width nvals, vals[nvals], cnt[dim], ell[width * dim]
// stdout: ok w0 w1 mag0 mag1, cnt[dim], pk0[4 * w0 * dim], pk1[4 * w1 * dim]
int main() {
  unsigned dim; int width, nv;
  if (scanf("%u %d %d", &dim, &width, &nv) != 3) return 1;
  std::vector<double> vals(nv);
  for (auto &v : vals) if (scanf("%lf", &v) != 1) return 1;
  std::vector<uint8_t> cnt(dim);
  std::vector<uint32_t> ell((size_t)width * dim);
  for (auto &c : cnt) { unsigned v; if (scanf("%u", &v) != 1) return 1; c = (uint8_t)v; }
  for (auto &e : ell) if (scanf("%u", &e) != 1) return 1;
  const int zero = nv;
  vals.push_back(0.0);
  int w2 = width;
  if (!qed::order_for_banks(ell, cnt, dim, w2, zero)) { printf("0 0 0 0 0\n"); return 0; }
  qed::PackedHops ph;
  const bool ok = qed::pack_hops16(ell, cnt, dim, vals, zero, ph);
  printf("%d %d %d %.17g %.17g\n", ok ? 1 : 0, ph.width[0], ph.width[1], ph.mag[0], ph.mag[1]);
  if (!ok) return 0;
  for (auto c : ph.cnt) printf("%u ", (unsigned)c);
  printf("\n");
  for (int c = 0; c < 2; ++c) {
    for (auto e : ph.pk[c]) printf("%u ", (unsigned)e);
    printf("\n");
  }
  return 0;
}
"""


@pytest.fixture(scope="module")
def driver():
    d = tempfile.mkdtemp(prefix="packed_hops_")
    src = os.path.join(d, "drv.cpp")
    exe = os.path.join(d, "drv")
    with open(src, "w") as f:
        f.write(DRIVER)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", CSRC, src, os.path.join(CSRC, "bank_order.cpp"), "-o", exe],
                   check=True)
    return exe


def _ell(T):
    """ELL table of the off-diagonal part of T (row i: y_i += T_ij x_j), with the
    value slots of the library's table build (v at 2k, -v at 2k + 1)."""
    T = T.tocsr()
    dim = T.shape[0]
    vals, slot = [], {}
    rows = []
    for i in range(dim):
        ent = []
        for j, v in zip(T.indices[T.indptr[i]:T.indptr[i + 1]], T.data[T.indptr[i]:T.indptr[i + 1]]):
            if j == i or v == 0.0:
                continue
            key = abs(v)
            if key not in slot:
                slot[key] = len(vals)
                vals += [key, -key]
            ent.append((int(j) << 8) | (slot[key] + (1 if v < 0 else 0)))
        rows.append(ent)
    width = max(len(r) for r in rows)
    ell = np.zeros((width, dim), dtype=np.uint64)
    cnt = np.array([len(r) for r in rows])
    for i, r in enumerate(rows):
        ell[:len(r), i] = r
    return vals, cnt, ell


def _run(driver, vals, cnt, ell):
    dim = ell.shape[1]
    inp = f"{dim} {ell.shape[0]} {len(vals)}\n" + " ".join(repr(float(v)) for v in vals) + "\n"
    inp += " ".join(map(str, cnt)) + "\n" + " ".join(map(str, ell.reshape(-1))) + "\n"
    out = subprocess.run([driver], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    ok, w0, w1, m0, m1 = out[0].split()
    if ok == "0":
        return None
    cnt = np.array(out[1].split(), dtype=np.int64)
    pk = [np.array(out[2 + c].split(), dtype=np.int64).reshape(int(w), dim, 4) for c, w in enumerate((w0, w1))]
    return cnt, pk, (float(m0), float(m1))


@pytest.mark.parametrize("lx,ly,tp,n", [(2, 7, 0.3, 7), (3, 4, 0.3, 5), (2, 6, 0.0, 6), (3, 3, 0.3, 4)])
def test_packed_table_decodes_to_the_operator(driver, lx, ly, tp, n):
    prob = W.hubbard_cluster(lx, ly, t=-1.0, tp=tp, U=4.0, mu=2.0)
    t_up, _, _ = port.collect_terms(prob)
    T, _ = port.hop_matrix(prob.n_orb, n, t_up)
    dim = T.shape[0]
    vals, cnt, ell = _ell(T)
    res = _run(driver, vals, cnt, ell)
    assert res is not None
    cw, pk, (m0, m1) = res
    rng = np.random.default_rng(3)
    x = rng.standard_normal(dim)
    xz = np.concatenate([x, np.zeros(8)])  # the zero slots dim .. dim + 7
    y = np.zeros(dim)
    mags = (m0, m1)
    nwords = [cw & 15, cw >> 4]
    for c in range(2):
        for i in range(dim):
            g0 = i - i % 8
            for k in range(nwords[c][i]):
                for q in range(4):
                    h = int(pk[c][k, i, q])
                    tgt = h & 0x3FFF
                    assert tgt < dim + 8 and not (h & 0x4000)
                    y[i] += (-mags[c] if h & 0x8000 else mags[c]) * xz[tgt]
                    if i == g0:  # the group's eight strings read distinct 16-byte bank groups
                        lanes = range(g0, min(g0 + 8, dim))
                        groups = [int(pk[c][k, l, q]) & 0x3FFF for l in lanes]
                        assert len({g % 8 for g in groups}) == len(groups), (c, i, k, q)
    import scipy.sparse as sp
    ref = (T - sp.diags(T.diagonal())) @ x
    assert np.max(np.abs(y - ref)) <= 1e-13 * np.max(np.abs(ref))
    full = len(cw) - len(cw) % 8
    assert (cw[:full].reshape(-1, 8) == cw[:full:8, None]).all()  # counts uniform per group of eight


def test_tables_outside_the_format_are_refused(driver):
    # three distinct magnitudes
    prob = W.hubbard_cluster(3, 3, t=-1.0, tp=0.3, U=4.0, mu=2.0)
    t_up, _, _ = port.collect_terms(prob)
    t_up = t_up.copy()
    t_up[0, 1] = t_up[1, 0] = -0.7
    T, _ = port.hop_matrix(prob.n_orb, 4, t_up)
    vals, cnt, ell = _ell(T)
    assert _run(driver, vals, cnt, ell) is None
    # more strings than 14-bit targets can address with the eight zero slots
    dim = (1 << 14) - 4
    ell = np.zeros((1, dim), dtype=np.uint64)
    cnt = np.zeros(dim, dtype=np.int64)
    assert _run(driver, [1.0, -1.0], cnt, ell) is None
