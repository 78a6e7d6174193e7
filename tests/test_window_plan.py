"""The window form of the per-spin hop operator (winhv.hpp), on the host.

The planner covers a lattice's hopping pairs with windows of eight consecutive
sites and builds the lane tables and warp schedule of the window kernels;
qed_window_plan applies exactly those tables on the host. Here it is compared
with a direct application of the hops, the rule of the reference's one-body
terms (binary_state::one_body, src_ed/binary_state.cpp:23-28: c+_r c_c allowed
when c is occupied and r empty, sign = parity of the occupied sites strictly
between r and c), with random amplitudes per directed pair (t[r][c] != t[c][r]).
The generated kernels are compiled with NVRTC (no device needed) and must not
spill."""
import re
from math import comb

import numpy as np
import pytest


def lattice_pairs(nx, ny, diagonal=True):
    site = lambda x, y: x + nx * y
    bonds = []
    for y in range(ny):
        for x in range(nx):
            if x + 1 < nx:
                bonds.append((site(x, y), site(x + 1, y)))
            if y + 1 < ny:
                bonds.append((site(x, y), site(x, y + 1)))
            if diagonal and x + 1 < nx and y + 1 < ny:
                bonds.append((site(x, y), site(x + 1, y + 1)))
            if diagonal and x >= 1 and y + 1 < ny:
                bonds.append((site(x, y), site(x - 1, y + 1)))
    pd, ps = [], []
    for a, b in bonds:
        pd += [a, b]
        ps += [b, a]
    return np.array(pd, np.int32), np.array(ps, np.int32)


def direct_hops(L, N, pd, ps, amp, x):
    bits = [s for s in range(1 << L) if bin(s).count("1") == N]
    rank = {s: i for i, s in enumerate(bits)}
    y = np.zeros(len(bits))
    for i, s in enumerate(bits):
        for q in range(len(pd)):
            r, c = int(pd[q]), int(ps[q])
            if not (s >> c) & 1 or (s >> r) & 1:
                continue
            ns = s ^ (1 << c) ^ (1 << r)
            lo, hi = min(r, c), max(r, c)
            between = ((1 << hi) - 1) & ~((2 << lo) - 1)
            sign = -1.0 if bin(ns & between).count("1") & 1 else 1.0
            y[i] += sign * amp[q] * x[rank[ns]]
    return y


@pytest.mark.parametrize("nx,ny,N,diag,nwin", [(4, 4, 5, True, 3), (4, 3, 6, True, 2), (2, 4, 3, True, 1),
                                               (6, 2, 5, False, 3), (5, 2, 5, False, 2), (3, 3, 4, True, 2),
                                               # edge cases: one window narrower than 8 sites, empty
                                               # and full fillings, one particle, one hole
                                               (2, 2, 2, True, 1), (2, 2, 0, True, 1), (2, 2, 4, True, 1),
                                               (4, 4, 1, True, 3), (4, 4, 15, True, 3)])
def test_window_form_equals_direct_hops(qed, nx, ny, N, diag, nwin):
    L = nx * ny
    pd, ps = lattice_pairs(nx, ny, diag)
    rng = np.random.default_rng(L * 31 + N)
    amp = rng.normal(size=len(pd))
    x = rng.normal(size=comb(L, N))
    nw, y = qed.window_plan(L, N, pd, ps, amp, x)
    assert nw == nwin
    want = direct_hops(L, N, pd, ps, amp, x)
    assert np.max(np.abs(y - want)) < 1e-13 * max(1.0, np.max(np.abs(want)))


def test_pairs_outside_windows_are_refused(qed):
    """Pairs that windows of eight sites cannot hold, or only with more than four
    windows, leave the sector to the staged kernels: the 7-wide ladder's t'
    diagonal (site x to x + 8), a ring's closing bond, and the 6-wide ladder's
    t' diagonal (site x to x + 7 for x = 0..4 needs a window starting at each x)."""
    pd, ps = lattice_pairs(7, 2, True)
    nw, y = qed.window_plan(14, 7, pd, ps, np.ones(len(pd)), np.ones(comb(14, 7)))
    assert nw == 0 and y is None
    ring_d = np.array([i for i in range(10)] + [(i + 1) % 10 for i in range(10)], np.int32)
    ring_s = np.array([(i + 1) % 10 for i in range(10)] + [i for i in range(10)], np.int32)
    nw, _ = qed.window_plan(10, 5, ring_d, ring_s, np.ones(20), np.ones(comb(10, 5)))
    assert nw == 0
    pd, ps = lattice_pairs(6, 2, True)
    nw, _ = qed.window_plan(12, 6, pd, ps, np.ones(len(pd)), np.ones(comb(12, 6)))
    assert nw == 0


def test_window_kernels_compile_without_spills(qed):
    """The 4x4 half-filled sector's kernels (groups of up to 70 strings held in
    registers) compile for sm_100a with no more than a few bytes of local-memory
    spill. They sit at the 255-register limit, where ptxas's allocation has varied
    by a few bytes between compiles of the same source; a register overflow of the
    generated code would spill hundreds."""
    pd, ps = lattice_pairs(4, 4, True)
    ok, log = qed.window_compile(16, 8, 8, pd, ps)
    assert ok, log
    for kernel in ("win_up_pass", "win_dn_pass"):
        assert kernel in log
    spills = [int(v) for v in re.findall(r"(\d+) bytes spill (?:stores|loads)", log)]
    assert spills and all(v <= 64 for v in spills), log
