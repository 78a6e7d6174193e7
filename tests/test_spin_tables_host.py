"""One spin's tables as the solver builds them on the host (qed_spin_table_host:
the code that builds the small tables of every sector), against a numpy
statement of the reference's rules, bit for bit:

* strings: the N-subsets of L bits in increasing order (ED_halfbasis,
  src_ed/ED_basis.cpp:142-165);
* hops: for each string, the pairs (r, c) in row order of the one-body matrix
  (|t| of at least SMALL_VALUE, off the diagonal); c+_r c_c applies when bit c is
  set and bit r empty, reaches the string with r and c exchanged, with the parity
  of the set bits strictly between r and c (HS_half_operator,
  src_ed/Operators/HS_half_operator.hpp:17-45; binary_state::one_body,
  src_ed/binary_state.cpp:23-28); the value slot holds t[r][c] at an even index
  and -t[r][c] after it;
* diagonal: sum over the set bits r of t[r][r] + sum over the set bits c >= r of
  vsame[r][c], in that order.

The bank-ordered table (bank_order=True) has the same entries per string up to
their order, plus zero-valued padding."""
import numpy as np
import pytest


def lattice_t(nx, ny, rng, diagonal=True):
    L = nx * ny
    t = np.zeros((L, L))
    site = lambda x, y: x + nx * y
    for y in range(ny):
        for x in range(nx):
            nbrs = [(x + 1, y), (x, y + 1)] + ([(x + 1, y + 1), (x - 1, y + 1)] if diagonal else [])
            for (a, b) in nbrs:
                if 0 <= a < nx and 0 <= b < ny:
                    t[site(x, y), site(a, b)] = rng.choice([-1.0, -0.3, 0.45])
                    t[site(a, b), site(x, y)] = rng.choice([-1.0, -0.3, 0.45])
    t[np.diag_indices(L)] = rng.normal(size=L)
    return t


def numpy_tables(L, N, t, vsame):
    bits = [s for s in range(1 << L) if bin(s).count("1") == N]
    rank = {s: i for i, s in enumerate(bits)}
    pairs, vals, slot_of = [], [], {}
    for r in range(L):
        for c in range(L):
            v = t[r, c]
            if r == c or abs(v) < 1e-12:
                continue
            if v not in slot_of:
                slot_of[v] = len(vals)
                vals += [v, -v]
            pairs.append((r, c, slot_of[v]))
    width = min(len(pairs), N * (L - N))
    dim = len(bits)
    ell = np.zeros((width, dim), np.uint32)
    cnt = np.zeros(dim, np.uint8)
    diag = np.zeros(dim)
    for i, s in enumerate(bits):
        k = 0
        for (r, c, slot) in pairs:
            if not (s >> c) & 1 or (s >> r) & 1:
                continue
            ns = s ^ (1 << c) ^ (1 << r)
            lo, hi = min(r, c), max(r, c)
            between = ((1 << hi) - 1) & ~((2 << lo) - 1)
            sgn = bin(ns & between).count("1") & 1
            if k < width:
                ell[k, i] = (rank[ns] << 8) | (slot + sgn)
            k += 1
        cnt[i] = min(k, width)
        d = 0.0
        for r in range(L):
            if (s >> r) & 1:
                d += t[r, r]
                for c in range(r, L):
                    if (s >> c) & 1:
                        d += vsame[r, c]
        diag[i] = d
    return np.array(bits, np.uint32), cnt, diag, ell, np.array(vals)


@pytest.mark.parametrize("nx,ny,N,diagonal", [(3, 2, 3, True), (4, 2, 3, False), (2, 2, 0, True), (3, 3, 9, True)])
def test_host_tables_follow_the_reference_rules(qed, nx, ny, N, diagonal):
    rng = np.random.default_rng(nx * 10 + N)
    L = nx * ny
    t = lattice_t(nx, ny, rng, diagonal)
    vsame = np.triu(rng.normal(size=(L, L)))
    got = qed.spin_table_host(L, N, t, vsame, bank_order=False)
    bits, cnt, diag, ell, vals = numpy_tables(L, N, t, vsame)
    assert np.array_equal(got["bits"], bits)
    assert np.array_equal(got["cnt"], cnt)
    assert np.array_equal(got["diag"], diag)  # same summation order: bit-exact
    assert got["width"] == ell.shape[0]
    for i in range(len(bits)):  # entries past cnt[i] are unused
        assert np.array_equal(got["ell"][:cnt[i], i], ell[:cnt[i], i]), i
    assert np.array_equal(got["vals"], vals)


def test_bank_ordered_table_keeps_every_hop(qed):
    """The bank-ordered ELL (up spin of sectors of at least 64 strings) holds the
    same (target, value) hops per string, reordered, plus padding entries aimed at
    the value slot 0.0."""
    rng = np.random.default_rng(3)
    nx, ny, N = 4, 2, 4
    L = nx * ny
    t = lattice_t(nx, ny, rng, True)
    vsame = np.zeros((L, L))
    plain = qed.spin_table_host(L, N, t, vsame, bank_order=False)
    ordered = qed.spin_table_host(L, N, t, vsame, bank_order=True)
    # the plain width is the bound N (L - N); the ordered one the groups' step count
    assert len(plain["bits"]) == 70 and ordered["width"] >= int(plain["cnt"].max())
    vz = ordered["vals"]
    assert vz[-1] == 0.0 and np.array_equal(vz[:-1], plain["vals"])
    for i in range(70):
        a = sorted((int(e) >> 8, plain["vals"][int(e) & 255]) for e in plain["ell"][:plain["cnt"][i], i])
        b = [(int(e) >> 8, vz[int(e) & 255]) for e in ordered["ell"][:ordered["cnt"][i], i]]
        assert sorted(x for x in b if x[1] != 0.0) == a, i
