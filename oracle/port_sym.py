"""CPU oracle, symmetry part: a numpy restatement of the reference's cluster point
group and of its Hamiltonian in the symmetry-adapted (mixed) basis.

TEST INFRASTRUCTURE ONLY -- used by tests/ to cross-check the compiled reference
and the product on small cases; written for readability, not speed.

  group               src_ed/symmetry_group.cpp:17-345 (elements in mixed-radix
                      order, character phases phi = sum_k a_k b_k g / n_k mod g)
  representative      src_ed/symmetry_group.cpp:118-150, 231-262
  mixed_basis         src_ed/ED_basis.cpp:185-385 (unmixed N, S sectors)
  mixed_hamiltonian   src_ed/Operators/HS_one_body_operator.hpp:17-37 and
                      src_ed/Operators/HS_interaction_operator.hpp:32-54 on that basis

States are 64-bit ints, spin up in bits 0..31, spin down in bits 32..63.
Phases are integers in units of pi / g.
"""
from __future__ import annotations

import itertools

import numpy as np
import scipy.sparse as sp


def group(n_sites, n_bath, gens0, bath_irrep):
    """gens0: generators 0-based, as ED::new_model takes them. Returns a dict
    with N, L, g, the elements (g lists of N ints) and phi (g x g)."""
    N = n_sites + n_bath
    bath_irrep = bool(bath_irrep) and bool(gens0)
    L = n_sites if bath_irrep else N
    gens = [list(x) for x in gens0] or [list(range(N))]

    def prod(x, y, g):
        return [x[y[i]] for i in range(L)] + [(x[i] + y[i]) % g for i in range(L, N)]

    ident = list(range(L)) + [0] * (N - L)
    orders = []
    for x in gens:
        p, n = ident, 1
        while True:
            p = prod(p, x, 1)
            if p[:L] == ident[:L]:
                break
            n += 1
        orders.append(n)
    g = int(np.prod(orders))

    def digits(k):
        d = []
        for n in orders:
            d.append(k % n)
            k //= n
        return d

    elems = []
    for k in range(g):
        p = ident
        for j, c in enumerate(digits(k)):
            for _ in range(c):
                p = prod(p, gens[j], g)
        elems.append(p)
    phi = np.zeros((g, g), dtype=int)
    for a in range(g):
        for b in range(g):
            da, db = digits(a), digits(b)
            phi[a, b] = sum(da[k] * db[k] * g // orders[k] for k in range(len(orders))) % g
    return dict(N=N, L=L, g=g, elems=elems, phi=phi)


def _apply_half(G, e, b):
    v = G["elems"][e]
    out, phase, q = 0, 0, []
    for i in range(G["L"]):
        if b >> i & 1:
            out |= 1 << v[i]
            q.append(v[i])
    for i in range(G["L"], G["N"]):
        if b >> i & 1:
            out |= 1 << i
            phase += 2 * v[i]
    inv = sum(1 for a, c in itertools.combinations(q, 2) if a > c)
    if inv % 2:
        phase += G["g"]
    return out, phase


def representative(G, b, r):
    """(rep, phase, length) of state b in irrep r; length 0 for a null state."""
    g = G["g"]
    rep, ph, h = b, 0, 1
    for e in range(1, g):
        up, p1 = _apply_half(G, e, b & 0xFFFFFFFF)
        dn, p2 = _apply_half(G, e, b >> 32)
        x = up | dn << 32
        q = (p1 + p2 + 2 * G["phi"][e, r]) % (2 * g)
        if x == b:
            h += 1
            if q != 0 and (2 * g) % q == 0:
                return rep, ph, 0
        if x < rep:
            rep, ph = x, q
    return rep, ph, g // h


def mixed_basis(G, r, n_up, n_dn):
    N = G["N"]
    ups = [b for b in range(1 << N) if bin(b).count("1") == n_up]
    dns = [b for b in range(1 << N) if bin(b).count("1") == n_dn]
    out = []
    for u in ups:
        for d in dns:
            b = u | d << 32
            rep, _, ln = representative(G, b, r)
            if ln and rep == b:
                out.append(b)
    return sorted(out)


def _mask(i, n):
    return 1 << (i - n + 32) if i >= n else 1 << i


def _between_sign(b, m1, m2):
    if m1 == m2:
        return 1
    lo, hi = min(m1, m2), max(m1, m2)
    inside = hi - (lo << 1)
    return -1 if bin(inside & b).count("1") & 1 else 1


def mixed_hamiltonian(prob, G, sector):
    """Sparse H of sector 'R<r>:N<N>:S<S>' in the mixed basis: for each basis state
    I and each one-body element (r, c, v) of the Hermitian-completed list,
    c+_r c_c |I> reaches the representative J with matrix element
    value * v * fermion sign * (-1 if the representative's phase else 1) *
    sqrt(len_I / len_J), added at (J, I); diagonal one-body and interaction
    elements as in the factorized basis, on b = up | dn << 32."""
    r_irrep, N, S = (int(t[1:]) for t in sector.split(":"))
    n = G["N"]
    basis = mixed_basis(G, r_irrep, (N + S) // 2, (N - S) // 2)
    index = {b: i for i, b in enumerate(basis)}
    D = len(basis)
    rows, cols, vals = [], [], []
    diag = np.zeros(D)
    for name, val in prob.params.items():
        if name not in prob.operators:
            continue
        typ, el = prob.operators[name]
        if typ == "one-body":
            full = []
            for (r, c, v) in el:
                if r < c:
                    full += [(r, c, v), (c, r, v)]
                elif r == c:
                    full.append((r, c, v))
            for I, b in enumerate(basis):
                lenI = representative(G, b, r_irrep)[2]
                for (r, c, v) in full:
                    if r == c:
                        if b & _mask(r, n):
                            diag[I] += val * v
                        continue
                    mc, mr = _mask(c, n), _mask(r, n)
                    if not (b & mc) or (b & mr):
                        continue
                    bp = b - mc + mr
                    sign = _between_sign(b, mc, mr)
                    rep, ph, ln = representative(G, bp, r_irrep)
                    J = index.get(rep)
                    if J is None:
                        continue
                    x = (-1.0 if ph else 1.0) * val * v * sign * np.sqrt(lenI / ln)
                    rows.append(J)
                    cols.append(I)
                    vals.append(x)
        else:
            for (r, c, v) in el:
                m = _mask(r, n) + _mask(c, n)
                for I, b in enumerate(basis):
                    if b & m == m:
                        diag[I] += val * v
    H = sp.coo_matrix((vals, (rows, cols)), shape=(D, D)).tocsr() + sp.diags(diag)
    return H.tocsr(), np.array(basis, dtype=np.uint64)
