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
  symmetric_orbitals  src_ed/symmetry_group.cpp:282-318 (real characters)
  destroy_matrix      Destroy (src_ed/ED_basis.cpp:62-78) and the destruction
                      operator of a symmetric orbital
                      (src_ed/Operators/destruction_operator.cpp:12-32)
  shift_irrep         symmetry_group::shift_sector (src_ed/symmetry_group.cpp:540-558)
  irrep_green_function the Lehmann Green function of one symmetric orbital by dense
                      diagonalisation (small sectors only)

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
    return dict(N=N, L=L, g=g, elems=elems, phi=phi, orders=orders)


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


def tensor(G, r1, r2):
    """Irrep product: digit-wise sum of the mixed-radix labels (Index(r1, r2))."""
    out, mult = 0, 1
    for n in G["orders"]:
        out += ((r1 % n + r2 % n) % n) * mult
        r1 //= n
        r2 //= n
        mult *= n
    return out


def conjugate(G, r):
    out, mult = 0, 1
    for n in G["orders"]:
        out += ((-(r % n)) % n) * mult
        r //= n
        mult *= n
    return out


def shift_irrep(G, r, pm, r_orb):
    return tensor(G, r, r_orb) if pm == 1 else tensor(G, r, conjugate(G, r_orb))


def symmetric_orbitals(G, n_sites):
    """Rows of S (real characters) and the irrep of each row, irreps in order."""
    g = G["g"]
    rows, irreps = [], []
    for r in range(g):
        covered = [False] * n_sites
        for site in range(n_sites):
            if covered[site]:
                continue
            covered[site] = True
            orb = np.zeros(n_sites)
            for e in range(g):
                t = G["elems"][e][site]
                covered[t] = True
                orb[t] += np.cos(2 * np.pi * G["phi"][r, e] / g)
            nrm = np.linalg.norm(orb)
            if nrm < 1e-12:
                continue
            rows.append(orb / nrm)
            irreps.append(r)
    return np.array(rows), irreps


def destroy_matrix(G, s_row, spin, basis_src, r_src, basis_tgt, r_tgt):
    """c of the symmetric orbital with site coefficients s_row (spin 0 up, 1 down),
    from the basis of irrep r_src to that of r_tgt, as a dense (D_tgt, D_src) array."""
    n, g = G["N"], G["g"]
    index = {b: i for i, b in enumerate(basis_tgt)}
    T = np.zeros((len(basis_tgt), len(basis_src)))
    for I, b in enumerate(basis_src):
        len_i = representative(G, b, r_src)[2]
        for site, coef in enumerate(s_row):
            if coef == 0.0:
                continue
            a = site + spin * n
            mask = 1 << (a - n + 32) if a >= n else 1 << a
            if not b & mask:
                continue
            rep, ph, ln = representative(G, b ^ mask, r_tgt)
            if ln == 0 or rep not in index:
                continue
            if bin(b & (mask - 1)).count("1") & 1:
                ph += g
            ph %= 2 * g
            T[index[rep], I] += (1.0 if ph == 0 else -1.0) * coef * np.sqrt(len_i / ln)
    return T


def irrep_green_function(prob, G, gs_sector, s_row, r_orb, z, spin=0):
    """G(z) of one symmetric orbital (row s_row of S, irrep r_orb) in the
    nondegenerate ground state of sector gs_sector, by dense diagonalisation of the
    ground-state and the two target sectors (creation and destruction)."""
    r0, N, S = (int(t[1:]) for t in gs_sector.split(":"))
    H0, B0 = mixed_hamiltonian(prob, G, gs_sector)
    e0, v0 = np.linalg.eigh(H0.toarray())
    E0, psi = e0[0], v0[:, 0]
    z = np.asarray(z, dtype=complex)
    out = np.zeros(len(z), dtype=complex)
    ds = -1 if spin else 1
    for pm in (1, -1):
        rt = shift_irrep(G, r0, pm, r_orb)
        sec = f"R{rt}:N{N + pm}:S{S + pm * ds}"
        Ht, Bt = mixed_hamiltonian(prob, G, sec)
        if Ht.shape[0] == 0:
            continue
        et, vt = np.linalg.eigh(Ht.toarray())
        if pm == 1:
            phi = destroy_matrix(G, s_row, spin, Bt, rt, B0, r0).T @ psi   # c+ psi
            w = (vt.T @ phi) ** 2
            out += (w[None, :] / (z[:, None] - (et[None, :] - E0))).sum(axis=1)
        else:
            phi = destroy_matrix(G, s_row, spin, B0, r0, Bt, rt) @ psi     # c psi
            w = (vt.T @ phi) ** 2
            out += (w[None, :] / (z[:, None] + (et[None, :] - E0))).sum(axis=1)
    return out, E0
