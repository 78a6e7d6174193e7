"""CPU oracle, part 2: a numpy/scipy restatement of the reference's ED path.

TEST INFRASTRUCTURE ONLY -- used by tests/ (to cross-check the compiled
reference and the product on small cases) and as the "port" CPU baseline.
It is written for readability at small sizes, not speed.

Each function follows the reference routine it cites:
  halfbasis / rank        src_ed/ED_basis.cpp:115-135 (sorted N-of-L strings, index = position)
  hop_matrix              src_ed/Operators/HS_half_operator.hpp:17-45 + binary_state.hpp:42-63
  diag_terms              src_ed/Operators/HS_interaction_operator.hpp:32-54 (mask-sum convention)
  sector_hamiltonian      src_ed/Operators/HS_factorized_operator.hpp:56-84 (x[up + du*dn])
  lanczos_ground_state    src_ed/Hamiltonian/Lanczos.hpp:41-143
  lanczos_green           src_ed/Hamiltonian/Lanczos.hpp:156-183
  band_lanczos            src_ed/Hamiltonian/Lanczos.hpp:214-395 + Hamiltonian_base.hpp:229-254
  cdag                    src_ed/model.cpp:160-180 with Destroy (src_ed/ED_basis.cpp:79-110)
  streamline / check_norm src_ed/Q_matrix.hpp:181-318
  solve                   src_ed/model_instance.hpp:245-347, 517-555, 711-817; model_instance.cpp:34-99
"""
from __future__ import annotations

import itertools
import math

import numpy as np
import scipy.linalg as sla
import scipy.sparse as sp

SMALL = 1e-12

DEFAULTS = dict(accur_lanczos=1e-12, max_iter_lanczos=1000, max_iter_BL=600, accur_band_lanczos=1e-12,
                accur_deflation=1e-7, max_iter_CF=400, accur_continued_fraction=0.01,
                Qmatrix_wtol=1e-5, Qmatrix_vtol=1e-10, accur_Q_matrix=1e-5)


# ---------------------------------------------------------------- basis ----

def halfbasis(L: int, N: int) -> np.ndarray:
    if N < 0 or N > L:
        return np.zeros(0, dtype=np.uint32)
    s = [sum(1 << p for p in c) for c in itertools.combinations(range(L), N)]
    return np.array(sorted(s), dtype=np.uint32)


def rank(b: int) -> int:
    """Colex rank sum_k C(p_k, k+1) over set bits p_0 < p_1 < ... (= sorted position)."""
    r, k = 0, 1
    p = 0
    while b:
        if b & 1:
            r += math.comb(p, k)
            k += 1
        b >>= 1
        p += 1
    return r


def popcount(x: int) -> int:
    return bin(x).count("1")


# ------------------------------------------------------------ operators ----

def collect_terms(prob):
    """Total one-body matrix per spin and the diagonal interaction terms, as masks.

    Interaction elements (r, c, v) are evaluated on b = dn | (up << 32) with the
    reference's literal mask(r) + mask(c), mask(i) = bit i (i < n) else bit i-n+32."""
    n = prob.n_orb
    t_up = np.zeros((n, n))
    t_dn = np.zeros((n, n))
    inter = []  # (v, mask64)
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
            for (r, c, v) in full:
                if r < n and c < n:
                    t_up[r, c] += val * v
                elif r >= n and c >= n:
                    t_dn[r - n, c - n] += val * v
                else:
                    raise ValueError("spin-flip term")
        else:
            for (r, c, v) in el:
                r, c = min(r, c), max(r, c)
                mk = lambda i: (1 << (i - n + 32)) if i >= n else (1 << i)
                inter.append((val * v, mk(r) + mk(c)))
    return t_up, t_dn, inter


def hop_matrix(L, N, t):
    """Sparse one-spin operator sum t[r][c] c^+_r c_c on the N-of-L strings."""
    B = halfbasis(L, N)
    d = len(B)
    rows, cols, vals = [], [], []
    diag = np.zeros(d)
    for I, b in enumerate(B.tolist()):
        for r in range(L):
            if (b >> r) & 1:
                diag[I] += t[r, r]
        for r in range(L):
            for c in range(L):
                if r == c or abs(t[r, c]) < SMALL:
                    continue
                if not ((b >> c) & 1) or ((b >> r) & 1):
                    continue
                nb = b ^ (1 << c) ^ (1 << r)
                lo, hi = min(r, c), max(r, c)
                between = ((1 << hi) - 1) & ~((2 << lo) - 1)
                sgn = -1.0 if popcount(nb & between) & 1 else 1.0
                rows.append(rank(nb))
                cols.append(I)
                vals.append(sgn * t[r, c])
    T = sp.csr_matrix((vals, (rows, cols)), shape=(d, d)) + sp.diags(diag)
    return T.tocsr(), B


def diag_terms(Bu, Bd, inter):
    du, dd = len(Bu), len(Bd)
    D = np.zeros((dd, du))
    up = Bu.astype(np.uint64)[None, :]
    dn = Bd.astype(np.uint64)[:, None]
    b = dn | (up << np.uint64(32))
    for v, m in inter:
        m = np.uint64(m)
        D += v * ((b & m) == m)
    return D.reshape(-1)


def sector_hamiltonian(prob, n_up, n_dn):
    L = prob.n_orb
    t_up, t_dn, inter = collect_terms(prob)
    Tu, Bu = hop_matrix(L, n_up, t_up)
    Td, Bd = hop_matrix(L, n_dn, t_dn)
    du, dd = len(Bu), len(Bd)
    H = sp.kron(Td, sp.identity(du)) + sp.kron(sp.identity(dd), Tu) + sp.diags(diag_terms(Bu, Bd, inter))
    return H.tocsr(), Bu, Bd


# --------------------------------------------------------------- Krylov ----

def _tridiag_lowest(alpha, beta):
    if len(alpha) == 1:
        return alpha[0], np.array([1.0])
    w, v = sla.eigh_tridiagonal(np.array(alpha), np.array(beta[:-1]))
    return w[0], v[:, 0]


def lanczos_ground_state(H, x0, opt=DEFAULTS):
    r = x0 / np.linalg.norm(x0)
    start = r.copy()
    q = np.zeros_like(r)
    alpha, beta = [], []
    ritz = 2 * opt["accur_lanczos"]
    while ritz > opt["accur_lanczos"]:
        if beta:
            r = r / beta[-1]
            q = -beta[-1] * q
        q = q + H @ r
        r, q = q, r
        a = q @ r
        alpha.append(a)
        r = r - a * q
        beta.append(np.linalg.norm(r))
        e0, ev = _tridiag_lowest(alpha, beta)
        ritz = abs(ev[-1] * beta[-1])
        if len(alpha) > opt["max_iter_lanczos"]:
            raise RuntimeError("Lanczos procedure exceeded the iteration cap")
    e0, ev = _tridiag_lowest(alpha, beta)
    gs = ev[0] * start
    r, q = start.copy(), np.zeros_like(start)
    for j in range(1, len(ev)):
        q = q + H @ r - alpha[j - 1] * r
        r, q = q / beta[j - 1], -beta[j - 1] * r
        gs = gs + ev[j] * r
    return e0, gs


def lanczos_green(H, psi, opt=DEFAULTS):
    q = np.zeros_like(psi)
    a, b = [], [1.0]
    prod = 1.0
    while prod > opt["accur_continued_fraction"] and abs(b[-1]) > opt["accur_continued_fraction"] \
            and len(a) < opt["max_iter_CF"]:
        if a:
            psi, q = q / b[-1], -b[-1] * psi
        q = q + H @ psi
        z = psi @ q
        a.append(z)
        q = q - z * psi
        zz = np.linalg.norm(q)
        b.append(zz)
        prod *= abs(zz)
    return a, b


def band_lanczos(H, phi, opt=DEFAULTS):
    """Returns (eigenvalues, Q = P[:, :p] U[:p, :]) or None."""
    p = len(phi)
    dim = H.shape[0]
    M0 = int(14 * p * math.log(1.0 * dim))
    assert M0 > 1
    pc = p
    M0 = min(M0, opt["max_iter_BL"])
    M0p = (M0 // p + 1) * p
    M0 = M0p - pc
    v = [None] * (M0p + 1)
    t = np.zeros((M0, M0))
    P = np.zeros((p, max(M0, 1)))
    defl = [0] * (M0 + 1)
    I = []
    for i in range(p):
        v[i] = phi[i].copy()
    ev_old = 1e12
    j = 0
    while j < M0:
        z = np.linalg.norm(v[j])
        if z < opt["accur_deflation"]:
            if j >= pc:
                I.append(j - pc)
                defl[j - pc] = 1
            pc -= 1
            if pc == 0:
                break
            for k in range(j, j + pc):
                v[k] = v[k + 1]
            v[j + pc] = None
            continue
        v[j] = v[j] / z
        if j >= pc:
            t[j, j - pc] = z
        for k in range(p):
            P[k, j] = phi[k] @ v[j]
        for k in range(j + 1, j + pc):
            zz = v[j] @ v[k]
            v[k] = v[k] - zz * v[j]
            if k >= pc:
                t[j, k - pc] = zz
        v[j + pc] = H @ v[j]
        k0 = 0
        if j > pc:
            k0 = j - pc
            if defl[k0 - 1] == 0:
                v[k0 - 1] = None
        for k in range(k0, j):
            t[k, j] = t[j, k]
            v[j + pc] = v[j + pc] - t[k, j] * v[k]
        for k in I:
            w = v[k] @ v[j + pc]
            v[j + pc] = v[j + pc] - w * v[k]
            t[k, j] = w
        w = v[j] @ v[j + pc]
        v[j + pc] = v[j + pc] - w * v[j]
        t[j, j] = w
        for k in I:
            t[j, k] = t[k, j]
        if j >= 4 * p and j % p == 0:
            ev = np.linalg.eigvalsh(t[:j, :j])
            test = abs(ev[0] - ev_old)
            ev_old = ev[0]
            if test < opt["accur_band_lanczos"]:
                break
        j += 1
    if j == 0:
        return None
    w, U = np.linalg.eigh(t[:j, :j])
    kmax = min(p, j)
    return w, P[:, :kmax] @ U[:kmax, :]


def cdag(psi, L, sec_nup, sec_ndn, pm, spin, orb):
    """c^{pm}_{orb,spin} |psi> on the factorized basis of sector (n_up, n_dn)."""
    Bu, Bd = halfbasis(L, sec_nup), halfbasis(L, sec_ndn)
    tnu = sec_nup + (pm if spin == 0 else 0)
    tnd = sec_ndn + (pm if spin == 1 else 0)
    Tu, Td = halfbasis(L, tnu), halfbasis(L, tnd)
    du_s, du_t = len(Bu), len(Tu)
    y = np.zeros(len(Tu) * len(Td))
    bit = 1 << orb
    for d, dn in enumerate(Td.tolist()):
        for u, up in enumerate(Tu.tolist()):
            if spin == 0:
                occ = bool(up & bit)
                if (pm < 0 and occ) or (pm > 0 and not occ):
                    continue
                s = up ^ bit
                ph = popcount((s if pm < 0 else up) & (bit - 1)) & 1
                src = rank(s) + du_s * d
            else:
                occ = bool(dn & bit)
                if (pm < 0 and occ) or (pm > 0 and not occ):
                    continue
                s = dn ^ bit
                ph = (popcount((s if pm < 0 else dn) & (bit - 1)) + popcount(up)) & 1
                src = u + du_s * rank(s)
            y[u + du_t * d] = -psi[src] if ph else psi[src]
    return y


def streamline(e, V, opt=DEFAULTS):
    wtol, vtol = opt["Qmatrix_wtol"], opt["Qmatrix_vtol"]
    L = V.shape[0]
    e2, cols = [], []
    i = 0
    M = len(e)
    while i < M:
        j = i + 1
        while j < M and abs(e[j] - e[i]) <= wtol:
            j += 1
        if j - i == 1:
            if V[:, i] @ V[:, i] >= vtol:
                e2.append(e[i])
                cols.append(V[:, i])
        else:
            QQ = V[:, i:j] @ V[:, i:j].T
            d, U = np.linalg.eigh(QQ)
            for k in range(L):
                if d[k] > vtol:
                    e2.append(e[i])
                    cols.append(U[:, k] * math.sqrt(d[k]))
        i = j
    return np.array(e2), (np.array(cols).T if cols else np.zeros((L, 0)))


# ---------------------------------------------------------------- driver ----

def parse_sector(s):
    N = int(s.split("N")[1].split(":")[0])
    S = int(s.split("S")[1].split(":")[0])
    return N, S


def solve(prob, gf_method="L", seed=0, opt=DEFAULTS):
    """Ground state over the listed sectors (T = 0) and the Green-function data.
    Returns dict(E0, sector, states=[(N, S, energy, weight, psi)], gf=...)."""
    L = prob.n_orb
    rng = np.random.default_rng(seed)
    found = []
    for s in prob.sectors.split("/"):
        N, S = parse_sector(s)
        nu, nd = (N + S) // 2, (N - S) // 2
        if nu > L or nd > L or nu < 0 or nd < 0:
            continue
        H, Bu, Bd = sector_hamiltonian(prob, nu, nd)
        e, psi = lanczos_ground_state(H, rng.standard_normal(H.shape[0]), opt)
        found.append((N, S, e, psi))
    emin = min(f[2] for f in found)
    states = [f for f in found if f[2] - emin <= SMALL]
    w = 1.0 / len(states)
    out = dict(E0=emin, states=[], gf_method=gf_method)
    up_down = any(S != 0 for (_, S, _, _) in states) or _has_up_down(prob)
    for (N, S, e, psi) in states:
        nu, nd = (N + S) // 2, (N - S) // 2
        entry = dict(N=N, S=S, energy=e, weight=w, psi=psi, gf={})
        for spin in ([0, 1] if up_down else [0]):
            entry["gf"][spin] = (_qmatrix if gf_method == "L" else _cf)(prob, nu, nd, e, w, psi, spin, opt)
        out["states"].append(entry)
    out["up_down"] = up_down
    return out


def _has_up_down(prob):
    t_up, t_dn, _ = collect_terms(prob)
    return not np.array_equal(t_up, t_dn)


def _target(prob, nu, nd, pm, spin):
    return (nu + pm, nd) if spin == 0 else (nu, nd + pm)


def _qmatrix(prob, nu, nd, e0, w, psi, spin, opt):
    L, p = prob.n_orb, prob.n_sites
    es, Vs = [], []
    for pm in (-1, 1):
        tnu, tnd = _target(prob, nu, nd, pm, spin)
        if not (0 <= tnu <= L and 0 <= tnd <= L):
            es.append(np.zeros(0)); Vs.append(np.zeros((p, 0)))
            continue
        H, _, _ = sector_hamiltonian(prob, tnu, tnd)
        phi = [cdag(psi, L, nu, nd, pm, spin, i) for i in range(p)]
        r = band_lanczos(H, phi, opt)
        if r is None:
            es.append(np.zeros(0)); Vs.append(np.zeros((p, 0)))
            continue
        ev, Q = r
        e = ev - e0
        if pm == -1:
            e = -e
        e, Q = streamline(e, Q, opt)
        es.append(e)
        Vs.append(Q)
    e = np.concatenate(es)
    V = np.concatenate(Vs, axis=1)
    return ("Q", e, V * math.sqrt(w))


def _cf(prob, nu, nd, e0, w, psi, spin, opt):
    L, n = prob.n_orb, prob.n_sites
    frac = {}
    for pm in (-1, 1):
        tnu, tnd = _target(prob, nu, nd, pm, spin)
        if not (0 <= tnu <= L and 0 <= tnd <= L):
            continue
        H, _, _ = sector_hamiltonian(prob, tnu, tnd)
        for o1 in range(n):
            for o2 in range(o1 + 1):
                x = cdag(psi, L, nu, nd, pm, spin, o1)
                if o1 != o2:
                    x = x + cdag(psi, L, nu, nd, pm, spin, o2)
                nrm = x @ x
                if nrm <= 1e-14:
                    continue
                a, b = lanczos_green(H, x / math.sqrt(nrm), opt)
                b = [bb * bb for bb in b]
                b[0] = nrm * w
                a = [ai - e0 for ai in a] if pm == 1 else [-ai + e0 for ai in a]
                frac[(o1, o2, pm)] = (np.array(a), np.array(b))
    return ("CF", frac, n)


def cf_eval(a, b, z):
    G = np.zeros_like(z)
    for i in range(len(a) - 1, -1, -1):
        G = b[i] / (z - a[i] - G)
    return G


def green_function(sol, z, spin_down=False):
    z = np.atleast_1d(np.asarray(z, dtype=complex))
    spin = 1 if (spin_down and sol["up_down"]) else 0
    G = None
    for st in sol["states"]:
        kind = st["gf"][spin]
        if kind[0] == "Q":
            _, e, V = kind
            D = 1.0 / (z[:, None] - e[None, :])
            g = np.einsum("ai,ki,bi->kab", V, D, V)
        else:
            _, frac, n = kind
            g = np.zeros((len(z), n, n), dtype=complex)
            ev = lambda o1, o2: sum(cf_eval(*frac[(o1, o2, pm)], z) for pm in (-1, 1) if (o1, o2, pm) in frac)
            gt = [ev(o, o) if any((o, o, pm) in frac for pm in (-1, 1)) else np.zeros_like(z) for o in range(n)]
            for o1 in range(n):
                g[:, o1, o1] += gt[o1]
                for o2 in range(o1):
                    e12 = ev(o1, o2) if any((o1, o2, pm) in frac for pm in (-1, 1)) else np.zeros_like(z)
                    tmp = 0.5 * (e12 - gt[o1] - gt[o2])
                    g[:, o1, o2] += tmp
                    g[:, o2, o1] += tmp
        G = g if G is None else G + g
    return G
