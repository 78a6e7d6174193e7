"""Lattice layer for VCA: the Potthoff (self-energy) functional of a lattice
tiled by one cluster, with the cluster solved by this package's GPU ED.

Mirrors the part of pyqcm's lattice layer that the variational cluster
approximation uses (pyqcm/__init__.py: cluster_model, cluster, lattice_model,
hopping_operator, interaction_operator, density_wave, set_target_sectors,
set_parameters, model_instance.Potthoff_functional, discrete_integration_grid,
set_wavevector_grid; src_qcm/lattice_model.cpp, src_qcm/lattice_model_instance.cpp,
src_qcm/CPT.cpp). Scope: one cluster without bath orbitals, one band, one-body
hoppings (tau = 1, sigma = 0), Hubbard interactions, density waves of types
Z and N, the chemical potential; the integral over frequencies and wavevectors
on a fixed grid (the reference's discrete-grid path). The (frequency, k) sum of
log|det(V(k) G(iw) - 1)| runs on the GPU (qed_sef_integrand_grid).

Conventions, as in the reference:
  * operator elements are consolidated (duplicates summed) per
    (site1, spin1, site2, spin2, superlattice neighbour),
    lattice_operator::consolidate (src_qcm/lattice_operator.cpp:196-237);
  * a hopping along `link` from site s1 lands on site s2 in the neighbouring
    super cell R (r_s1 + link = r_s2 + R . superlattice); it contributes
    (s1, s2, R) and (s2, s1, -R) (lattice_model::hopping_operator,
    src_qcm/lattice_model.cpp:968-1020);
  * V(k) = t(k) - t' with phases exp(2 pi i k.R), k in the superdual basis
    (set_V, src_qcm/CPT.cpp:22-64);
  * Omega = (omega_trace - omega_diag + omega_cluster) / n_sites
    (lattice_model_instance::Potthoff_functional, src_qcm/lattice_model_instance.cpp:503-590).
"""
from __future__ import annotations

import numpy as np

import pyqcm_b200 as qed

_grid = {"freqs": None, "weights": None, "nk": (32, 32, 1)}


def discrete_integration_grid(freqs, weights):
    """Frequencies (along the positive imaginary axis) and weights of the fixed-grid
    integral (pyqcm.discrete_integration_grid, pyqcm/__init__.py:3092-3115)."""
    _grid["freqs"] = np.ascontiguousarray(freqs, dtype=np.float64)
    _grid["weights"] = np.ascontiguousarray(weights, dtype=np.float64)


def set_wavevector_grid(nkx: int, nky: int, nkz: int = 1):
    """Number of wavevectors along each superdual direction (pyqcm.set_wavevector_grid)."""
    if min(nkx, nky, nkz) <= 0:
        raise ValueError("set_wavevector_grid: nkx, nky and nkz must all be strictly positive")
    _grid["nk"] = (int(nkx), int(nky), int(nkz))


def _resolve(params: dict, equiv) -> dict:
    """Independent values plus dependences name = multiplier * reference
    (parameter_set, src_qcm/parameter_set.cpp)."""
    out = dict(params)
    pending = list(equiv)
    for _ in range(len(pending) + 1):
        rest = []
        for name, mult, ref in pending:
            if ref in out:
                out[name] = mult * out[ref]
            else:
                rest.append((name, mult, ref))
        pending = rest
    if pending:
        raise ValueError(f"unresolved parameter dependences: {pending}")
    return out


class LatticeModel:
    """One-cluster lattice model (pyqcm's lattice_model with a single cluster)."""

    _count = 0

    def __init__(self, prob, cluster_model: str | None = None):
        self.prob = prob
        self.n = prob.n_sites
        self.n_bath = getattr(prob, "n_bath", 0)
        self.n_orb = self.n + self.n_bath
        self.dim = len(prob.superlattice)
        self.sites = np.array(prob.sites, dtype=np.int64)
        self.S = np.array(prob.superlattice, dtype=np.int64)  # rows: superlattice vectors
        LatticeModel._count += 1
        self.cluster_model = cluster_model or f"{prob.name}_clus{LatticeModel._count}"
        self.site_index = {tuple(int(c) for c in r): i for i, r in enumerate(self.sites)}
        # elements[op] = {(s1, spin1, s2, spin2, R): value}
        self.elements: dict[str, dict] = {}
        self.interactions = list(prob.interactions)
        self._add("mu", {(s, sp, s, sp, (0, 0, 0)): -1.0 for s in range(self.n) for sp in (0, 1)})
        for name, link, amp in prob.hoppings:
            self._hopping(name, np.asarray(link, dtype=np.int64), float(amp))
        for name, typ, Q in prob.density_waves:
            self._density_wave(name, typ, np.asarray(Q, dtype=np.float64))
        self._define_cluster_model()
        self.values = _resolve(prob.params, prob.equiv)
        self.mixing = 4 if any(self._spin_asymmetric(op) for op in self.elements) else 0

    # ---- geometry ------------------------------------------------------------
    def fold(self, p):
        """(site index, superlattice coordinates R) with p = r_site + R . superlattice."""
        d = self.dim
        St = self.S[:, :d].T.astype(np.float64)
        for s, r in enumerate(self.sites):
            diff = np.asarray(p, dtype=np.int64) - r
            if np.any(diff[d:] != 0):
                continue
            R = np.linalg.solve(St, diff[:d].astype(np.float64))
            Ri = np.rint(R)
            if np.allclose(R, Ri, atol=1e-9):
                out = np.zeros(3, dtype=np.int64)
                out[:d] = Ri.astype(np.int64)
                return s, tuple(int(x) for x in out)
        raise ValueError(f"lattice point {tuple(p)} is not covered by the cluster tiling")

    # ---- operators -----------------------------------------------------------
    def _add(self, name, el):
        E = self.elements.setdefault(name, {})
        for k, v in el.items():
            E[k] = E.get(k, 0.0) + v

    def _hopping(self, name, link, amp):
        el = {}
        for s1, r in enumerate(self.sites):
            s2, R = self.fold(r + link)
            Rm = tuple(-x for x in R)
            for sp in (0, 1):
                el[(s1, sp, s2, sp, R)] = el.get((s1, sp, s2, sp, R), 0.0) + amp
                el[(s2, sp, s1, sp, Rm)] = el.get((s2, sp, s1, sp, Rm), 0.0) + amp
        self._add(name, el)

    def _density_wave(self, name, typ, Q):
        # lattice_model::density_wave (src_qcm/lattice_model.cpp:1149-1230), phase 0, amplitude 1
        if typ not in ("Z", "spin", "N", "cdw"):
            raise ValueError(f"density wave of type {typ}: only Z and N are supported here")
        # Q (in units of pi) must be commensurate with the superlattice: Q.S even for
        # every superlattice vector S (the reference's check, src_qcm/lattice_model.cpp:1186-1190)
        for S in self.S:
            q = float(np.dot(Q, S))
            if abs(q / 2.0 - np.floor(q / 2.0 + 1e-6)) > 1e-5:
                raise ValueError(f"density-wave vector for {name} is incommensurate with the superlattice")
        el = {}
        for i, r in enumerate(self.sites):
            z = np.cos(np.pi * float(np.dot(Q, r)))
            if abs(z) <= 1e-8:
                continue
            el[(i, 0, i, 0, (0, 0, 0))] = z
            el[(i, 1, i, 1, (0, 0, 0))] = -z if typ in ("Z", "spin") else z
        self._add(name, el)

    def _spin_asymmetric(self, op):
        E = self.elements[op]
        for (s1, sp1, s2, sp2, R), v in E.items():
            if sp1 == 0 and abs(E.get((s1, 1, s2, 1, R), 0.0) - v) > 1e-14:
                return True
        return False

    def _define_cluster_model(self):
        """The cluster's ED model: its own operators (bath energies and
        hybridisations), then every lattice operator restricted to the cluster
        (neighbour 0), orbitals s (up) and s + n_orb (down), as the reference's
        lattice_model::build_cluster_operators names them."""
        no = self.n_orb
        qed.new_model(self.cluster_model, self.n, self.n_bath)
        for name, (typ, el) in getattr(self.prob, "cluster_operators", {}).items():
            qed.new_operator(self.cluster_model, name, typ, el)
        for name in self.interactions:
            qed.new_operator(self.cluster_model, name, "interaction", [(i, i + no, 1.0) for i in range(self.n)])
        for name, E in self.elements.items():
            el = [(s1 + no * sp1, s2 + no * sp2, v) for (s1, sp1, s2, sp2, R), v in sorted(E.items())
                  if R == (0, 0, 0) and abs(v) > 1e-12]
            if el:
                qed.new_operator(self.cluster_model, name, "one-body", el)

    # ---- one-body matrices ---------------------------------------------------
    def lattice_blocks(self, values: dict):
        """(H[spin], inter[spin]) for lattice parameter values: H the
        k-independent (neighbour 0) one-body matrix, inter the list of
        (r, c, R, v) elements across super cells."""
        n = self.n
        H = [np.zeros((n, n), dtype=np.complex128) for _ in range(2)]
        inter = [[], []]
        for name, E in self.elements.items():
            pv = values.get(name)
            if pv is None:
                continue
            for (s1, sp1, s2, sp2, R), v in E.items():
                if R == (0, 0, 0):
                    H[sp1][s1, s2] += v * pv
                else:
                    inter[sp1].append((s1, s2, R, v * pv))
        return H, inter

    def cluster_values(self, values: dict) -> dict:
        """ED instance values: cluster parameters (suffix _1), nonzero ones and mu
        (lattice_model_instance ctor, src_qcm/lattice_model_instance.cpp:57-66)."""
        out = {}
        for name, v in values.items():
            if name.endswith("_1"):
                op = name[:-2]
                if v != 0.0 or op == "mu":
                    out[op] = v
        return out

    def instance(self, label: int, **values) -> "LatticeInstance":
        vals = dict(self.prob.params)
        vals.update(values)
        return LatticeInstance(self, label, _resolve(vals, self.prob.equiv))


class LatticeInstance:
    """One parameter point: the cluster's ED instance (label) and the lattice values."""

    def __init__(self, model: LatticeModel, label: int, values: dict):
        self.model = model
        self.label = label
        self.values = values
        cv = model.cluster_values(values)
        if not cv:
            raise ValueError("system 0 has no nonzero operators")
        qed.new_model_instance(model.cluster_model, cv, model.prob.sectors, label)

    def erase(self):
        qed.erase_model_instance(self.label)

    def ground_state(self):
        return qed.ground_state_solve(self.label)

    def Green_function_solve(self):
        qed.Green_function_solve(self.label)

    def V_blocks(self):
        """Per spin block: (V0 = H - Hc, inter-cluster elements)."""
        H, inter = self.model.lattice_blocks(self.values)
        out = []
        for sd in range(2 if self.model.mixing == 4 else 1):
            Hc = qed.hopping_matrix(spin_down=bool(sd), label=self.label)
            out.append((H[sd] - Hc, inter[sd], H[sd], Hc))
        return out

    def V(self, k, spin_down=False):
        """V(k) for k in the superdual basis (set_V, src_qcm/CPT.cpp:22-64)."""
        V0, inter, _, _ = self.V_blocks()[1 if (spin_down and self.model.mixing == 4) else 0]
        kk = np.zeros(3)
        kk[:len(k)] = k
        Vk = V0.copy()
        for r, c, R, v in inter:
            Vk[r, c] += v * np.exp(2j * np.pi * float(np.dot(kk, R)))
        return Vk

    def sef_integrand(self, freqs, nk):
        """Per frequency: sum over spin blocks of 1/Nk sum_k log|det(V(k)G - 1)|
        (times 2 without spin asymmetry), on the GPU."""
        tot = np.zeros(len(freqs))
        blocks = self.V_blocks()
        for sd, (V0, inter, _, _) in enumerate(blocks):
            r = [e[0] for e in inter]
            c = [e[1] for e in inter]
            R = [e[2] for e in inter]
            v = [e[3] for e in inter]
            tot += qed.sef_integrand_grid(V0, r, c, R, v, freqs, nk, spin_down=bool(sd), label=self.label)
        if len(blocks) == 1:
            tot *= 2.0
        return tot

    def Potthoff_functional(self, freqs=None, weights=None, nk=None) -> float:
        """Omega per site on the fixed (frequency, k) grid
        (lattice_model_instance::Potthoff_functional, src_qcm/lattice_model_instance.cpp:503-590)."""
        freqs = _grid["freqs"] if freqs is None else np.asarray(freqs, dtype=np.float64)
        weights = _grid["weights"] if weights is None else np.asarray(weights, dtype=np.float64)
        nk = _grid["nk"] if nk is None else nk
        if freqs is None:
            raise ValueError("no frequency grid: call discrete_integration_grid first")
        omega_clus = qed.Potthoff_functional(self.label)
        I = self.sef_integrand(freqs, nk)
        omega_trace = -float(np.dot(I, weights))
        blocks = self.V_blocks()
        omega_diag = 0.0
        for _, _, H, Hc in blocks:
            omega_diag -= float(np.real(np.trace(H - Hc)))
        if len(blocks) == 1:
            omega_diag *= 2.0
        omega_diag *= 0.5
        return (omega_trace - omega_diag + omega_clus) / self.model.n


# -------------------------------------------------------------------- CDMFT --

def _blocks(model):
    return (False, True) if model.mixing == 4 else (False,)


def projected_green_function(inst: LatticeInstance, freqs, side: int = 32, spin_down: bool = False):
    """Grid average of the CPT Green function per frequency (projected_Green_function,
    src_qcm/CPT.cpp:283-346): side points per superlattice direction at offsets
    (i + 0.5)/side; with bath orbitals V(k) carries -Gamma(iw) of the cluster."""
    freqs = np.asarray(freqs, dtype=np.float64)
    m = inst.model
    H, inter = m.lattice_blocks(inst.values)
    sd = 1 if (spin_down and m.mixing == 4) else 0
    Hc = qed.hopping_matrix(spin_down=bool(sd), label=inst.label)
    V0 = np.repeat((H[sd] - Hc)[None, :, :], len(freqs), axis=0).astype(np.complex128)
    if m.n_bath:
        V0 -= qed.hybridization_function(1j * freqs, spin_down=bool(sd), label=inst.label)
    el = inter[sd]
    nk = [side if i < m.dim else 1 for i in range(3)]
    return qed.cpt_projected_green_function(V0, [e[0] for e in el], [e[1] for e in el], [e[2] for e in el],
                                            [e[3] for e in el], freqs, nk, 0.5, spin_down=bool(sd),
                                            label=inst.label)


def CDMFT_host(inst: LatticeInstance, freqs, side: int = 32):
    """Host function per spin block and frequency (lattice_model_instance::CDMFT_host,
    src_qcm/CPT.cpp:356-425): G_host = Gproj^{-1} + Sigma_c(iw) + H_c - iw."""
    freqs = np.asarray(freqs, dtype=np.float64)
    out = []
    for sd in _blocks(inst.model):
        P = projected_green_function(inst, freqs, side, spin_down=sd)
        S = qed.self_energy(1j * freqs, spin_down=sd, label=inst.label)
        Hc = qed.hopping_matrix(spin_down=sd, label=inst.label)
        eye = np.eye(inst.model.n)
        out.append(np.linalg.inv(P) + S + Hc[None] - 1j * freqs[:, None, None] * eye[None])
    return out


def CDMFT_distance(model: LatticeModel, host, freqs, weights, varia, points, base_values, label0: int = 800000):
    """Distance of the cluster hybridisation to the host for a batch of bath
    points (lattice_model_instance::CDMFT_distance, src_qcm/CPT.cpp:519-560):
    sum over frequencies and spin blocks of weight * |Gamma(iw) + G_host(iw)|^2,
    doubled without spin asymmetry, times the frequency step, over dim^2. The
    hybridisation needs no ground state: each point is only an ED instance."""
    freqs = np.asarray(freqs, dtype=np.float64)
    weights = np.asarray(weights, dtype=np.float64)
    dw = freqs[1] - freqs[0]
    dim = model.n
    out = []
    for k, p in enumerate(np.atleast_2d(points)):
        vals = dict(base_values)
        vals.update({v: float(x) for v, x in zip(varia, p)})
        inst = model.instance(label0 + k, **vals)
        try:
            d = 0.0
            for h, sd in zip(host, _blocks(model)):
                g = qed.hybridization_function(1j * freqs, spin_down=sd, label=inst.label)
                d += float(np.sum(weights[:, None, None] * np.abs(g + h) ** 2))
        finally:
            inst.erase()
        if model.mixing == 0:
            d *= 2.0
        out.append(d * dw / (dim * dim))
    return np.array(out)
