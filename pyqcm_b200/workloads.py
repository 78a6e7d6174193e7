"""Cluster-model builders for the synthetic workloads this solver is measured on.

Each builder returns a plain description (orbital counts, operator element
lists, parameter values, sector string) that can be fed to either this
package's ED API or the CPU oracle, so both solve the identical problem.

Conventions follow the reference's cluster-model definitions:
  * orbital index i < n_orb is spin up, i + n_orb is spin down
    (src_ed/model.hpp:34-41, src_ed/binary_state.hpp:60-63);
  * a one-body element (r, c, v) means v c^+_r c_c, given with r <= c; the
    Hermitian partner is added by the solver (src_ed/Operators/one_body_operator.hpp:63-71);
  * an interaction element (r, c, v) means v n_r n_c (src_ed/Operators/HS_interaction_operator.hpp:44-53);
  * the chemical potential enters as -mu * N (diagonal elements -1), so mu = U/2
    is half filling for a bipartite cluster.
All indices here are 0-based.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class ClusterProblem:
    name: str
    n_sites: int
    n_bath: int
    operators: dict = field(default_factory=dict)   # name -> (type, [(r, c, v), ...])
    params: dict = field(default_factory=dict)      # name -> value
    sectors: str = "R0"
    generators: list | None = None   # pyqcm's symmetry generators (1-based sites)
    bath_irrep: bool = False

    @property
    def n_orb(self) -> int:
        return self.n_sites + self.n_bath


def _both_spins(n_orb, pairs):
    out = []
    for (r, c, v) in pairs:
        out.append((r, c, v))
        out.append((r + n_orb, c + n_orb, v))
    return out


def lattice_bonds(nx: int, ny: int, diagonal: bool = False):
    """Open-boundary nx x ny cluster: site index x + nx*y. Returns (nn, nnn) bond lists."""
    nn, nnn = [], []
    for y in range(ny):
        for x in range(nx):
            i = x + nx * y
            if x + 1 < nx:
                nn.append((i, i + 1))
            if y + 1 < ny:
                nn.append((i, i + nx))
            if diagonal and x + 1 < nx and y + 1 < ny:
                nnn.append((i, i + nx + 1))
            if diagonal and x > 0 and y + 1 < ny:
                nnn.append((i, i + nx - 1))
    return nn, nnn


def hubbard_cluster(nx: int, ny: int, t: float = -1.0, tp: float | None = None, U: float = 4.0,
                    mu: float | None = None, M: float | None = None, n_up: int | None = None,
                    n_dn: int | None = None, name: str | None = None) -> ClusterProblem:
    """Hubbard model on an open nx x ny cluster (chains: ny = 1).

    Operators: 't' (nearest-neighbour hop), optional "t'" (next-nearest), 'U'
    (on-site), 'mu' (-N), optional 'M' (staggered Neel field, +1 up / -1 down on
    sublattice A and the opposite on B, which makes the two spins different).
    """
    L = nx * ny
    nn, nnn = lattice_bonds(nx, ny, diagonal=tp is not None)
    prob = ClusterProblem(name or f"hub{nx}x{ny}", L, 0)
    prob.operators["t"] = ("one-body", _both_spins(L, [(a, b, 1.0) for a, b in nn]))
    if tp is not None and nnn:
        prob.operators["tp"] = ("one-body", _both_spins(L, [(a, b, 1.0) for a, b in nnn]))
        prob.params["tp"] = tp
    prob.operators["U"] = ("interaction", [(i, i + L, 1.0) for i in range(L)])
    prob.operators["mu"] = ("one-body", _both_spins(L, [(i, i, -1.0) for i in range(L)]))
    prob.params.update({"t": t, "U": U, "mu": U / 2 if mu is None else mu})
    if M is not None:
        el = []
        for y in range(ny):
            for x in range(nx):
                i = x + nx * y
                s = 1.0 if (x + y) % 2 == 0 else -1.0
                el.append((i, i, s))
                el.append((i + L, i + L, -s))
        prob.operators["M"] = ("one-body", el)
        prob.params["M"] = M
    nu = L // 2 if n_up is None else n_up
    nd = L // 2 if n_dn is None else n_dn
    prob.sectors = f"R0:N{nu + nd}:S{nu - nd}"
    return prob


def plaquette_bath(eps, hyb, U: float = 8.0, t: float = -1.0, mu: float | None = None,
                   name: str = "plaq8b") -> ClusterProblem:
    """2x2 plaquette with 8 bath orbitals, two per cluster site.

    eps[b] is the energy of bath orbital b, hyb[b] its hybridisation with
    cluster site b // 2. Orbitals 0-3 are the plaquette, 4-11 the bath.
    """
    ns, nb = 4, 8
    L = ns + nb
    nn, _ = lattice_bonds(2, 2)
    prob = ClusterProblem(name, ns, nb)
    prob.operators["t"] = ("one-body", _both_spins(L, [(a, b, 1.0) for a, b in nn]))
    prob.operators["U"] = ("interaction", [(i, i + L, 1.0) for i in range(ns)])
    prob.operators["mu"] = ("one-body", _both_spins(L, [(i, i, -1.0) for i in range(ns)]))
    prob.params.update({"t": t, "U": U, "mu": U / 2 if mu is None else mu})
    for b in range(nb):
        prob.operators[f"eb{b}"] = ("one-body", _both_spins(L, [(ns + b, ns + b, 1.0)]))
        prob.operators[f"tb{b}"] = ("one-body", _both_spins(L, [(b // 2, ns + b, 1.0)]))
        prob.params[f"eb{b}"] = float(eps[b])
        prob.params[f"tb{b}"] = float(hyb[b])
    prob.sectors = "R0:N12:S0"
    return prob


def matsubara(n: int = 256, beta: float = 50.0) -> np.ndarray:
    """Fermionic Matsubara frequencies i(2k+1)pi/beta, k = 0..n-1."""
    return 1j * (2 * np.arange(n) + 1) * math.pi / beta


# Named workloads (the five synthetic configurations this solver is judged on).
def chain8() -> ClusterProblem:
    """1D chain L=8, open, t=-1, U=4, mu=2, sector N_up=N_dn=4 (dim 4900)."""
    return hubbard_cluster(8, 1, t=-1.0, U=4.0, mu=2.0, name="chain8")


def square4x4() -> ClusterProblem:
    """4x4 open square, t=-1, t'=0.3, U=8, half filling (dim 12870^2)."""
    return hubbard_cluster(4, 4, t=-1.0, tp=0.3, U=8.0, mu=4.0, name="sq4x4")


def random_batch(n: int = 1024, seed: int = 12345, geoms=None):
    """Seeded draw of independent clusters with every (N_up, N_dn) sector listed.

    Geometry uniform over 2x2, 2x3, 2x4, chain 8, chain 10 (or `geoms`), t=-1,
    U ~ U[0,12], mu ~ U[0,U], staggered Neel field M ~ U[0,0.3]."""
    rng = np.random.default_rng(seed)
    geoms = geoms or [(2, 2), (2, 3), (2, 4), (8, 1), (10, 1)]
    out = []
    for k in range(n):
        nx, ny = geoms[rng.integers(len(geoms))]
        U = float(rng.uniform(0, 12))
        mu = float(rng.uniform(0, U))
        M = float(rng.uniform(0, 0.3))
        p = hubbard_cluster(nx, ny, t=-1.0, U=U, mu=mu, M=M, name=f"b{nx}x{ny}")
        L = nx * ny
        secs = [f"R0:N{a + b}:S{a - b}" for a in range(L + 1) for b in range(L + 1)]
        p.sectors = "/".join(secs)
        out.append(p)
    return out


def random_baths(n: int = 256, seed: int = 4242):
    """Seeded bath-parameter points for the 2x2 + 8-bath cluster."""
    rng = np.random.default_rng(seed)
    return [plaquette_bath(rng.uniform(-2, 2, 8), rng.uniform(0, 1, 8)) for _ in range(n)]


# ------------------------------------------------------------------ lattices --

@dataclass
class LatticeProblem:
    """A lattice model tiled by one cluster, in the vocabulary of pyqcm's
    lattice_model (pyqcm/__init__.py: cluster_model, cluster, lattice_model,
    hopping_operator, interaction_operator, density_wave, set_parameters).

    sites: cluster site positions (integer 3-vectors); superlattice: the
    superlattice vectors (their number is the spatial dimension);
    hoppings: (name, link, amplitude); interactions: Hubbard operator names;
    density_waves: (name, type, Q in multiples of pi); params: independent
    parameter values; equiv: (name, multiplier, reference) dependences, as in
    pyqcm's "name = multiplier * reference" syntax. Cluster (Weiss) parameters
    carry the suffix _1."""
    name: str
    sites: list
    superlattice: list
    hoppings: list = field(default_factory=list)
    interactions: list = field(default_factory=list)
    density_waves: list = field(default_factory=list)
    sectors: str = "R0"
    params: dict = field(default_factory=dict)
    equiv: list = field(default_factory=list)
    n_bath: int = 0
    cluster_operators: dict = field(default_factory=dict)  # name -> (type, [(r, c, v)]) on the cluster model

    @property
    def n_sites(self) -> int:
        return len(self.sites)


def square_lattice_vca(nx: int, ny: int, U: float = 8.0, M1: float = 0.1, mu1: float | None = None,
                       t: float = 1.0, mu: float | None = None, name: str | None = None,
                       superlattice=None) -> LatticeProblem:
    """Square lattice (nearest-neighbour hopping -t) tiled by an nx x ny cluster,
    Hubbard U, chemical potential mu (U/2 by default, half filling) and a Neel
    Weiss field M on the cluster only (M_1, density wave of type Z at Q = (pi, pi)).
    mu1, when given, is a separate cluster chemical potential mu_1 (else mu_1 = mu)."""
    n = nx * ny
    sites = [(x, y, 0) for y in range(ny) for x in range(nx)]
    params = {"t": t, "U": U, "mu": U / 2 if mu is None else mu, "M": 0.0, "M_1": M1}
    equiv = [("t_1", 1.0, "t"), ("U_1", 1.0, "U")]
    if mu1 is None:
        equiv.append(("mu_1", 1.0, "mu"))
    else:
        params["mu_1"] = mu1
    sl = [tuple(v) for v in superlattice] if superlattice is not None else [(nx, 0, 0), (0, ny, 0)]
    return LatticeProblem(name or f"sq{nx}x{ny}_vca", sites, sl,
                          hoppings=[("t", (1, 0, 0), -1.0), ("t", (0, 1, 0), -1.0)], interactions=["U"],
                          density_waves=[("M", "Z", (1.0, 1.0, 0.0))], sectors=f"R0:N{n}:S0",
                          params=params, equiv=equiv)


def vca_2x5(U: float = 8.0, M1: float = 0.1, dmu: float = 0.0) -> LatticeProblem:
    """2x5 clusters tiling the square lattice (t = 1, amplitude -1), half filling
    (mu = U/2), Neel Weiss field M_1 and cluster chemical potential mu_1 = U/2 + dmu.
    The superlattice (2,0), (1,5) keeps Q = (pi, pi) commensurate with the tiling."""
    return square_lattice_vca(2, 5, U=U, M1=M1, mu1=U / 2 + dmu, name="vca2x5",
                              superlattice=[(2, 0, 0), (1, 5, 0)])


def cdmft_2x2_bath(eps, hyb, U: float = 8.0, t: float = 1.0) -> LatticeProblem:
    """Square lattice (hopping -t) tiled by 2x2 plaquettes, each with nb = len(eps)
    bath orbitals (4 or 8: one or two per site): bath energies eb{b}_1 = eps[b],
    hybridisations tb{b}_1 = hyb[b] with cluster site b // (nb / 4), half filling
    (mu = U/2, sector R0:N{4 + nb}:S0). With eight bath orbitals the cluster model
    is that of plaquette_bath."""
    ns, nb = 4, len(eps)
    if nb not in (4, 8) or len(hyb) != nb:
        raise ValueError("cdmft_2x2_bath: 4 or 8 bath orbitals, one energy and one hybridisation each")
    L = ns + nb
    per = nb // ns
    sites = [(x, y, 0) for y in range(2) for x in range(2)]
    cops = {}
    params = {"t": t, "U": U, "mu": U / 2}
    for b in range(nb):
        cops[f"eb{b}"] = ("one-body", _both_spins(L, [(ns + b, ns + b, 1.0)]))
        cops[f"tb{b}"] = ("one-body", _both_spins(L, [(b // per, ns + b, 1.0)]))
        params[f"eb{b}_1"] = float(eps[b])
        params[f"tb{b}_1"] = float(hyb[b])
    return LatticeProblem(f"cdmft2x2b{nb}", sites, [(2, 0, 0), (0, 2, 0)], hoppings=[("t", (1, 0, 0), -1.0),
                          ("t", (0, 1, 0), -1.0)], interactions=["U"], sectors=f"R0:N{ns + nb}:S0", params=params,
                          equiv=[("t_1", 1.0, "t"), ("U_1", 1.0, "U"), ("mu_1", 1.0, "mu")], n_bath=nb,
                          cluster_operators=cops)


def regular_frequency_grid(wc: float, n1: int, n2: int):
    """Uniform grid of n1 points on [0, wc] and n2 points uniform in 1/w on
    [0, 1/wc] (midpoint rule), weights including the 1/pi of the imaginary-axis
    integral: the grid of pyqcm's regular_frequency_grid (pyqcm/__init__.py:3069-3089)."""
    w = np.zeros(n1 + n2)
    p = np.zeros(n1 + n2)
    dw = wc / n1
    w[:n1] = np.linspace(0.5 * dw, wc - 0.5 * dw, n1)
    p[:n1] = dw / np.pi
    dw = 1.0 / (n2 * wc)
    w[n1:] = np.flip(1.0 / np.linspace(0.5 * dw, 1.0 / wc - 0.5 * dw, n2))
    p[n1:] = w[n1:] * w[n1:] * dw / np.pi
    return w, p
