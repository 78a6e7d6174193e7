"""CDMFT on this package's GPU ED: pyqcm's self-consistency loop for a lattice
tiled by one cluster with bath orbitals (class CDMFT, pyqcm/cdmft.py:156-720),
and a learned surrogate that proposes the starting bath (BathSurrogate).

One CDMFT step (CDMFT_step, pyqcm/cdmft.py:478-640): for the current bath
parameters x the cluster's ground state and Green function are solved by ED on
the GPU; the host function G_host(iw) = Gproj(iw)^-1 + Sigma_c(iw) + H_c - iw comes
from the lattice layer (lattice.CDMFT_host, its k-sum on the GPU); x then moves
to the minimum of the distance

    d(x) = dw / dim^2 * f * sum_n w_n ||Gamma_x(iw_n) + G_host(iw_n)||_F^2

(lattice_model_instance::CDMFT_distance, src_qcm/CPT.cpp:519-560; f = 2 without
spin asymmetry), and the sequence of x is iterated by Broyden or by damped fixed
point (pyqcm/__init__.py:2773-2898) until the convergence tests pass
(convergence_manager, pyqcm/cdmft.py:9-110).

The distance is minimised here without ED instances: the hybridisation of the
bath, Gamma_x(z) = T (z - E)^-1 T^+ (T the cluster-bath block of the cluster's
one-body matrix, E the bath block), is linear-fractional in the bath parameters,
whose operators enter the one-body matrix linearly, so the residuals of
lattice_model_instance::CDMFT_residuals (src_qcm/CPT.cpp:572-618) and their exact
Jacobian dGamma = dT R T^+ + T R dT^+ + T R dE R T^+ (R = (z - E)^-1) are dense
numpy algebra on (frequencies x n_bath x n_bath) arrays. The reference
differentiates the same residuals by central differences (CDMFT_gradient,
src_qcm/CPT.cpp:635-670). The minimisers and their tolerances are the reference's
(optimize, pyqcm/cdmft.py:1533-1700): least squares ('trf', 'BFGS' -> 'lm') with
the Jacobian, or Nelder-Mead on the distance.

BathSurrogate: a network trained (on the GPU, by this package's tensor-core
kernels) on converged baths that this solver computes at points of the lattice
parameters; it proposes the starting bath of a new CDMFT run, which the ED loop
then verifies and converges. Without it the run starts from the model's bath.
"""
from __future__ import annotations

import math

import numpy as np
import scipy.optimize

from . import lattice as LT

# ------------------------------------------------------------ frequency grids --


def legendre_frequency_grid(w1, w2, n1, n2, n3):
    """Gauss-Legendre nodes and weights (1/pi included) in [0, w1], [w1, w2] and,
    in 1/w, in [w2, inf) (pyqcm.legendre_frequency_grid, pyqcm/__init__.py:3040-3066)."""
    w = np.zeros(n1 + n2 + n3)
    p = np.zeros(n1 + n2 + n3)
    x, a = np.polynomial.legendre.leggauss(n1)
    w[:n1] = 0.5 * w1 * (x + 1)
    p[:n1] = 0.5 * w1 * a
    x, a = np.polynomial.legendre.leggauss(n2)
    w[n1:n1 + n2] = w1 + 0.5 * (w2 - w1) * (x + 1)
    p[n1:n1 + n2] = 0.5 * (w2 - w1) * a
    x, a = np.polynomial.legendre.leggauss(n3)
    u = 0.5 * (x[::-1] + 1) / w2
    w[n1 + n2:] = 1.0 / u
    p[n1 + n2:] = 0.5 / w2 * a[::-1] * w[n1 + n2:] ** 2
    return w, p / np.pi


class frequency_grid:
    """Imaginary-frequency grid of the distance function (pyqcm/cdmft.py:821-890):
    'legendre' (w1, w2, n1, n2, n3), 'matsubara' (wc, beta), 'matsubara+'
    (wc, beta, n2), 'regular' (wc, n1, n2). As in the reference, the distance
    weights (cdmft_weight) are 1 for every grid unless opt is 'ifreq' (1/w,
    normalised) or 'self' (the norm of Sigma(iw) - Sigma(inf), normalised, updated
    at every step); `weight` are the integration weights."""

    def __init__(self, grid_type: str = "legendre", specs=(1, 10, 5, 10, 5), opt: str = ""):
        from . import workloads as W
        g = grid_type.lower()
        if g == "legendre":
            w1, w2, n1, n2, n3 = specs
            self.wr, self.weight = legendre_frequency_grid(w1, w2, n1, n2, n3)
            self.name = f"legendre({w1:g}-{w2:g}-{n1:d}-{n2:d}-{n3:d})"
        elif g == "matsubara":
            wc, beta = specs
            self.wr = np.arange(np.pi / beta, wc + 1e-6, 2 * np.pi / beta)
            self.weight = (2 * np.pi / beta) * np.ones_like(self.wr)
            self.name = f"matsubara({wc:g}-{beta:g})"
        elif g == "matsubara+":
            wc, beta, n2 = specs
            n1 = int(np.ceil(wc * beta / (2 * np.pi)))
            self.wr, self.weight = W.regular_frequency_grid(wc, n1, n2)
            self.name = f"Matsubara+({wc:g}-{beta:g}-{n2:d})"
        elif g == "regular":
            wc, n1, n2 = specs
            self.wr, self.weight = W.regular_frequency_grid(wc, n1, n2)
            self.name = f"regular({wc:g}-{n1:d}-{n2:d})"
        else:
            raise ValueError("Unknown type of frequency grid " + grid_type)
        self.nw = len(self.wr)
        self.cdmft_weight = np.ones_like(self.wr)
        self.self_norm = False
        if opt == "ifreq":
            t = 1.0 / self.wr
            self.cdmft_weight = t / t.sum()
            self.name += "_ifreq"
        elif opt == "self":
            self.self_norm = True
            self.name += "_self"
        elif opt != "":
            raise ValueError("Unknown option " + opt + " in frequency_grid()")

    def update(self, inst):
        """With opt='self': weights from the current instance's self-energy."""
        if not self.self_norm:
            return
        import pyqcm_b200 as qed
        s_inf = qed.self_energy(np.array([1.0e6j]), label=inst.label)[0]
        S = qed.self_energy(1j * self.wr, label=inst.label)
        wts = np.array([np.linalg.norm(S[i] - s_inf) for i in range(self.nw)])
        self.cdmft_weight = wts / wts.sum()


# ------------------------------------------------- bath hybridisation and distance --


class BathDistance:
    """The bath's hybridisation Gamma_x(z), the CDMFT residuals and their Jacobian
    as functions of the CDMFT variational parameters x (names with the cluster
    suffix, e.g. 'eb3_1'), for a LatticeModel whose cluster has bath orbitals.

    The one-body matrix of the cluster is H(x) = H0 + sum_p x_p O_p, where O_p is
    the matrix of the cluster operator behind parameter p (its elements, Hermitian
    completion of off-diagonal ones) and H0 holds every other cluster operator at
    the base values. Only the bath rows enter Gamma, so only the cluster
    operators with bath elements are needed."""

    def __init__(self, model: LT.LatticeModel, varia, base_values: dict):
        self.model = model
        self.varia = list(varia)
        ns, nb = model.n, model.n_bath
        if nb == 0:
            raise ValueError("CDMFT needs a cluster with bath orbitals")
        no = model.n_orb
        cops = getattr(model.prob, "cluster_operators", {})
        nblk = 2 if model.mixing == 4 else 1
        self.nblk = nblk

        def op_matrix(name):
            typ, el = cops[name]
            if typ != "one-body":
                raise ValueError(f"CDMFT variational parameter on a {typ} operator: {name}")
            M = np.zeros((2, no, no))
            for r, c, v in el:
                sr, sc = r // no, c // no
                if sr != sc:
                    raise ValueError(f"operator {name} mixes spins: not supported")
                i, j = r % no, c % no
                M[sr, i, j] += v
                if i != j:
                    M[sr, j, i] += v
            return M

        for v in self.varia:
            if not v.endswith("_1"):
                raise ValueError(f"{v} cannot be a CDMFT variational parameter")
            if v[:-2] not in cops:
                raise ValueError(f"{v}: no cluster operator {v[:-2]} with bath elements")
        cv = model.cluster_values(base_values)
        H0 = np.zeros((2, no, no))
        for name in cops:
            if name in cv and name + "_1" not in self.varia:
                H0 += cv[name] * op_matrix(name)
        self.H0 = H0[:nblk]
        self.O = np.array([op_matrix(v[:-2])[:nblk] for v in self.varia])  # (p, blk, no, no)
        self.ns, self.nb = ns, nb

    def _blocks(self, x):
        H = self.H0 + np.tensordot(np.asarray(x, dtype=np.float64), self.O, axes=1)
        ns = self.ns
        return H[:, :ns, ns:], H[:, ns:, ns:]  # T (blk, ns, nb), E (blk, nb, nb)

    def gamma(self, x, freqs):
        """Gamma_x(iw) per spin block: (blk, nw, ns, ns) complex."""
        T, E = self._blocks(x)
        z = 1j * np.asarray(freqs, dtype=np.float64)
        out = []
        for b in range(self.nblk):
            R = np.linalg.inv(z[:, None, None] * np.eye(self.nb)[None] - E[b][None])
            out.append(T[b][None] @ R @ T[b].T[None])
        return np.array(out)

    def residuals(self, x, host, freqs, weights, jac: bool = False):
        """r = sqrt(w_n) (Gamma_x + G_host) as [Re, Im] per frequency and block
        (the layout of CDMFT_residuals) and, with jac, dr/dx (rows x n_var)."""
        T, E = self._blocks(x)
        z = 1j * np.asarray(freqs, dtype=np.float64)
        sw = np.sqrt(np.asarray(weights, dtype=np.float64))
        ns, nb, nw = self.ns, self.nb, len(z)
        r, J = [], []
        for b in range(self.nblk):
            R = np.linalg.inv(z[:, None, None] * np.eye(nb)[None] - E[b][None])  # (nw, nb, nb)
            RT = R @ T[b].T[None]                                              # (nw, nb, ns)
            G = T[b][None] @ RT + np.asarray(host[b])                           # (nw, ns, ns)
            G = sw[:, None, None] * G
            r.append(np.concatenate([G.real.reshape(nw, -1), G.imag.reshape(nw, -1)], axis=1).ravel())
            if jac:
                TR = T[b][None] @ R                                             # (nw, ns, nb)
                cols = []
                for p in range(len(self.varia)):
                    dT = self.O[p, b, :ns, ns:]
                    dE = self.O[p, b, ns:, ns:]
                    dG = dT[None] @ RT + TR @ dT.T[None] + TR @ dE[None] @ RT
                    dG = sw[:, None, None] * dG
                    cols.append(np.concatenate([dG.real.reshape(nw, -1), dG.imag.reshape(nw, -1)], axis=1).ravel())
                J.append(np.array(cols).T)
        r = np.concatenate(r)
        return (r, np.concatenate(J, axis=0)) if jac else r

    def scale(self, freqs):
        """Factor taking sum r^2 to the reported distance (dw / dim^2, doubled
        without spin asymmetry)."""
        dw = float(freqs[1] - freqs[0]) if len(freqs) > 1 else 1.0
        return (2.0 if self.model.mixing == 0 else 1.0) * dw / (self.ns * self.ns)

    def distance(self, x, host, freqs, weights):
        r = self.residuals(x, host, freqs, weights)
        return self.scale(freqs) * float(r @ r)


def optimize_bath(bd: BathDistance, x0, host, freqs, weights, method: str = "trf", initial_step: float = 0.1,
                  accur: float = 1e-6, accur_dist: float = 1e-8, maxfev: int = 2000):
    """Minimum of the distance from x0 (optimize, pyqcm/cdmft.py:1533-1700):
    'trf' / 'BFGS' (Levenberg-Marquardt) / 'L-BFGS-B' (dogbox) by least squares on
    the residuals with their Jacobian; 'Nelder-Mead' (adaptive, initial simplex of
    step initial_step) on the distance. Returns (x, evaluations, distance)."""
    x0 = np.asarray(x0, dtype=np.float64)
    m = method.lower()
    if m in ("trf", "bfgs", "l-bfgs-b"):
        ls = {"trf": "trf", "bfgs": "lm", "l-bfgs-b": "dogbox"}[m]
        sol = scipy.optimize.least_squares(lambda x: bd.residuals(x, host, freqs, weights), x0,
                                           jac=lambda x: bd.residuals(x, host, freqs, weights, jac=True)[1],
                                           method=ls, max_nfev=maxfev, ftol=accur_dist, xtol=accur, gtol=1e-12)
        x, nfev = sol.x, sol.nfev
    elif method == "Nelder-Mead":
        n = len(x0)
        simplex = np.repeat(x0[None], n + 1, axis=0)
        simplex[1:] += initial_step * np.eye(n)
        sol = scipy.optimize.minimize(lambda x: bd.distance(x, host, freqs, weights), x0, method="Nelder-Mead",
                                      options={"maxfev": maxfev, "xatol": accur, "fatol": accur_dist,
                                               "initial_simplex": simplex, "adaptive": True})
        x, nfev = sol.x, sol.nfev
    else:
        raise ValueError(f"unknown minimisation method {method}")
    if np.any(np.isnan(x)):
        raise RuntimeError("NaN found in optimization of bath parameters")
    return x, int(nfev), bd.distance(x, host, freqs, weights)


# ------------------------------------------------------------ the CDMFT loop --


class convergence_manager:
    """One convergence test (pyqcm/cdmft.py:9-110): converged when the difference
    of the current value with each of the `depth` previous ones is below tol."""

    def __init__(self, name, diff_func, tol, depth: int = 2):
        self.name, self.diff_func, self.tol, self.depth = name, diff_func, tol, depth
        self.diff = np.zeros(depth)
        self.iter = 0
        self.X = []
        self.converged = False

    def test(self, x) -> bool:
        self.iter += 1
        if self.iter <= self.depth:
            self.X.append(x)
            return False
        for i in range(self.depth):
            self.diff[i] = self.diff_func(x, self.X[i])
        ok = bool(np.all(self.diff <= self.tol))
        self.X = self.X[1:] + [x]
        self.converged = ok
        return ok


class TooManyIterationsError(RuntimeError):
    pass


class CDMFT:
    """A CDMFT computation (the reference's class CDMFT, pyqcm/cdmft.py:156-720);
    the constructor runs it. Scope: one cluster with bath orbitals, normal
    (spin-conserving) baths, host function from the lattice layer.

    model: lattice.LatticeModel; varia: the bath parameter names (suffix _1);
    values: lattice parameter values (start bath included; defaults: the model's);
    start: starting values of varia (overrides `values`); grid: frequency_grid
    (default: the reference's Legendre grid); side: k points per superlattice
    direction of the host's k-sum. iteration 'broyden' (alpha: 1 + alpha is the
    initial inverse Jacobian) or 'fixed_point' (alpha: damping, or (damping,
    after n iterations); default (0.3, 16)); convergence: 'parameters',
    'distance', 'GS energy', 'hybridization', 'self-energy' (or a sequence, with
    accur a matching sequence).

    Results: x (converged bath), niter, dist, E0 (ground-state energy of the last
    step), history (bath per step), n_solves (ED ground state + Green function
    solves), I (the last lattice instance, kept)."""

    def __init__(self, model: LT.LatticeModel, varia, values: dict | None = None, start=None, grid=None,
                 maxiter: int = 32, miniter: int = 0, convergence="parameters", depth: int = 2,
                 accur_bath: float = 1e-6, accur=1e-4, accur_dist: float = 1e-8, iteration: str = "broyden",
                 alpha=0.0, method: str = "Nelder-Mead", initial_step: float = 0.1, max_function_eval: int = 1_000_000,
                 side: int = 32, label: int = 880000, max_value: float = 100.0, verbose: bool = False):
        if iteration not in ("broyden", "fixed_point"):
            raise ValueError("the argument 'iteration' of CDMFT() should be one of 'broyden', 'fixed_point'")
        self.model = model
        self.varia = list(varia)
        self.values = dict(model.prob.params if values is None else values)
        if start is not None:
            self.values.update({v: float(s) for v, s in zip(self.varia, start)})
        self.grid = grid if grid is not None else frequency_grid()
        self.side, self.label0, self.max_value, self.verbose = side, label, max_value, verbose
        self.method, self.initial_step = method, initial_step
        self.accur_bath, self.accur_dist = accur_bath, accur_dist
        self.maxfev = max_function_eval if method == "Nelder-Mead" else min(max_function_eval, 2000)
        self.x = np.array([self.values[v] for v in self.varia], dtype=np.float64)
        self.history, self.dist, self.E0, self.n_solves, self.I = [], 1e6, None, 0, None
        self.host, self.sigma = None, None
        self.bd = BathDistance(model, self.varia, self.values)
        convergence = (convergence,) if isinstance(convergence, str) else tuple(convergence)
        accur = (accur,) if np.isscalar(accur) else tuple(accur)
        if len(convergence) != len(accur):
            raise ValueError('The number of convergence tests must be the same as the length of "accur"')
        self.tests = []
        for name, tol in zip(convergence, accur):
            if name == "parameters":
                f = lambda a, b: np.linalg.norm(a - b) / a.shape[0]
            elif name in ("hybridization", "self-energy"):
                f = self._diff_matrix
            elif name == "GS energy":
                f = lambda a, b: abs(a - b)
            elif name == "distance":
                f = lambda a, b: abs(a - b) / b
            else:
                raise ValueError(f'type of convergence test "{name}" in CDMFT does not exist')
            self.tests.append(convergence_manager(name, f, tol, depth))
        if iteration == "fixed_point" and not (isinstance(alpha, tuple) or (isinstance(alpha, float) and alpha > 0)):
            alpha = (0.3, 16)
        self.iter = 0
        try:
            if iteration == "broyden":
                self.x, self.niter = self._broyden(self.x, alpha, maxiter, miniter)
            else:
                self.x, self.niter = self._fixed_point(self.x, alpha, maxiter, miniter)
        except BaseException:
            if self.I is not None:  # a failed run leaves no ED instance behind
                self.I.erase()
                self.I = None
            raise

    # ---- one step -----------------------------------------------------------
    def step(self, x):
        """CDMFT_step: ED at bath x, host, minimisation; returns the new bath."""
        vals = dict(self.values)
        vals.update({v: float(s) for v, s in zip(self.varia, x)})
        if self.I is not None:
            self.I.erase()
        self.I = self.model.instance(self.label0 + self.iter, **vals)
        e0, _ = self.I.ground_state()
        self.I.Green_function_solve()
        self.n_solves += 1
        self.E0 = e0
        self.grid.update(self.I)
        self.host = LT.CDMFT_host(self.I, self.grid.wr, side=self.side)
        xn, nfev, d = optimize_bath(self.bd, x, self.host, self.grid.wr, self.grid.cdmft_weight, self.method,
                                    self.initial_step, self.accur_bath, self.accur_dist, self.maxfev)
        if nfev > self.maxfev:
            raise RuntimeError(f"number of function evaluations exceeds preset maximum of {self.maxfev}")
        if np.any(np.abs(xn) > self.max_value):
            raise RuntimeError("a bath parameter left the allowed range |x| <= max_value")
        self.dist = d
        self.history.append(np.copy(xn))
        if self.verbose:
            print(f"CDMFT step {self.iter + 1}: E0 = {e0:.12f}, distance = {d:.4g}, {nfev} evaluations")
        self.iter += 1
        return xn

    def _diff_matrix(self, X, Y):
        g = self.grid
        return float(sum(g.weight[i] * np.linalg.norm(X[b][i] - Y[b][i]) ** 2
                         for b in range(len(X)) for i in range(g.nw)))

    def _converged(self) -> bool:
        """The convergence tests on the last step (its minimised bath, distance,
        energy, host), as the reference's check_convergence after CDMFT_step."""
        ok = True
        for C in self.tests:
            if C.name == "parameters":
                ok = C.test(np.copy(self.history[-1])) and ok
            elif C.name == "distance":
                ok = C.test(self.dist) and ok
            elif C.name == "GS energy":
                ok = C.test(self.E0) and ok
            elif C.name == "hybridization":
                ok = C.test([np.copy(h) for h in self.host]) and ok
            elif C.name == "self-energy":
                import pyqcm_b200 as qed
                ok = C.test([qed.self_energy(1j * self.grid.wr, label=self.I.label)]) and ok
        return ok

    # ---- iterations (pyqcm/__init__.py:2773-2898) ----------------------------
    def _fixed_point(self, x0, damping, maxiter, miniter):
        alpha = damping if isinstance(damping, float) else 0.0
        it = 0
        x0 = np.copy(x0)
        while True:
            if isinstance(damping, tuple) and it >= damping[1] and alpha == 0:
                alpha = damping[0]
            fx = self.step(x0)
            x0 = alpha * x0 + (1.0 - alpha) * fx  # x0 + (alpha - 1) (x0 - step(x0))
            it += 1
            if self._converged():
                break
            if it > maxiter:
                raise TooManyIterationsError(f"CDMFT did not converge in {maxiter} iterations")
        return x0, it

    def _broyden(self, x0, iJ0, maxiter, miniter, xtol=1e-6):
        n = len(x0)
        Inv = (1.0 + iJ0) * np.eye(n) if np.isscalar(iJ0) else np.array(iJ0, dtype=np.float64)
        F = lambda x: x - self.step(x)
        x = np.copy(x0)
        f0 = F(x)
        it = 0
        while True:
            dxv = -Inv @ f0
            if np.any(np.isnan(dxv)):
                raise ValueError("NaN produced in Broyden method")
            x = x + dxv
            if np.linalg.norm(dxv) < xtol and it >= miniter:
                self._converged()
                break
            if self._converged() and it >= miniter:
                break
            f = F(x)
            df = f - f0
            f0 = np.copy(f)
            Inv = Inv + np.outer(dxv - Inv @ df, dxv) @ Inv / (dxv @ (Inv @ df))
            it += 1
            if it > maxiter:
                raise TooManyIterationsError(f"CDMFT did not converge in {maxiter} iterations")
        return x, it


# --------------------------------------------------------- learned starting bath --


def canonical_bath(x, energies, hybs, site_of):
    """One representative of a bath among those with the same hybridisation
    function: Gamma is unchanged by the sign of each bath orbital's hybridisation
    and by permutations of the bath orbitals attached to the same cluster site,
    so hybridisations are made non-negative and, per site, the orbitals are
    ordered by energy. energies[b] / hybs[b]: indices in x of orbital b's energy
    and hybridisation; site_of[b]: its cluster site."""
    x = np.array(x, dtype=np.float64)
    out = np.copy(x)
    site_of = np.asarray(site_of)
    for s in np.unique(site_of):
        orbs = np.flatnonzero(site_of == s)
        order = orbs[np.argsort(x[np.asarray(energies)[orbs]], kind="stable")]
        for dst, src in zip(orbs, order):
            out[energies[dst]] = x[energies[src]]
            out[hybs[dst]] = abs(x[hybs[src]])
    return out


class BathSurrogate:
    """Surrogate of the converged CDMFT bath as a function of lattice parameters.

    One network (the package's BF16 tensor-core MLP, trained by Adam on the GPU)
    maps (scaled lattice parameters, a code of the bath parameter's index) to that
    bath parameter at convergence; the code is the index's bits as +-1, so all
    bath parameters share the network and its training data. Trained on baths
    converged by CDMFT at points of `box` (the training points are generated and
    solved by `generate`); `propose` returns the starting bath of a new run."""

    def __init__(self, inputs, box, varia, width: int = 256, seed: int = 0):
        from .surrogate import MLP
        self.inputs, self.varia = list(inputs), list(varia)
        self.lo = np.array([b[0] for b in box], dtype=np.float64)
        self.hi = np.array([b[1] for b in box], dtype=np.float64)
        self.nbits = max(1, math.ceil(math.log2(max(2, len(self.varia)))))
        if len(self.inputs) + self.nbits > 16:
            raise ValueError("too many inputs for the surrogate network")
        self.net = MLP(n_in=len(self.inputs) + self.nbits, width=width, seed=seed)
        self.mean = np.zeros(len(self.varia))
        self.std = np.ones(len(self.varia))

    def _features(self, P):
        P = np.atleast_2d(np.asarray(P, dtype=np.float64))
        s = 2.0 * (P - self.lo) / (self.hi - self.lo) - 1.0
        nv = len(self.varia)
        code = np.array([[1.0 if (k >> j) & 1 else -1.0 for j in range(self.nbits)] for k in range(nv)])
        X = np.concatenate([np.repeat(s, nv, axis=0), np.tile(code, (len(s), 1))], axis=1)
        return X.astype(np.float32)

    def fit(self, P, baths, epochs: int = 600, batch: int = 64, lr: float = 2e-3, seed: int = 0):
        """Trains on lattice points P (n x n_inputs) and converged baths (n x n_var)."""
        B = np.asarray(baths, dtype=np.float64)
        self.mean = B.mean(axis=0)
        self.std = np.maximum(B.std(axis=0), 1e-3)
        X = self._features(P)
        Y = ((B - self.mean) / self.std).astype(np.float32).ravel()
        rows = len(X)
        batch = max(16, min(batch, rows // 16 * 16))
        return self.net.train(X, Y, epochs=epochs, batch=batch, lr=lr, seed=seed)

    def propose(self, p) -> np.ndarray:
        """The proposed starting bath at lattice point p (n_inputs values)."""
        y = self.net(self._features(p)).astype(np.float64)
        return self.mean + self.std * y


def converge_baths(model: LT.LatticeModel, varia, inputs, points, start, canonical=None, **cdmft_args):
    """Training data: CDMFT converged at each point (values of `inputs`), in order,
    each run started from the last converged bath (the first from `start`);
    `canonical` (optional) maps each converged bath to its representative. A point
    whose run fails (no convergence, a bath parameter out of range) is left out.
    Returns (indices of the converged points, their baths, their iteration counts)."""
    ok, baths, iters = [], [], []
    x = np.asarray(start, dtype=np.float64)
    vals0 = dict(model.prob.params)
    label0 = cdmft_args.pop("label", 870000)
    for k, p in enumerate(np.atleast_2d(points)):
        vals = dict(vals0)
        vals.update({n: float(v) for n, v in zip(inputs, p)})
        try:
            run = CDMFT(model, varia, values=vals, start=x, label=label0 + 1000 * k, **cdmft_args)
        except (TooManyIterationsError, RuntimeError, ValueError):
            continue
        x = run.x
        ok.append(k)
        baths.append(np.copy(canonical(x) if canonical else x))
        iters.append(run.niter)
        run.I.erase()
    return np.array(ok, dtype=np.int64), np.array(baths), np.array(iters)
