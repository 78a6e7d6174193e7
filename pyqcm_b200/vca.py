"""Variational cluster approximation: stationary points of the Potthoff
functional Omega over cluster (Weiss) parameters, with the cluster problems
solved by this package's GPU ED.

The search is the reference's Newton-Raphson method (pyqcm/vca.py:239-430):
every iteration fits a quadratic form through 1 + 2n + n(n-1)/2 points around
the current x (the n +/- step pairs and n(n-1)/2 off-diagonal points at
0.707 step), moves by dx = -H^{-1} g, then resets each step to |dx_i|, at least
twice the accuracy (the reference also compares with twice the initial step,
but its "initial step" names the same array as the step, so that bound never
applies; it does not here either); it stops when every |dx_i| <= accur_i or
|g| < gtol. Here the points of one iteration are solved
as one batch (their ground states and Green functions concurrently on the GPU,
then their Omega on the GPU grid).
"""
from __future__ import annotations

import os
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

import pyqcm_b200 as qed
from pyqcm_b200 import lattice as LT


class OmegaEvaluator:
    """Omega at batches of points of the variational parameters `varia` (or of
    any point -> parameter-values map `to_values`)."""

    def __init__(self, model: LT.LatticeModel, varia, freqs, weights, nk, fixed=None, threads: int = 0,
                 label0: int = 700000, to_values=None):
        self.model = model
        self.to_values = to_values
        self.varia = list(varia)
        self.freqs = np.asarray(freqs, dtype=np.float64)
        self.weights = np.asarray(weights, dtype=np.float64)
        self.nk = tuple(nk)
        self.fixed = dict(fixed or {})
        self.threads = threads
        self.label = label0
        self.n_evals = 0
        self.seconds = 0.0

    def __call__(self, X) -> np.ndarray:
        t0 = time.perf_counter()
        X = np.atleast_2d(np.asarray(X, dtype=np.float64))
        insts = []
        for x in X:
            vals = dict(self.fixed)
            if self.to_values is not None:
                vals.update(self.to_values(x))
            else:
                vals.update({k: float(v) for k, v in zip(self.varia, x)})
            self.label += 1
            insts.append(self.model.instance(self.label, **vals))
        labels = [I.label for I in insts]
        try:
            qed.ground_state_solve_batch(labels, threads=self.threads)
            qed.Green_function_solve_batch(labels, threads=self.threads)
            # the (frequency, k) sums of the instances on host threads: each call
            # holds only its own instance and its thread's stream, and the C calls
            # release the interpreter lock
            omega = lambda I: I.Potthoff_functional(self.freqs, self.weights, self.nk)
            nt = min(len(insts), self.threads or min(16, os.cpu_count() or 1))
            if nt > 1:
                with ThreadPoolExecutor(max_workers=nt) as pool:
                    out = np.array(list(pool.map(omega, insts)))
            else:
                out = np.array([omega(I) for I in insts])
        finally:
            for I in insts:
                I.erase()
        self.n_evals += len(X)
        self.seconds += time.perf_counter() - t0
        return out


def nr_quadratic_fit(func, x, step):
    """Value, gradient and Hessian at x from the quadratic form through the
    1 + 2n + n(n-1)/2 stencil points (_NR_Hessian, pyqcm/vca.py:241-313)."""
    x = np.asarray(x, dtype=np.float64)
    n = len(x)
    N = 1 + 2 * n + (n * (n - 1)) // 2
    xp = np.tile(x, (N, 1))
    k = 0
    for i in range(n):
        k += 1
        xp[k, i] += step[i]
        k += 1
        xp[k, i] -= step[i]
    for i in range(n):
        for j in range(i):
            k += 1
            xp[k, i] += 0.707 * (2 * (i % 2) - 1) * step[i]
            xp[k, j] += 0.707 * (2 * (j % 2) - 1) * step[j]
    y = func(xp)
    A = np.empty((N, N))
    A[:, 0] = 1.0
    A[:, 1:n + 1] = xp
    m = n + 1
    for i in range(n):
        for j in range(i + 1):
            A[:, m] = xp[:, i] * xp[:, j] * (0.5 if i == j else 1.0)
            m += 1
    c = np.linalg.solve(A, y)
    hess = np.zeros((n, n))
    val = c[0]
    grad = c[1:n + 1].copy()
    val += np.sum(grad * x)
    m = n + 1
    for i in range(n):
        for j in range(i + 1):
            hess[i, j] = hess[j, i] = c[m]
            val += x[i] * x[j] * c[m] * (0.5 if i == j else 1.0)
            m += 1
    grad += hess @ x
    return val, grad, hess


def central_fit(func, x, step):
    """Value, gradient and Hessian at x from the full 3^n central-difference
    stencil (x + {-1, 0, 1} step_i in every direction): gradient and Hessian are
    exact for cubic terms along each axis, where the 1 + 2n + n(n-1)/2 point fit
    lets them leak through its single off-diagonal point. The 3^n points are
    one batch of concurrent GPU solves."""
    x = np.asarray(x, dtype=np.float64)
    n = len(x)
    s = np.asarray(step, dtype=np.float64)
    offs = np.array(np.meshgrid(*[[-1, 0, 1]] * n, indexing="ij")).reshape(n, -1).T
    y = func(x + offs * s)
    idx = {tuple(o): i for i, o in enumerate(offs)}
    e = lambda *o: y[idx[tuple(o)]]
    z = [0] * n
    f0 = e(*z)
    grad = np.zeros(n)
    hess = np.zeros((n, n))
    for i in range(n):
        p, m = list(z), list(z)
        p[i], m[i] = 1, -1
        grad[i] = (e(*p) - e(*m)) / (2 * s[i])
        hess[i, i] = (e(*p) + e(*m) - 2 * f0) / (s[i] * s[i])
        for j in range(i):
            q = [list(z) for _ in range(4)]
            for k, (a, b) in enumerate(((1, 1), (1, -1), (-1, 1), (-1, -1))):
                q[k][i], q[k][j] = a, b
            hess[i, j] = hess[j, i] = (e(*q[0]) - e(*q[1]) - e(*q[2]) + e(*q[3])) / (4 * s[i] * s[j])
    return f0, grad, hess


def newton_raphson(func, start, step, accur, gtol: float = 1e-4, max_iteration: int = 30, stencil: str = "central",
                   certify: float | None = None, certify_step: float = 1e-4):
    """Newton-Raphson search for a stationary point (_newton_raphson, pyqcm/vca.py:318-410).
    stencil "reference" fits the reference's 1 + 2n + n(n-1)/2 points;
    "central" (the default here) uses the 3^n central differences of central_fit.

    Both of the reference's exits can fire away from the stationary point: the
    gradient test reads a gradient fitted over the current (possibly large)
    steps, whose cubic terms bias it, and the |dx| <= accur test trusts a Newton
    step from that same fit. With `certify` set, the point where the search stops
    is then certified: the gradient is taken again from a central stencil of
    step `certify_step` (truncation error ~ Omega''' h^2 / 6, round-off ~ noise / h:
    both ~1e-8 at h = 1e-4 for Omega accurate to 1e-12), and Newton steps from
    that small-step fit continue until its |gradient| < certify. The returned
    gradient and Hessian are then the certifying fit's.
    Returns (x, Omega at the last fit point, gradient, Hessian, iterations)."""
    fit = nr_quadratic_fit if stencil == "reference" else central_fit
    x = np.array(start, dtype=np.float64)
    step = np.array(step, dtype=np.float64)
    accur = np.asarray(accur, dtype=np.float64)
    result = None
    for it in range(1, max_iteration + 1):
        val, grad, hess = fit(func, x, step)
        if np.linalg.norm(grad) < gtol:
            result = (x, val, grad, hess, it)
            break
        dx = -np.linalg.solve(hess, grad)
        x = x + dx
        step = np.maximum(np.abs(dx), 2.0 * accur)
        if np.all(np.abs(dx) <= accur):
            result = (x, val, grad, hess, it)
            break
    if result is None:
        raise RuntimeError(f"VCA Newton-Raphson: no convergence after {max_iteration} iterations")
    if certify is None:
        return result
    x, _, _, _, it = result
    cstep = np.full(len(x), float(certify_step))
    for extra in range(max_iteration):
        val, grad, hess = central_fit(func, x, cstep)
        if np.linalg.norm(grad) < certify:
            return x, val, grad, hess, it + extra
        x = x - np.linalg.solve(hess, grad)
    raise RuntimeError(f"VCA Newton-Raphson: gradient not below {certify} after {max_iteration} certifying steps")


def quasi_newton(func, start, step, accur, gtol: float = 1e-4, bfgs: bool = False, max_iteration: int = 30):
    """The reference's quasi-Newton search (_quasi_newton / _quasi_newton_step,
    pyqcm/vca.py:92-236), as it runs: each iteration evaluates the 2n + 1 points
    x, x +/- step_i e_i (one batch), takes the central-difference gradient, and
    moves by dx = -H g. H is diag(step_i^2 / second difference) at the first
    iteration; afterwards the symmetric-rank-1 (or BFGS) update with y = g - g_prev
    is applied to the identity, because the reference's step function starts
    from a fresh identity each call instead of the previous inverse Hessian. The
    gradient test comes after the move; steps are reset as in newton_raphson.
    Returns (x, gradient, inverse-Hessian estimate, iterations)."""
    x = np.array(start, dtype=np.float64)
    step = np.array(step, dtype=np.float64)
    accur = np.asarray(accur, dtype=np.float64)
    n = len(x)
    g = np.zeros(n)
    dx = np.zeros(n)
    for it in range(max_iteration):
        xp = np.tile(x, (2 * n + 1, 1))
        for i in range(n):
            xp[2 * i + 1, i] += step[i]
            xp[2 * i + 2, i] -= step[i]
        F = func(xp)
        g0 = g.copy()
        g = np.array([(F[2 * i + 1] - F[2 * i + 2]) / (2 * step[i]) for i in range(n)])
        ih = np.eye(n)
        if it == 0:
            for i in range(n):
                ih[i, i] = step[i] * step[i] / (F[2 * i + 1] + F[2 * i + 2] - 2 * F[0])
        else:
            y = g - g0
            if bfgs:
                z1 = 1.0 / (1.0e-14 + np.dot(y, dx))
                X = np.eye(n) - z1 * np.outer(y, dx)
                ih = X.T @ ih @ X + z1 * np.outer(dx, dx)
            else:
                dx = dx - ih @ y
                z1 = 1.0 / (1.0e-14 + np.dot(y, dx))
                ih = ih + z1 * np.outer(dx, dx)
        dx = -ih @ g
        x = x + dx
        if np.linalg.norm(g) < gtol or np.all(np.abs(dx) <= accur):
            return x, g, ih, it + 1
        step = np.maximum(np.abs(dx), 2.0 * accur)
    raise RuntimeError(f"VCA quasi-Newton: no convergence after {max_iteration} iterations")


class VCAError(RuntimeError):
    """Failure of the VCA search (pyqcm.SolverError in the reference)."""


class VCA:
    """A VCA computation; the constructor runs it (pyqcm.vca.VCA, pyqcm/vca.py:520-800,
    methods 'NR', 'SYMR1', 'BFGS2').

    model: a lattice.LatticeModel; varia: names of the variational parameters (or
    var2sef: point -> parameter values); start, steps, accur, max: per variable
    (scalars are broadcast); accur_grad: gradient tolerance; freqs, weights, nk: the
    fixed (frequency, k) grid of the Potthoff functional. stencil: 'reference' (the
    reference's 1 + 2n + n(n-1)/2 point fit, default) or 'central' (3^n points, see
    newton_raphson). func: a batched Omega (points -> values) to use instead of the
    GPU evaluator. After the run: x, omega (at x), gradient, hessian, iterations,
    omega_evaluations."""

    def __init__(self, model=None, var2sef=None, varia=None, start=None, steps=0.01, accur=1e-4, max=100,
                 accur_grad=1e-6, max_iter=30, method="NR", freqs=None, weights=None, nk=None, fixed=None,
                 threads: int = 0, stencil: str = "reference", func=None):
        varia = [varia] if isinstance(varia, str) else list(varia or [])
        start = np.atleast_1d(np.asarray(start, dtype=np.float64))
        nvar = len(start)
        steps, accur, maxv = (np.broadcast_to(np.asarray(v, dtype=np.float64), (nvar,)).copy()
                              for v in (steps, accur, max))
        if func is None:
            to_values = var2sef if var2sef is not None else (lambda x: {k: float(v) for k, v in zip(varia, x)})
            func = OmegaEvaluator(model, varia, freqs, weights, nk, fixed=fixed, threads=threads,
                                  to_values=to_values)
        self.omega_evaluations = 0

        def batch(P):
            P = np.atleast_2d(P)
            bad = np.abs(P) > maxv
            if np.any(bad):
                i = int(np.argwhere(bad)[0][1])
                name = varia[i] if i < len(varia) else str(i)
                raise VCAError(f"Failure of the VCA method: parameter {name} is out of bounds!")
            self.omega_evaluations += len(P)
            return np.asarray(func(P), dtype=np.float64)

        try:
            if method == "NR":
                x, _, g, H, it = newton_raphson(batch, start, steps, accur, gtol=accur_grad, max_iteration=max_iter,
                                                stencil=stencil)
            elif method in ("SYMR1", "BFGS2"):
                x, g, iH, it = quasi_newton(batch, start, steps, accur, gtol=accur_grad, bfgs=(method == "BFGS2"),
                                            max_iteration=max_iter)
                H = np.linalg.inv(iH)
            else:
                raise ValueError(f"method {method} unknown in VCA")
        except RuntimeError as e:
            if isinstance(e, VCAError):
                raise
            raise VCAError("Failure of the VCA method") from e
        self.x = x
        self.gradient = g
        self.hessian = H
        self.iterations = it
        self.omega = float(batch(np.array([x]))[0])  # final, converged value


# ------------------------------------------------------------ surrogate path --

def vca_values(x):
    """(U, M', dmu) -> lattice parameters: mu = U/2, M_1 = M', mu_1 = U/2 + dmu."""
    U, M, dmu = (float(v) for v in x)
    return {"U": U, "mu": U / 2, "M_1": M, "mu_1": U / 2 + dmu}


class SurrogateVCA:
    """Potthoff functional surrogate over (U, M', dmu) in a box, trained on ED data.

    Omega varies across the box mostly with U (by about 1 per unit of U) and
    only by 1e-4 to 1e-3 with the variational parameters, below what BF16
    activations resolve on that scale. So the surrogate is a least-squares
    polynomial of total degree 4 in the scaled coordinates (FP64, on the host)
    plus the network fitted to its residual, standardised. Network features:
    the three coordinates scaled to [-1, 1] and the square of the scaled M'.
    `propose(U)` returns the stationary point of the surrogate at that U
    (Newton-Raphson on the surrogate), which the ED search then refines."""

    DEGREE = 4

    def __init__(self, box, width: int = 256, seed: int = 0):
        from pyqcm_b200 import surrogate as S
        self.box = np.asarray(box, dtype=np.float64)  # [[lo, hi] for U, M', dmu]
        self.net = S.MLP(n_in=4, width=width, seed=seed)
        self.mean = 0.0
        self.scale = 1.0
        self.coef = None

    def _scaled(self, X):
        X = np.atleast_2d(np.asarray(X, dtype=np.float64))
        lo, hi = self.box[:, 0], self.box[:, 1]
        return 2.0 * (X - lo) / (hi - lo) - 1.0

    def features(self, X):
        s = self._scaled(X)
        return np.c_[s, s[:, 1] ** 2].astype(np.float32)

    def _poly(self, X):
        s = self._scaled(X)
        cols = [np.ones(len(s))]
        for a in range(self.DEGREE + 1):
            for b in range(self.DEGREE + 1 - a):
                for c in range(self.DEGREE + 1 - a - b):
                    if a + b + c:
                        cols.append(s[:, 0] ** a * s[:, 1] ** b * s[:, 2] ** c)
        return np.stack(cols, axis=1)

    def fit(self, X, y, epochs: int = 400, batch: int = 256, lr: float = 1e-3, seed: int = 0):
        y = np.asarray(y, dtype=np.float64)
        A = self._poly(X)
        self.coef = np.linalg.lstsq(A, y, rcond=None)[0]
        r = y - A @ self.coef
        self.mean = float(np.mean(r))
        self.scale = float(np.std(r)) or 1.0
        return self.net.train(self.features(X), ((r - self.mean) / self.scale).astype(np.float32),
                              epochs=epochs, batch=batch, lr=lr, seed=seed)

    def __call__(self, X, use_net: bool = True):
        base = self._poly(X) @ self.coef
        if not use_net:
            return base
        return base + self.net(self.features(X)).astype(np.float64) * self.scale + self.mean

    def propose(self, U, start, step, accur=(2e-3, 2e-3), use_net: bool = True):
        """Stationary point of the surrogate at U (use_net=False: of the polynomial
        alone). The network's BF16 activations resolve about 1e-3 of the box, so
        the quadratic fits keep steps of that order (accur); the ED search
        refines the proposal."""
        f = lambda P: self(np.c_[np.full(len(P), U), P], use_net=use_net)
        try:
            x, _, _, _, _ = newton_raphson(f, start, step, accur, gtol=0.0, max_iteration=40)
        except (RuntimeError, np.linalg.LinAlgError):
            return np.asarray(start, dtype=np.float64)
        lo, hi = self.box[1:, 0], self.box[1:, 1]
        return np.clip(x, lo, hi)


def training_points(n: int, box, seed: int = 0):
    rng = np.random.default_rng(seed)
    box = np.asarray(box, dtype=np.float64)
    return box[:, 0] + (box[:, 1] - box[:, 0]) * rng.random((n, len(box)))
