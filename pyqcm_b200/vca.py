"""Variational cluster approximation: stationary points of the Potthoff
functional Omega over cluster (Weiss) parameters, with the cluster problems
solved by this package's GPU ED.

The search is the reference's Newton-Raphson method (pyqcm/vca.py:239-430):
every iteration fits a quadratic form through 1 + 2n + n(n-1)/2 points around
the current x (the n +/- step pairs and n(n-1)/2 off-diagonal points at
0.707 step), moves by dx = -H^{-1} g, then resets each step to |dx_i| (at most
twice the initial step, at least twice the accuracy); it stops when every
|dx_i| <= accur_i or |g| < gtol. Here the points of one iteration are solved
as one batch (their ground states and Green functions concurrently on the GPU,
then their Omega on the GPU grid).
"""
from __future__ import annotations

import time

import numpy as np

import pyqcm_b200 as qed
from pyqcm_b200 import lattice as LT


class OmegaEvaluator:
    """Omega at batches of points of the variational parameters `varia`."""

    def __init__(self, model: LT.LatticeModel, varia, freqs, weights, nk, fixed=None, threads: int = 0,
                 label0: int = 700000):
        self.model = model
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
            vals.update({k: float(v) for k, v in zip(self.varia, x)})
            self.label += 1
            insts.append(self.model.instance(self.label, **vals))
        labels = [I.label for I in insts]
        try:
            qed.ground_state_solve_batch(labels, threads=self.threads)
            qed.Green_function_solve_batch(labels, threads=self.threads)
            out = np.array([I.Potthoff_functional(self.freqs, self.weights, self.nk) for I in insts])
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


def newton_raphson(func, start, step, accur, gtol: float = 1e-4, max_iteration: int = 30):
    """Newton-Raphson search for a stationary point (_newton_raphson, pyqcm/vca.py:318-410).
    Returns (x, Omega at x from the last fit, gradient, Hessian, iterations)."""
    x = np.array(start, dtype=np.float64)
    step0 = np.array(step, dtype=np.float64)
    step = step0.copy()
    accur = np.asarray(accur, dtype=np.float64)
    for it in range(1, max_iteration + 1):
        val, grad, hess = nr_quadratic_fit(func, x, step)
        if np.linalg.norm(grad) < gtol:
            return x, val, grad, hess, it
        dx = -np.linalg.solve(hess, grad)
        x = x + dx
        step = np.abs(dx)
        step = np.where(step > step0, 2.0 * step0, step)
        step = np.where(step < 2.0 * accur, 2.0 * accur, step)
        if np.all(np.abs(dx) <= accur):
            return x, val, grad, hess, it
    raise RuntimeError(f"VCA Newton-Raphson: no convergence after {max_iteration} iterations")
