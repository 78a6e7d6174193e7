"""The VCA Newton-Raphson restatement (pyqcm_b200.vca) against the reference's own
functions run on an analytic function (golden values from
tests/golden/make_vca_golden.py): the stencil fit and the whole search with the
reference's stencil; and the central stencil reaching the same stationary point."""
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
G = json.load(open(os.path.join(HERE, "golden", "vca_nr.json")))
A = np.array(G["A"])
X0 = np.array(G["X0"])


def f1(x):
    d = np.asarray(x) - X0
    return 0.5 * d @ A @ d + 0.1 * np.sum(np.sin(3 * x)) + 0.05 * x[0] ** 2 * x[1]


def fb(X):
    return np.array([f1(x) for x in np.atleast_2d(X)])


def test_reference_stencil_fit_matches_the_reference():
    from pyqcm_b200 import vca
    val, grad, hess = vca.nr_quadratic_fit(fb, np.array(G["fit_x"]), np.array(G["fit_step"]))
    assert abs(val - G["fit_val"]) < 1e-12
    assert np.max(np.abs(grad - np.array(G["fit_grad"]))) < 1e-10
    assert np.max(np.abs(hess - np.array(G["fit_hess"]))) < 1e-8


def test_newton_raphson_matches_the_reference():
    from pyqcm_b200 import vca
    x, *_ = vca.newton_raphson(fb, G["nr_start"], G["nr_step"], G["nr_accur"], stencil="reference")
    assert np.max(np.abs(x - np.array(G["nr_x"]))) < 1e-9, (x, G["nr_x"])
    xc, *_ = vca.newton_raphson(fb, G["nr_start"], G["nr_step"], G["nr_accur"])  # central stencil
    assert np.max(np.abs(xc - np.array(G["nr_x"]))) < 1e-5, (xc, G["nr_x"])


def test_frequency_grid_matches_the_reference():
    from pyqcm_b200 import workloads as W
    w, p = W.regular_frequency_grid(2.0, 32, 32)
    assert np.max(np.abs(w - np.array(G["grid_w"]))) < 1e-14 * np.max(w)
    assert np.max(np.abs(p - np.array(G["grid_p"]))) < 1e-14 * np.max(p)


def test_quasi_newton_matches_the_reference():
    from pyqcm_b200 import vca
    B = np.array(G["B"])

    def fq(X):
        out = []
        for x in np.atleast_2d(X):
            d = x - X0
            out.append(0.5 * d @ B @ d + 0.1 * np.sum(np.sin(3 * x)))
        return np.array(out)

    for key, bfgs in (("sr1", False), ("bfgs", True)):
        x, *_ = vca.quasi_newton(fq, [0.3, -0.1], [0.02, 0.02], [1e-6, 1e-6], bfgs=bfgs, max_iteration=60)
        assert np.max(np.abs(x - np.array(G["qn_x"][key]))) < 1e-9, (key, x, G["qn_x"][key])


def test_vca_class_methods_and_bounds():
    """pyqcm.vca.VCA's interface on a batched analytic Omega: the three Newton-type
    methods reach the stationary point; a point beyond `max` fails the search."""
    import pytest
    from pyqcm_b200 import vca
    B = np.array(G["B"])

    def fq(X):
        return np.array([0.5 * (x - X0) @ B @ (x - X0) + 0.1 * np.sum(np.sin(3 * x)) for x in np.atleast_2d(X)])

    xs = []
    for method in ("NR", "SYMR1", "BFGS2"):
        V = vca.VCA(varia=["a", "b"], start=[0.3, -0.1], steps=0.02, accur=1e-6, method=method, func=fq,
                    max_iter=60)
        assert V.omega_evaluations > 0 and V.hessian.shape == (2, 2)
        xs.append(V.x)
    assert np.max(np.abs(np.array(xs) - xs[0])) < 1e-4
    with pytest.raises(vca.VCAError, match="out of bounds"):
        vca.VCA(varia=["a", "b"], start=[0.3, -0.1], steps=0.02, accur=1e-6, max=0.2, func=fq)


def test_certified_stationary_point():
    """A functional with strong cubic terms and a flat direction: the reference's
    gradient exit (gtol 1e-4, read off the large-step fit) stops away from the
    stationary point; with certify the search continues on a 1e-4 central stencil
    until |grad| < 1e-6, and ends within 1e-5 of the exact stationary point."""
    from pyqcm_b200 import vca
    from scipy.optimize import fsolve

    def f(x):
        return 0.285 * x[0] ** 2 - 0.0075 * x[1] ** 2 + 0.8 * x[0] ** 3 + 0.02 * x[0] * x[1] - 0.1 * x[0]

    fb2 = lambda X: np.array([f(x) for x in np.atleast_2d(X)])
    grad = lambda x: np.array([0.57 * x[0] + 2.4 * x[0] ** 2 + 0.02 * x[1] - 0.1, -0.015 * x[1] + 0.02 * x[0]])
    xs = fsolve(grad, [0.15, 0.0], xtol=1e-14)
    assert np.linalg.norm(grad(xs)) < 1e-12
    x, *_ = vca.newton_raphson(fb2, [0.3, 0.1], [0.05, 0.05], [2e-5, 2e-5], gtol=1e-3)
    xc, _, g, _, _ = vca.newton_raphson(fb2, [0.3, 0.1], [0.05, 0.05], [2e-5, 2e-5], gtol=1e-3, certify=1e-6)
    assert np.linalg.norm(grad(x)) > 1e-6  # the uncertified exit is not stationary to 1e-6
    assert np.linalg.norm(g) < 1e-6 and np.linalg.norm(grad(xc)) < 2e-6
    assert np.max(np.abs(xc - xs)) < 1e-4, (xc, xs)
