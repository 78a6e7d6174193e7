"""Generates tests/golden/vca_nr.json: the reference's own Newton-Raphson VCA step
functions (_NR_Hessian, _newton_raphson_step, _newton_raphson of pyqcm/vca.py) run
on an analytic test function, and its regular_frequency_grid(2, 32, 32)
(pyqcm/__init__.py), as golden values for pyqcm_b200.vca and workloads.

The functions are taken out of the reference's module source with `ast` (pyqcm
itself cannot be imported here: its compiled extension is not built) and run
with stand-ins for the module globals they read (no MPI, no Hartree couplings,
pyqcm.get_global_parameter('accur_SEF') = 1e-8, prints silenced).

    python tests/golden/make_vca_golden.py
"""
import ast
import json
import os
import sys
import types
import warnings

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from oracle.refpath import reference_file  # noqa: E402

REF = reference_file("pyqcm/vca.py")
REF_INIT = reference_file("pyqcm/__init__.py")  # regular_frequency_grid
WANT = ("_evalF", "_NR_Hessian", "_newton_raphson_step", "_vca_accuracy_warning", "_newton_raphson",
        "_QN_values", "_quasi_newton_step", "_quasi_newton")

A = np.array([[1.3, 0.4], [0.4, -0.7]])
X0 = np.array([0.12, -0.05])


def f(x):
    d = np.asarray(x) - X0
    return 0.5 * d @ A @ d + 0.1 * np.sum(np.sin(3 * x)) + 0.05 * x[0] ** 2 * x[1]


B = np.array([[1.3, 0.4], [0.4, 0.9]])  # positive definite: a minimum for the quasi-Newton runs


def fq(x):
    d = np.asarray(x) - X0
    return 0.5 * d @ B @ d + 0.1 * np.sum(np.sin(3 * x))


def load():
    tree = ast.parse(open(REF).read())
    funcs = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in WANT]
    mod = ast.Module(body=funcs, type_ignores=[])
    stub = types.SimpleNamespace(get_global_parameter=lambda name: 1e-8,
                                 TooManyIterationsError=RuntimeError)
    ns = {"np": np, "pyqcm": stub, "comm": None, "root": False, "verbose": False, "warnings": warnings,
          "current_instance": None, "print": lambda *a, **k: None}
    exec(compile(mod, REF, "exec"), ns)
    return ns


def load_grid():
    tree = ast.parse(open(REF_INIT).read())
    funcs = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name == "regular_frequency_grid"]
    ns = {"np": np}
    exec(compile(ast.Module(body=funcs, type_ignores=[]), REF_INIT, "exec"), ns)
    return ns["regular_frequency_grid"]


def main():
    ns = load()
    gw, gp = load_grid()(2.0, 32, 32)
    x = np.array([0.3, -0.1])
    step = np.array([0.02, 0.03])
    val, grad, hess = ns["_NR_Hessian"](f, x.copy(), step.copy())
    xs, gs, hs = ns["_newton_raphson"](func=f, start=np.array([0.3, -0.1]), step=np.array([0.02, 0.02]),
                                      accur=np.array([1e-6, 1e-6]), max_iteration=30)
    qn = {}
    for bfgs in (False, True):
        xq, gq, hq = ns["_quasi_newton"](func=fq, start=np.array([0.3, -0.1]), step=np.array([0.02, 0.02]),
                                        accur=np.array([1e-6, 1e-6]), bfgs=bfgs, max_iteration=60)
        qn["bfgs" if bfgs else "sr1"] = np.asarray(xq).tolist()
    out = {"qn_x": qn, "B": B.tolist(), "A": A.tolist(), "X0": X0.tolist(), "fit_x": x.tolist(), "fit_step": step.tolist(),
           "fit_val": float(val), "fit_grad": np.asarray(grad).tolist(), "fit_hess": np.asarray(hess).tolist(),
           "nr_start": [0.3, -0.1], "nr_step": [0.02, 0.02], "nr_accur": [1e-6, 1e-6],
           "nr_x": np.asarray(xs).tolist(), "grid_w": np.asarray(gw).tolist(), "grid_p": np.asarray(gp).tolist()}
    with open(os.path.join(HERE, "vca_nr.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print(out)


if __name__ == "__main__":
    main()
