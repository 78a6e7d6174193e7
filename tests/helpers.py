"""Shared helpers for the parity tests: run one cluster problem through the
product solver and through the CPU oracle with identical options."""
from __future__ import annotations

import numpy as np


def set_both(qed, oracle, **opts):
    for k, v in opts.items():
        qed.set_global_parameter(k, v)
        oracle.set_param(k, v)


def load_both(qed, oracle, prob, suffix, label, fmt="F"):
    """Loads `prob` into both libraries under a unique model name and label.
    fmt is the Hamiltonian_format of both ('F' factorized, 'S' CSR: sectors below
    max_dim_full are diagonalised densely)."""
    name = prob.name + suffix
    qed.load_problem(prob, label, model_name=name, fmt=fmt)
    oracle.load_problem(prob, label, model_name=name, fmt=fmt)
    return name


def rel_err(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(a - b)) / den)
