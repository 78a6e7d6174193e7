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


# The reference's C2v record (tests/golden/c2v_8b.json, made by
# tests/golden/make_c2v_golden.py): symmetric orbitals of the four cluster sites
# in the reference's irrep order. Irrep r = a + 2b is odd under the first
# generator (sites 1<->2, 3<->4) when a = 1 and under the second (1<->3, 2<->4)
# when b = 1, as the character phases phi(r, element) = r . element of
# symmetry_group::build (src_ed/symmetry_group.cpp:270-280) order them.
C2V_ORBITALS = 0.5 * np.array([[1, 1, 1, 1], [1, -1, 1, -1], [1, 1, -1, -1], [1, -1, -1, 1]], float)
C2V_Z = np.array([0.1j, 0.5j, 1j, 2j, 5j, -1 + 0.2j, 2 + 0.3j])


def c2v_golden():
    import json
    import os
    return json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c2v_8b.json")))


def c2v_problem(golden, with_generators: bool):
    """The record's cluster as a workloads.ClusterProblem; without the generators
    it is the same Hamiltonian on the unsymmetrised (g = 1) basis."""
    from pyqcm_b200 import workloads as W
    m = golden["model"]
    p = W.ClusterProblem(m["name"], m["n_sites"], m["n_bath"],
                         {k: (t, [tuple(e) for e in el]) for k, (t, el) in golden["operators"].items()},
                         dict(golden["params"]), golden["sectors"])
    if with_generators:
        p.generators, p.bath_irrep = m["generators"], m["bath_irrep"]
    return p


def c2v_irrep_gf(golden, z):
    """G_r(z) = sum_i v_i^2 / (z - e_i) from the record's poles, one row per irrep."""
    out = []
    for blk in golden["irrep_poles"]:
        e, v = np.array(blk["e"]), np.array(blk["v"])
        out.append([np.sum(v * v / (zz - e)) for zz in z])
    return np.array(out)


def project_irreps(G):
    """G: (nz, 4, 4) site-basis Green functions -> (4, nz) irrep diagonal s_r^T G s_r."""
    return np.einsum("ra,zab,rb->rz", C2V_ORBITALS, G, C2V_ORBITALS)
