"""Host-side accessors of a model instance (no GPU needed) against the
reference's ED on the same model: model_size, exists, matrix_elements,
complex_HS, hopping_matrix, hopping_matrix_full, interactions."""
import numpy as np
import pytest

from pyqcm_b200 import workloads as W
from tests.helpers import load_both


def _bath_model():
    p = W.plaquette_bath(np.linspace(-1.5, 1.5, 8), np.linspace(0.2, 0.9, 8), name="accbath")
    p.operators["tbb"] = ("one-body", [(4, 5, 1.0), (16, 17, 1.0)])  # makes the bath non-diagonal
    p.params["tbb"] = 0.3
    return p


CASES = [
    ("bath", _bath_model),
    ("neel2x4", lambda: W.hubbard_cluster(4, 2, U=5.0, mu=1.7, M=0.25)),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_accessors_match_reference(qed, oracle, fresh, case):
    name, mk = CASES[case]
    prob = mk()
    suffix, label = fresh()
    mname = load_both(qed, oracle, prob, suffix, label, fmt="F")
    assert qed.model_size(mname) == oracle.model_size(mname)
    for op in list(prob.operators) + ["not_an_operator"]:
        assert qed.exists(mname, op) == oracle.exists(mname, op)
    for op in prob.operators:
        assert qed.matrix_elements(mname, op) == oracle.matrix_elements(mname, op), op
    assert qed.complex_HS(label) is False
    assert sorted(qed.interactions(label)) == sorted(oracle.interactions(label))
    up_down = bool(qed.mixing(label) & 4)
    for sd in ([False, True] if up_down else [False]):
        assert np.array_equal(qed.hopping_matrix(sd, label), oracle.hopping_matrix(label, sd))
        if prob.n_bath:
            a = qed.hopping_matrix_full(sd, False, label)
            assert np.array_equal(a, oracle.hopping_matrix_full(label, sd, False))
        else:  # the reference keeps no undiagonalised bath matrices then, and fails
            with pytest.raises(qed.QEDError):
                qed.hopping_matrix_full(sd, False, label)
            with pytest.raises(oracle.OracleError):
                oracle.hopping_matrix_full(label, sd, False)
        # with the bath diagonalised, eigenvector columns are defined up to sign
        a = qed.hopping_matrix_full(sd, True, label)
        b = oracle.hopping_matrix_full(label, sd, True)
        assert np.max(np.abs(np.abs(a) - np.abs(b))) < 1e-12
        assert np.max(np.abs(np.diag(a) - np.diag(b))) < 1e-12
    if not up_down:
        with pytest.raises(qed.QEDError):
            qed.hopping_matrix_full(True, False, label)
