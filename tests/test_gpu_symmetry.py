"""The Hamiltonian in the symmetry-adapted basis on the GPU (csrc/mixed.cu)
against the reference's own CSR Hamiltonian over its ED_mixed_basis (the
compiled oracle): the basis (sorted representatives) bit-exact, H x to 1e-13."""
import numpy as np
import pytest

from pyqcm_b200 import workloads as W
from tests.helpers import c2v_golden, c2v_problem

pytestmark = pytest.mark.gpu


def _sq2x3_c2v():
    prob = W.hubbard_cluster(3, 2, tp=0.3, U=6.0, mu=2.5)
    prob.generators = [[3, 2, 1, 6, 5, 4], [4, 5, 6, 1, 2, 3]]
    return prob


@pytest.mark.parametrize("case,sectors", [
    ("sq2x3_c2v", ["R0:N6:S0", "R1:N6:S0", "R2:N6:S0", "R3:N6:S0", "R1:N5:S1"]),
    ("c2v_8b_record", ["R0:N12:S0", "R2:N11:S1"]),
])
def test_mixed_hamiltonian_matches_reference_csr(qed, oracle, fresh, case, sectors):
    prob = c2v_problem(c2v_golden(), True) if case == "c2v_8b_record" else _sq2x3_c2v()
    suffix, label = fresh()
    name = "mix" + suffix
    qed.load_problem(prob, label, model_name=name)
    oracle.load_problem(prob, label, model_name=name, fmt="S")
    for sec in sectors:
        H = qed.MixedHamiltonian(label, sec)
        ref_states = oracle.mixed_basis(prob.n_sites, prob.n_bath, prob.generators, prob.bath_irrep, sec)
        assert np.array_equal(H.states(), ref_states), sec
        R = oracle.RefHamiltonian(label, sec, csr=True)
        assert R.dim == H.dim
        x = np.random.default_rng(5).standard_normal(H.dim)
        y0 = np.random.default_rng(6).standard_normal(H.dim)
        y, yr = y0.copy(), y0.copy()
        H.mult_add(x, y)
        R.mult_add(x, yr)
        assert np.max(np.abs(y - yr)) <= 1e-13 * max(1.0, np.max(np.abs(yr))), sec
        del H, R
