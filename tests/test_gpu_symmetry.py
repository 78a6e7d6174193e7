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


@pytest.mark.parametrize("case,sectors", [
    ("sq2x3_c2v", ["R0:N6:S0", "R3:N6:S0", "R1:N5:S1"]),
    ("c2v_8b_record", ["R0:N12:S0", "R2:N11:S1"]),
])
def test_mixed_on_the_fly_products_match_the_stored_matrix(qed, oracle, fresh, case, sectors):
    """With no stored matrix (mixed_on_the_fly: every product recomputes the
    entries) H x and the sector's lowest level are those of the CSR form and of
    the reference's CSR Hamiltonian."""
    prob = c2v_problem(c2v_golden(), True) if case == "c2v_8b_record" else _sq2x3_c2v()
    suffix, label = fresh()
    name = "otf" + suffix
    qed.load_problem(prob, label, model_name=name)
    oracle.load_problem(prob, label, model_name=name, fmt="S")
    for sec in sectors:
        qed.set_global_parameter("mixed_on_the_fly", False)
        Hc = qed.MixedHamiltonian(label, sec)
        qed.set_global_parameter("mixed_on_the_fly", True)
        try:
            Ho = qed.MixedHamiltonian(label, sec)
        finally:
            qed.set_global_parameter("mixed_on_the_fly", False)
        R = oracle.RefHamiltonian(label, sec, csr=True)
        x = np.random.default_rng(8).standard_normal(Hc.dim)
        yc, yo, yr = np.zeros(Hc.dim), np.zeros(Hc.dim), np.zeros(Hc.dim)
        Hc.mult_add(x, yc)
        Ho.mult_add(x, yo)
        R.mult_add(x, yr)
        scale = max(1.0, np.max(np.abs(yr)))
        assert np.max(np.abs(yo - yc)) <= 1e-13 * scale and np.max(np.abs(yo - yr)) <= 1e-13 * scale, sec
        if Hc.dim > 256:
            ec, _ = Hc.ground_state_energy()
            eo, _ = Ho.ground_state_energy()
            assert abs(eo - ec) <= 1e-12 * abs(ec), (sec, eo, ec)
        del Hc, Ho, R


def test_mixed_basis_ground_state_matches_reference_record(qed, oracle, fresh):
    """Lanczos on the device in the symmetry-adapted basis of the reference's C2v
    record: the record's ground-state energy (6 digits) and the compiled
    reference's own ground state of that sector (CSR format) to 1e-10."""
    gold = c2v_golden()
    prob = c2v_problem(gold, True)
    suffix, label = fresh()
    name = "mixgs" + suffix
    qed.load_problem(prob, label, model_name=name)
    oracle.set_param("GF_method", "L")
    oracle.load_problem(prob, label, model_name=name, fmt="S")
    e_ref, _ = oracle.ground_state(label)
    H = qed.MixedHamiltonian(label, gold["sectors"])
    e, it = H.ground_state_energy()
    assert abs(e - gold["gs"]["energy"]) < 5.1e-5, e
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref), (e, e_ref, it)


def test_mixed_basis_lowest_levels_per_irrep(qed, fresh):
    """The lowest level of every irrep of a 2x3 Hubbard cluster with C2v
    generators against dense diagonalisation of the numpy restatement's
    mixed-basis matrix (oracle/port_sym.py); the ground-state vector (second
    Lanczos pass) is a unit eigenvector of that matrix."""
    from oracle import port_sym
    prob = _sq2x3_c2v()
    suffix, label = fresh()
    qed.load_problem(prob, label, model_name="mixirr" + suffix)
    G = port_sym.group(6, 0, [[v - 1 for v in g] for g in prob.generators], False)
    for r in range(4):
        sec = f"R{r}:N6:S0"
        Hp, _ = port_sym.mixed_hamiltonian(prob, G, sec)
        e_dense = np.linalg.eigvalsh(Hp.toarray())[0]
        H = qed.MixedHamiltonian(label, sec)
        e, _ = H.ground_state_energy()
        assert abs(e - e_dense) < 1e-10, (sec, e, e_dense)
        e2, psi = H.ground_state()
        assert abs(e2 - e) < 1e-12
        assert abs(np.linalg.norm(psi) - 1.0) < 1e-9
        assert np.linalg.norm(Hp @ psi - e * psi) < 1e-6, sec  # eigenvector of the restated matrix
    # one-electron irreps hold one or two states: the Krylov space is exhausted
    # after one or two steps (a zero beta ends the recurrence and the replay)
    for r in range(4):
        sec = f"R{r}:N1:S1"
        Hp, _ = port_sym.mixed_hamiltonian(prob, G, sec)
        if Hp.shape[0] == 0:
            continue
        assert Hp.shape[0] <= 2, (sec, Hp.shape)
        e_dense = np.linalg.eigvalsh(Hp.toarray())[0]
        H = qed.MixedHamiltonian(label, sec)
        e2, psi = H.ground_state()
        assert abs(e2 - e_dense) < 1e-10, (sec, e2, e_dense)
        assert abs(np.linalg.norm(psi) - 1.0) < 1e-9
        assert np.linalg.norm(Hp @ psi - e2 * psi) < 1e-8, sec


def _solve_both(qed, oracle, prob, label, name, fmt="S"):
    qed.set_global_parameter("GF_method", "L")
    oracle.set_param("GF_method", "L")
    qed.load_problem(prob, label, model_name=name, fmt=fmt)
    oracle.load_problem(prob, label, model_name=name, fmt=fmt)
    return qed.ground_state_solve(label), oracle.ground_state(label)


def test_record_green_function_in_the_symmetry_adapted_basis(qed, oracle, fresh):
    """The reference's C2v record (2x2 plaquette + 8 bath orbitals, generators,
    bath irreps) solved through the ED entries in the symmetry-adapted basis:
    ground state and sector against the record (6 digits) and the compiled
    reference's own solve of the same model (1e-10); G(z) in the site basis,
    built from the per-irrep band-Lanczos Q-matrices, against the reference's
    (5e-8) and, projected on each irrep's symmetric orbital, against the record's
    14-digit poles (1e-7, the oracle's own pin); the averages of every operator
    against the reference's (1e-9).

    Why 5e-8 against the compiled reference. The reference does not reproduce
    this model's G more closely than about 1e-8 from one solve to the next. Its
    CSR Hamiltonian adds the operator terms in the order of a map keyed by the
    operators' heap addresses (src_ed/Hamiltonian/Hamiltonian_CSR.hpp:137-141).
    So the summation order of its sector matrix changes with the heap layout, and
    round-off then moves where its band Lanczos stops. Measured on a B200 over
    seven solves of this model, the same for this solver to the bit, this
    solver's G differed from the reference's by 1.2e-9 to 1.35e-8. The record's
    poles stay the fixed pin."""
    from tests.helpers import C2V_Z, c2v_irrep_gf, project_irreps
    gold = c2v_golden()
    prob = c2v_problem(gold, True)
    suffix, label = fresh()
    (e, sec), (e_ref, sec_ref) = _solve_both(qed, oracle, prob, label, "mixgf" + suffix)
    assert sec == sec_ref == gold["gs"]["sector"]
    assert abs(e - gold["gs"]["energy"]) < 5.1e-5, e
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref), (e, e_ref)
    G = qed.Green_function(C2V_Z, label=label)
    G_ref = oracle.green_function(label, C2V_Z)
    assert np.max(np.abs(G - G_ref)) < 5e-8
    assert np.max(np.abs(project_irreps(G) - c2v_irrep_gf(gold, C2V_Z))) < 1e-7
    z = W.matsubara(64)
    assert np.max(np.abs(qed.Green_function(z, label=label) - oracle.green_function(label, z))) < 5e-8
    ave = {n: (a, v) for n, a, v in qed.cluster_averages(label)}
    for n, a, v in oracle.cluster_averages(label):
        assert abs(ave[n][0] - a) < 1e-9 * max(1.0, abs(a)), (n, ave[n], a)
        assert abs(ave[n][1] - v) < 1e-8 * max(1.0, abs(v)), (n, ave[n], v)


@pytest.mark.parametrize("sectors", ["R0:N6:S0/R1:N6:S0/R2:N6:S0/R3:N6:S0", "R0:N5:S1/R1:N5:S1/R2:N5:S1/R3:N5:S1"])
def test_cluster_with_generators_matches_reference(qed, oracle, fresh, sectors):
    """A 2x3 Hubbard cluster with t' and C2v generators: the lowest state over
    the four irreps of the half-filled (or one-hole) sectors, G(i w_n) on 64
    Matsubara frequencies and the Potthoff functional against the compiled
    reference's symmetry-adapted solve. The hole and electron targets are small
    enough that some go through full diagonalisation (below max_dim_full)."""
    prob = _sq2x3_c2v()
    prob.sectors = sectors
    suffix, label = fresh()
    (e, sec), (e_ref, sec_ref) = _solve_both(qed, oracle, prob, label, "mix23" + suffix)
    assert sec == sec_ref, (sec, sec_ref)
    assert abs(e - e_ref) <= 1e-10 * abs(e_ref), (e, e_ref)
    z = W.matsubara(64)
    assert np.max(np.abs(qed.Green_function(z, label=label) - oracle.green_function(label, z))) < 1e-8
    if "S1" in sectors:
        Gd = qed.Green_function(z, spin_down=True, label=label)
        assert np.max(np.abs(Gd - oracle.green_function(label, z, spin_down=True))) < 1e-8
    assert abs(qed.Potthoff_functional(label) - oracle.potthoff(label)) < 1e-9
