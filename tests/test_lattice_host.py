"""Lattice layer (VCA) host logic against the reference's own lattice layer
(the compiled oracle): the cluster's ED operators, the cluster one-body matrix
and V(k) = t(k) - t' on a few wavevectors. No GPU calls."""
import numpy as np
import pytest

from pyqcm_b200 import workloads as W


@pytest.mark.parametrize("geom", [(2, 2, 0.1, None), (2, 4, 0.05, 3.7), (4, 2, 0.2, None)])
def test_lattice_operators_and_V_match_reference(qed, oracle, geom):
    from pyqcm_b200 import lattice as LT
    nx, ny, M1, mu1 = geom
    prob = W.square_lattice_vca(nx, ny, U=8.0, M1=M1, mu1=mu1)
    oracle.set_param("GF_method", "L")
    oracle.load_lattice(prob, 0)
    M = LT.LatticeModel(prob)
    mix, dim_gf, nsys = oracle.lattice_dims()
    assert (mix, dim_gf, nsys) == (M.mixing, M.n, 1)
    for op in ("t", "mu", "U"):
        assert sorted(oracle.matrix_elements("clus", op)[1]) == sorted(qed.matrix_elements(M.cluster_model, op)[1]), op
    I = M.instance(900 + nx * 10 + ny)
    rng = np.random.default_rng(5)
    for sd in (False, True):
        Hc = qed.hopping_matrix(spin_down=sd, label=I.label)
        assert np.max(np.abs(Hc - oracle.lattice_cluster_hopping(0, sd))) < 1e-14
        for k in [(0.0, 0.0), (0.5, 0.5), tuple(rng.uniform(0, 1, 2))]:
            assert np.max(np.abs(I.V(k, sd) - oracle.lattice_V(0, 0.5j, k, sd))) < 1e-13, (sd, k)


def test_frequency_grid_weights():
    """The midpoint grid integrates 1/pi * int_0^inf dw/(1 + w^2) = 1/2 closely."""
    w, p = W.regular_frequency_grid(2.0, 200, 200)
    assert abs(np.sum(p / (1 + w * w)) - 0.5) < 1e-4
    assert np.all(np.diff(w) > 0)


def test_nr_fit_recovers_a_quadratic():
    from pyqcm_b200 import vca
    A = np.array([[2.0, 0.3], [0.3, -1.0]])
    x0 = np.array([0.1, -0.2])
    f = lambda X: np.array([0.5 * (x - x0) @ A @ (x - x0) + 3.0 for x in np.atleast_2d(X)])
    val, g, H = vca.nr_quadratic_fit(f, np.array([0.3, 0.1]), [0.01, 0.01])
    assert np.allclose(H, A, atol=1e-8) and np.allclose(g, A @ (np.array([0.3, 0.1]) - x0), atol=1e-8)
    x, *_ = vca.newton_raphson(f, [0.3, 0.1], [0.01, 0.01], [1e-8, 1e-8])
    assert np.allclose(x, x0, atol=1e-8)


def test_bath_lattice_model_matches_reference(qed, oracle):
    """The CDMFT model (2x2 plaquettes with eight bath orbitals): the cluster's ED
    operators, its one-body matrix and V(k) = t(k) - t' - Gamma(w) against the
    reference's lattice layer."""
    from pyqcm_b200 import lattice as LT
    rng = np.random.default_rng(3)
    prob = W.cdmft_2x2_bath(rng.uniform(-2, 2, 8), rng.uniform(0.2, 1, 8))
    oracle.set_param("GF_method", "L")
    oracle.load_lattice(prob, 0)
    M = LT.LatticeModel(prob)
    for op in ("t", "mu", "U", "eb3", "tb5"):
        assert sorted(oracle.matrix_elements("clus", op)[1]) == sorted(qed.matrix_elements(M.cluster_model, op)[1]), op
    I = M.instance(990)
    assert np.max(np.abs(qed.hopping_matrix(label=I.label) - oracle.lattice_cluster_hopping(0))) < 1e-14
    w = 0.5j
    gamma = qed.hybridization_function(w, label=I.label)
    for k in [(0.0, 0.0), (0.25, 0.5), tuple(rng.uniform(0, 1, 2))]:
        assert np.max(np.abs(I.V(k) - gamma - oracle.lattice_V(0, w, k))) < 1e-13, k


def test_tilted_superlattice_2x5_matches_reference(qed, oracle):
    """The VCA bench's lattice: 2x5 clusters on the superlattice (2,0), (1,5), which
    keeps the Neel vector commensurate; operators, H_c and V(k) against the reference."""
    from pyqcm_b200 import lattice as LT
    prob = W.vca_2x5(U=7.0, M1=0.12, dmu=0.1)
    oracle.set_param("GF_method", "L")
    oracle.load_lattice(prob, 0)
    M = LT.LatticeModel(prob)
    assert oracle.lattice_dims()[:2] == (M.mixing, M.n)
    for op in ("t", "mu", "U"):  # (the Weiss field enters through H_c, compared below)
        assert sorted(oracle.matrix_elements("clus", op)[1]) == sorted(qed.matrix_elements(M.cluster_model, op)[1]), op
    I = M.instance(995)
    rng = np.random.default_rng(9)
    for sd in (False, True):
        assert np.max(np.abs(qed.hopping_matrix(spin_down=sd, label=I.label) -
                             oracle.lattice_cluster_hopping(0, sd))) < 1e-14
        for k in [(0.0, 0.0), (0.3, 0.7), tuple(rng.uniform(0, 1, 2))]:
            assert np.max(np.abs(I.V(k, sd) - oracle.lattice_V(0, 0.4j, k, sd))) < 1e-13, (sd, k)


def test_incommensurate_density_wave_is_rejected_like_the_reference(qed, oracle):
    """A Neel vector incommensurate with a 2x3 tiling: both lattice layers refuse it."""
    from pyqcm_b200 import lattice as LT
    prob = W.square_lattice_vca(2, 3, U=8.0, M1=0.1)
    with pytest.raises(oracle.OracleError, match="incommensurate"):
        oracle.load_lattice(prob, 0)
    with pytest.raises(ValueError, match="incommensurate"):
        LT.LatticeModel(prob)
