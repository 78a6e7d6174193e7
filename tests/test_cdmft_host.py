"""CDMFT host logic against the reference's lattice layer (the compiled oracle),
on the CPU: the bath hybridisation Gamma(iw) of the analytic bath distance, the
distance itself against lattice_model_instance::CDMFT_distance with the
reference's own host function, the exact Jacobian of the residuals, the
frequency grids, and the CDMFT iterations on a fake step."""
import numpy as np
import pytest

from pyqcm_b200 import workloads as W

NAMES8 = [f"eb{b}_1" for b in range(8)] + [f"tb{b}_1" for b in range(8)]
NAMES4 = [f"eb{b}_1" for b in range(4)] + [f"tb{b}_1" for b in range(4)]


def test_bath_hybridisation_matches_reference(qed, oracle):
    from pyqcm_b200 import cdmft, lattice as LT
    rng = np.random.default_rng(11)
    prob = W.cdmft_2x2_bath(rng.uniform(-2, 2, 8), rng.uniform(0.2, 1, 8))
    oracle.load_lattice(prob, 0)
    M = LT.LatticeModel(prob)
    bd = cdmft.BathDistance(M, NAMES8, prob.params)
    freqs = np.linspace(0.05, 6.0, 17)
    x = np.array([prob.params[n] for n in NAMES8])
    g = bd.gamma(x, freqs)[0]
    want = oracle.hybridization_function(oracle.lattice_ed_label(0), 1j * freqs)
    assert np.max(np.abs(g - want)) < 1e-13
    # another bath point: the product's own ED instance at those values
    x2 = x + rng.normal(0, 0.3, len(x))
    I = M.instance(6100, **dict(zip(NAMES8, x2)))
    want2 = qed.hybridization_function(1j * freqs, label=I.label)  # host data only: no solve, no erase
    assert np.max(np.abs(bd.gamma(x2, freqs)[0] - want2)) < 1e-13


def test_bath_distance_matches_reference(oracle):
    """The reference computes its host function (ED on its own solver, 4 bath
    orbitals: dimension 4900) and its distance at several bath points; the
    analytic distance with that host agrees."""
    from pyqcm_b200 import cdmft, lattice as LT
    rng = np.random.default_rng(5)
    prob = W.cdmft_2x2_bath(rng.uniform(-2, 2, 4), rng.uniform(0.3, 1, 4), U=6.0)
    oracle.set_param("GF_method", "L")
    oracle.set_param("kgrid_side", 8)
    oracle.load_lattice(prob, 0)
    oracle.cdmft_variational_set(NAMES4)
    grid = cdmft.frequency_grid("matsubara", (3.0, 40.0))
    oracle.cdmft_host(0, grid.wr, grid.cdmft_weight)
    host = np.array([[oracle.get_cdmft_host(0, i) for i in range(grid.nw)]])
    M = LT.LatticeModel(prob)
    bd = cdmft.BathDistance(M, NAMES4, prob.params)
    x0 = np.array([prob.params[n] for n in NAMES4])
    for k in range(4):
        x = x0 + (0 if k == 0 else 1) * rng.normal(0, 0.2, len(x0))
        d = bd.distance(x, host, grid.wr, grid.cdmft_weight)
        d_ref = oracle.cdmft_distance(0, x)
        assert abs(d - d_ref) <= 1e-10 * d_ref, (k, d, d_ref)


def test_residual_jacobian_is_exact(qed):
    from pyqcm_b200 import cdmft, lattice as LT
    rng = np.random.default_rng(2)
    prob = W.cdmft_2x2_bath(rng.uniform(-2, 2, 8), rng.uniform(0.2, 1, 8))
    M = LT.LatticeModel(prob)
    bd = cdmft.BathDistance(M, NAMES8, prob.params)
    freqs = cdmft.frequency_grid().wr
    w = np.ones_like(freqs)
    host = -bd.gamma(np.array([prob.params[n] for n in NAMES8]) + 0.1, freqs)
    x = np.array([prob.params[n] for n in NAMES8])
    r, J = bd.residuals(x, host, freqs, w, jac=True)
    h = 1e-6
    for p in range(len(x)):
        e = np.zeros_like(x)
        e[p] = h
        fd = (bd.residuals(x + e, host, freqs, w) - bd.residuals(x - e, host, freqs, w)) / (2 * h)
        assert np.max(np.abs(fd - J[:, p])) < 1e-7 * max(1.0, np.max(np.abs(J[:, p]))), p


def test_bath_minimiser_recovers_a_known_bath(qed):
    """With the host set to -Gamma of a known bath, least squares from a nearby
    start returns a bath with the same hybridisation (distance ~ 0)."""
    from pyqcm_b200 import cdmft, lattice as LT
    rng = np.random.default_rng(9)
    prob = W.cdmft_2x2_bath(rng.uniform(-2, 2, 8), rng.uniform(0.2, 1, 8))
    M = LT.LatticeModel(prob)
    bd = cdmft.BathDistance(M, NAMES8, prob.params)
    grid = cdmft.frequency_grid()
    xt = np.array([prob.params[n] for n in NAMES8])
    host = -bd.gamma(xt, grid.wr)
    x, nfev, d = cdmft.optimize_bath(bd, xt + rng.normal(0, 0.05, len(xt)), host, grid.wr, grid.cdmft_weight)
    assert d < 1e-14, d
    assert np.max(np.abs(bd.gamma(x, grid.wr) - bd.gamma(xt, grid.wr))) < 1e-6


def test_frequency_grids_follow_the_reference():
    from pyqcm_b200 import cdmft
    g = cdmft.frequency_grid()  # Legendre (1, 10, 5, 10, 5)
    assert g.nw == 20 and np.all(np.diff(g.wr) > 0) and g.wr[0] > 0
    # Gauss-Legendre weights integrate 1/pi * int_0^inf dw / (1 + w^2) = 1/2 closely
    assert abs(np.sum(g.weight / (1 + g.wr ** 2)) - 0.5) < 1e-4
    assert np.all(g.cdmft_weight == 1.0)
    m = cdmft.frequency_grid("matsubara", (2.0, 50.0))
    assert np.allclose(m.wr, (2 * np.arange(len(m.wr)) + 1) * np.pi / 50) and m.wr[-1] <= 2.0 + 1e-6
    f = cdmft.frequency_grid("regular", (2.0, 10, 10), opt="ifreq")
    assert abs(f.cdmft_weight.sum() - 1.0) < 1e-14
    with pytest.raises(ValueError):
        cdmft.frequency_grid("gauss")


class _FakeCDMFT:
    """The iteration drivers of CDMFT on a contraction map standing in for the
    ED step (no GPU): x -> A x + b has the fixed point (1 - A)^-1 b."""

    def __init__(self, iteration, alpha):
        from pyqcm_b200 import cdmft
        self.c = cdmft
        obj = cdmft.CDMFT.__new__(cdmft.CDMFT)
        rng = np.random.default_rng(0)
        A = 0.4 * rng.uniform(-1, 1, (3, 3)) / 3
        b = rng.uniform(-1, 1, 3)
        obj.history, obj.dist, obj.E0, obj.host = [], 0.0, 0.0, None
        obj.tests = [cdmft.convergence_manager("parameters", lambda a, c: np.linalg.norm(a - c) / a.shape[0], 1e-9, 2)]

        def step(x):
            xn = A @ x + b
            obj.history.append(np.copy(xn))
            return xn

        obj.step = step
        self.obj, self.fixed = obj, np.linalg.solve(np.eye(3) - A, b)
        x0 = np.zeros(3)
        if iteration == "broyden":
            self.x, self.n = obj._broyden(x0, alpha, 64, 0)
        else:
            self.x, self.n = obj._fixed_point(x0, alpha, 64, 0)


@pytest.mark.parametrize("iteration,alpha", [("broyden", 0.0), ("fixed_point", 0.0), ("fixed_point", (0.3, 4))])
def test_cdmft_iterations_reach_the_fixed_point(iteration, alpha):
    run = _FakeCDMFT(iteration, alpha)
    assert np.max(np.abs(run.x - run.fixed)) < 1e-7, (run.x, run.fixed)
    assert run.n < 64


def test_canonical_bath_keeps_the_hybridisation(qed):
    from pyqcm_b200 import cdmft, lattice as LT
    rng = np.random.default_rng(4)
    prob = W.cdmft_2x2_bath(rng.uniform(-2, 2, 8), rng.uniform(-1, 1, 8))
    M = LT.LatticeModel(prob)
    bd = cdmft.BathDistance(M, NAMES8, prob.params)
    x = np.array([prob.params[n] for n in NAMES8])
    c = cdmft.canonical_bath(x, list(range(8)), list(range(8, 16)), [b // 2 for b in range(8)])
    freqs = np.linspace(0.1, 5, 9)
    assert np.max(np.abs(bd.gamma(c, freqs) - bd.gamma(x, freqs))) < 1e-14
    assert np.all(c[8:] >= 0) and all(c[2 * s] <= c[2 * s + 1] for s in range(4))
    perm = x.copy()
    perm[[0, 1]] = x[[1, 0]]
    perm[[8, 9]] = -x[[9, 8]]
    assert np.array_equal(cdmft.canonical_bath(perm, list(range(8)), list(range(8, 16)), [b // 2 for b in range(8)]), c)
