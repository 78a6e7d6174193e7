"""Variational cluster approximation on the GPU: the Newton-Raphson search on
ED Potthoff functionals, and the surrogate-guided search reaching the same
stationary point."""
import numpy as np
import pytest

from pyqcm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _evaluator(qed, U=None):
    from pyqcm_b200 import lattice as LT, vca
    qed.set_global_parameter("GF_method", "L")
    model = LT.LatticeModel(W.square_lattice_vca(2, 2, U=8.0, M1=0.1, mu1=4.0))
    w, p = W.regular_frequency_grid(2.0, 24, 24)
    return model, vca.OmegaEvaluator(model, [], w, p, (16, 16), to_values=vca.vca_values)


def test_surrogate_guided_vca_reaches_the_ed_stationary_point(qed):
    from pyqcm_b200 import vca
    model, ev = _evaluator(qed)
    U = 8.0
    f_ed = lambda P: ev(np.c_[np.full(len(P), U), P])
    acc = [2e-5, 2e-5]
    n0 = ev.n_evals
    x_ed, _, g_ed, _, _ = vca.newton_raphson(f_ed, [0.15, 0.0], [0.02, 0.02], acc, certify=1e-6)
    n_ed = ev.n_evals - n0
    box = [[7.0, 9.0], [0.0, 0.4], [-0.5, 0.5]]
    X = vca.training_points(512, box, seed=1)
    y = ev(X)
    sur = vca.SurrogateVCA(box, width=256, seed=0)
    sur.fit(X, y, epochs=400)
    x0 = sur.propose(U, [0.2, 0.0], [0.02, 0.02])
    n0 = ev.n_evals
    x_s, _, g_s, _, _ = vca.newton_raphson(f_ed, x0, [0.005, 0.005], acc, certify=1e-6)
    n_s = ev.n_evals - n0
    # both end points are certified stationary: |grad Omega| < 1e-6 from a 1e-4 central stencil
    assert np.linalg.norm(g_ed) < 1e-6 and np.linalg.norm(g_s) < 1e-6, (g_ed, g_s)
    assert n_s < n_ed, (n_s, n_ed)  # what the trained surrogate saves: ED evaluations
    om = ev(np.c_[[U, U], np.vstack([x_ed, x_s])])
    assert abs(om[0] - om[1]) < 1e-8, (x_ed, x_s, om)
    assert np.max(np.abs(x_ed - x_s)) < 1e-3


def test_vca_stationary_point_matches_reference(qed, oracle):
    """The same Newton-Raphson search on the reference's Potthoff functional (the
    compiled lattice layer, CPU) and on this solver's (GPU): same stationary point,
    same Omega there within 1e-8."""
    from pyqcm_b200 import vca
    model, ev = _evaluator(qed)
    prob = model.prob
    oracle.set_param("GF_method", "L")
    oracle.load_lattice(prob, 0)
    oracle.set_grids(ev.freqs, ev.weights, ev.nk)
    U = 8.0
    lab = [100]

    def f_ref(P):
        out = []
        for x in np.atleast_2d(P):
            lab[0] += 1
            oracle.lattice_new_instance(lab[0], **vca.vca_values([U, *x]))
            out.append(oracle.lattice_potthoff(lab[0]))
        return np.array(out)

    f_gpu = lambda P: ev(np.c_[np.full(len(P), U), P])
    acc = [2e-5, 2e-5]
    x_ref, *_ = vca.newton_raphson(f_ref, [0.15, 0.0], [0.02, 0.02], acc, certify=1e-6)
    x_gpu, *_ = vca.newton_raphson(f_gpu, [0.15, 0.0], [0.02, 0.02], acc, certify=1e-6)
    assert np.max(np.abs(x_ref - x_gpu)) < 1e-4, (x_ref, x_gpu)
    om_ref = f_ref(np.array([x_ref]))[0]
    om_gpu = f_gpu(np.array([x_gpu]))[0]
    assert abs(om_ref - om_gpu) < 1e-8, (om_ref, om_gpu)
