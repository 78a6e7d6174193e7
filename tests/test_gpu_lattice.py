"""Potthoff functional of the lattice layer (VCA) on the GPU against the
reference's own lattice layer (the compiled oracle) on the same fixed
(frequency, k) grid: the GPU grid integrand against a numpy evaluation from
the same Green function, then Omega itself."""
import numpy as np
import pytest

from pyqcm_b200 import workloads as W

pytestmark = pytest.mark.gpu

OMEGA_TOL = 1e-8   # absolute, per site


def _setup(qed, oracle, nx, ny, M1, mu1, label):
    from pyqcm_b200 import lattice as LT
    prob = W.square_lattice_vca(nx, ny, U=8.0, M1=M1, mu1=mu1)
    qed.set_global_parameter("GF_method", "L")
    oracle.set_param("GF_method", "L")
    oracle.load_lattice(prob, 0)
    M = LT.LatticeModel(prob)
    return M, M.instance(label)


def test_sef_integrand_grid_kernel(qed, oracle):
    """Per-frequency k average of log|det(V(k) G(iw) - 1)| from the GPU against
    numpy with the same V(k) and the same (GPU) cluster Green function."""
    M, I = _setup(qed, oracle, 2, 2, 0.1, None, 4101)
    w = np.array([0.05, 0.4, 1.3, 7.0])
    nk = (6, 5)
    for sd, (V0, inter, _, _) in enumerate(I.V_blocks()):
        got = qed.sef_integrand_grid(V0, [e[0] for e in inter], [e[1] for e in inter], [e[2] for e in inter],
                                     [e[3] for e in inter], w, nk, spin_down=bool(sd), label=I.label)
        G = qed.Green_function(1j * w, spin_down=bool(sd), label=I.label)
        want = np.zeros(len(w))
        for a in range(nk[0]):
            for b in range(nk[1]):
                Vk = I.V((a / nk[0], b / nk[1]), bool(sd))
                for i in range(len(w)):
                    want[i] += np.log(abs(np.linalg.det(Vk @ G[i] - np.eye(M.n))))
        want /= nk[0] * nk[1]
        assert np.max(np.abs(got - want)) < 1e-12 * max(1.0, np.max(np.abs(want))), (sd, got, want)
    I.erase()


@pytest.mark.parametrize("case", [(2, 2, 0.1, None), (2, 2, 0.0, None), (2, 4, 0.07, 3.8)])
def test_potthoff_functional_matches_reference(qed, oracle, case):
    nx, ny, M1, mu1 = case
    M, I = _setup(qed, oracle, nx, ny, M1, mu1, 4200 + nx * 10 + ny)
    w, p = W.regular_frequency_grid(2.0, 24, 24)
    nk = (16, 16)
    oracle.set_grids(w, p, nk)
    om_ref = oracle.lattice_potthoff(0)
    om = I.Potthoff_functional(w, p, nk)
    assert abs(om - om_ref) < OMEGA_TOL, (case, om, om_ref)
    I.erase()
