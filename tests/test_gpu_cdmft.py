"""CDMFT host function and distance (the lattice layer's CDMFT part) on the GPU
against the reference's own lattice layer (the compiled oracle): 2x2 plaquettes
with eight bath orbitals tiling the square lattice."""
import numpy as np
import pytest

from pyqcm_b200 import workloads as W

pytestmark = pytest.mark.gpu

NAMES = [f"eb{b}_1" for b in range(8)] + [f"tb{b}_1" for b in range(8)]


def test_cdmft_host_and_distance_match_reference(qed, oracle):
    from pyqcm_b200 import lattice as LT
    rng = np.random.default_rng(7)
    prob = W.cdmft_2x2_bath(rng.uniform(-2, 2, 8), rng.uniform(0.2, 1, 8))
    side = 8
    freqs = (2 * np.arange(20) + 1) * np.pi / 50
    weights = np.ones(20) / 20
    qed.set_global_parameter("GF_method", "L")
    oracle.set_param("GF_method", "L")
    oracle.set_param("kgrid_side", side)
    oracle.load_lattice(prob, 0)
    oracle.cdmft_variational_set(NAMES)
    oracle.cdmft_host(0, freqs, weights)
    M = LT.LatticeModel(prob)
    I = M.instance(4300)
    I.ground_state()
    I.Green_function_solve()
    host = LT.CDMFT_host(I, freqs, side=side)
    assert len(host) == 1  # no spin asymmetry: one block
    for iw in range(len(freqs)):
        ref_h = oracle.get_cdmft_host(0, iw)
        assert np.max(np.abs(host[0][iw] - ref_h)) < 1e-6 * max(1.0, np.max(np.abs(ref_h))), iw
    p0 = np.array([prob.params[n] for n in NAMES])
    P = np.vstack([p0, p0 + 0.05, p0 - 0.03 * rng.standard_normal(len(p0))])
    d = LT.CDMFT_distance(M, host, freqs, weights, NAMES, P, base_values=I.values)
    d_ref = np.array([oracle.cdmft_distance(0, p) for p in P])
    assert np.max(np.abs(d - d_ref) / d_ref) < 1e-6, (d, d_ref)
    I.erase()
