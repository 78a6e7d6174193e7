"""The CDMFT self-consistency loop on the GPU ED (pyqcm_b200.cdmft) and the
learned starting bath.

* The converged bath is a fixed point of the reference's own CDMFT map: at that
  bath the reference (the compiled oracle, ED on the CPU) computes a host function
  equal to ours, and minimising its distance from there leaves the bath in place.
* The bath surrogate, trained on baths this solver converges, starts CDMFT runs at
  new lattice parameters closer to self-consistency than the model's own bath:
  the runs take fewer ED solves and reach the same solution."""
import time

import numpy as np
import pytest

from pyqcm_b200 import workloads as W

pytestmark = pytest.mark.gpu

NAMES4 = [f"eb{b}_1" for b in range(4)] + [f"tb{b}_1" for b in range(4)]
NAMES8 = [f"eb{b}_1" for b in range(8)] + [f"tb{b}_1" for b in range(8)]


def test_cdmft_fixed_point_matches_reference(qed, oracle):
    from pyqcm_b200 import cdmft, lattice as LT
    rng = np.random.default_rng(42)
    prob = W.cdmft_2x2_bath(rng.uniform(-2, 2, 4), rng.uniform(0.2, 1, 4), U=6.0)
    qed.set_global_parameter("GF_method", "L")
    side = 16
    grid = cdmft.frequency_grid()
    M = LT.LatticeModel(prob)
    run = cdmft.CDMFT(M, NAMES4, method="trf", accur=1e-7, maxiter=60, side=side, label=610000, grid=grid)
    x = run.x
    # the reference at the converged bath
    oracle.set_param("GF_method", "L")
    oracle.set_param("kgrid_side", side)
    vals = dict(prob.params)
    vals.update(dict(zip(NAMES4, x)))
    prob_x = W.LatticeProblem(**{**prob.__dict__, "params": vals})
    oracle.load_lattice(prob_x, 0)
    oracle.cdmft_variational_set(NAMES4)
    oracle.cdmft_host(0, grid.wr, grid.cdmft_weight)
    host_ref = np.array([[oracle.get_cdmft_host(0, i) for i in range(grid.nw)]])
    I = M.instance(610999, **dict(zip(NAMES4, x)))
    I.ground_state()
    I.Green_function_solve()
    host = np.array(LT.CDMFT_host(I, grid.wr, side=side))
    I.erase()
    run.I.erase()
    assert np.max(np.abs(host - host_ref)) < 1e-8 * max(1.0, np.max(np.abs(host_ref)))
    bd = cdmft.BathDistance(M, NAMES4, prob.params)
    x2, _, d2 = cdmft.optimize_bath(bd, x, host_ref, grid.wr, grid.cdmft_weight, method="trf")
    assert np.max(np.abs(x2 - x)) < 1e-5, np.max(np.abs(x2 - x))
    assert abs(oracle.cdmft_distance(0, x2) - d2) <= 1e-10 * d2


def test_bath_surrogate_shortens_cdmft(qed):
    """2x2 plaquette with eight bath orbitals (the cluster of the bath-point batch),
    half filling, U in [6.5, 10]: baths converged by continuation at 15 values of U
    train the network; at three U between them the run from the proposed bath takes
    fewer ED solves than the run from the model's bath and ends at the same
    hybridisation function. (Below U ~ 6 this cluster has a second, metallic
    solution branch, and in the range where both exist the two starts may end on
    different branches; the box stays on the insulating one.)"""
    from pyqcm_b200 import cdmft, lattice as LT
    rng = np.random.default_rng(7)
    prob = W.cdmft_2x2_bath(rng.uniform(-2, 2, 8), rng.uniform(0.3, 1, 8), U=6.0)
    qed.set_global_parameter("GF_method", "L")
    M = LT.LatticeModel(prob)
    canon = lambda x: cdmft.canonical_bath(x, list(range(8)), list(range(8, 16)), [b // 2 for b in range(8)])
    args = dict(method="trf", accur=1e-5, maxiter=60, side=16)
    Us = np.linspace(6.5, 10.0, 15)
    x0 = np.array([prob.params[n] for n in NAMES8])
    t0 = time.time()
    ok, baths, iters = cdmft.converge_baths(M, NAMES8, ["U"], Us[:, None], x0, canonical=canon, label=620000,
                                            **args)
    t_data = time.time() - t0
    print(f"training points converged: {len(ok)} of {len(Us)}, iterations {iters.tolist()}")
    assert len(ok) >= 12
    sur = cdmft.BathSurrogate(["U"], [(6.5, 10.0)], NAMES8, seed=1)
    losses = sur.fit(Us[ok, None], baths, epochs=800, seed=2)
    assert losses[-1] < 0.05 * losses[0]
    gains = []
    for k, U in enumerate((7.1, 8.3, 9.4)):
        vals = dict(prob.params, U=U)
        plain = cdmft.CDMFT(M, NAMES8, values=vals, label=630000 + 10 * k, **args)
        guided = cdmft.CDMFT(M, NAMES8, values=vals, start=sur.propose([U]), label=640000 + 10 * k, **args)
        g1 = cdmft.BathDistance(M, NAMES8, vals).gamma(plain.x, plain.grid.wr)
        g2 = cdmft.BathDistance(M, NAMES8, vals).gamma(guided.x, guided.grid.wr)
        plain.I.erase()
        guided.I.erase()
        assert np.max(np.abs(g1 - g2)) < 1e-3, (U, np.max(np.abs(g1 - g2)))
        assert abs(plain.E0 - guided.E0) < 1e-4 * abs(plain.E0)
        gains.append((plain.n_solves, guided.n_solves))
    print(f"training data {t_data:.1f} s; ED solves (plain, surrogate) per U: {gains}")
    assert all(g <= p for p, g in gains) and sum(g for _, g in gains) < sum(p for p, _ in gains)
