"""GPU parity of the hot path against the reference's own ED (the CPU oracle).

Tolerances: basis indices, ranks and signs bit-exact; H.v within 1e-13
relative (FP64 round-off of a different summation order); ground-state
energies within 1e-10 relative; G(i w_n) within 1e-8 (absolute, on the
Matsubara grid of beta = 50, where |G| <= 1/w_0 ~ 16).
"""
import numpy as np
import pytest

from pyqcm_b200 import workloads as W
from tests.helpers import load_both, rel_err, set_both

pytestmark = pytest.mark.gpu

GS_TOL = 1e-10
GF_TOL = 1e-8


@pytest.mark.parametrize("L,N", [(4, 2), (8, 4), (8, 3), (10, 5), (12, 6), (16, 8), (16, 9), (7, 0), (7, 7)])
def test_halfbasis_bit_exact(qed, oracle, L, N):
    a = qed.halfbasis(L, N)
    b = oracle.halfbasis(L, N)
    assert a.dtype == np.uint32 and np.array_equal(a, b)
    r = qed.halfbasis_rank(L, N, b)
    assert np.array_equal(r, np.arange(len(b), dtype=np.uint32))
    # strings outside the basis rank to dim (ED_halfbasis::index)
    bad = np.array([0xFFFFFFFF, (1 << L) | 1], dtype=np.uint32)
    assert np.all(qed.halfbasis_rank(L, N, bad) == len(b))


@pytest.mark.parametrize("L,nu,nd,a", [(6, 3, 3, 0), (6, 3, 3, 5), (6, 3, 2, 7), (6, 3, 3, 11), (8, 4, 4, 3),
                                       (8, 4, 4, 12), (5, 1, 4, 9)])
def test_destroy_table_bit_exact(qed, oracle, L, nu, nd, a):
    t1, p1 = qed.destroy_table(L, nu, nd, a)
    t2, p2 = oracle.destroy_table(L, nu, nd, a)
    assert np.array_equal(t1, t2)
    assert np.array_equal(p1[t1 >= 0], p2[t2 >= 0] % 2)


def _hv_problems():
    return [
        ("chain8", W.chain8(), "R0:N8:S0"),
        ("chain8_N7", W.hubbard_cluster(8, 1, U=3.0, n_up=4, n_dn=3), "R0:N7:S1"),
        ("sq2x3_tp", W.hubbard_cluster(3, 2, tp=0.3, U=6.0), "R0:N6:S0"),
        ("neel2x4", W.hubbard_cluster(4, 2, U=5.0, mu=1.7, M=0.25), "R0:N8:S0"),
        ("plaq8b", W.plaquette_bath(np.linspace(-1.5, 1.5, 8), np.linspace(0.2, 0.9, 8)), "R0:N12:S0"),
        ("plaq8b_p", W.plaquette_bath(np.linspace(-1.5, 1.5, 8), np.linspace(0.2, 0.9, 8)), "R0:N13:S1"),
        # spin tables of 3432 / 3003 strings: the staged-row kernels with packed hops
        # (both passes; dd odd in the second; du odd in the third takes the ELL kernels)
        ("sq2x7_tp", W.hubbard_cluster(7, 2, tp=0.3, U=6.0, mu=2.9), "R0:N14:S0"),
        ("sq2x7_tp_N13", W.hubbard_cluster(7, 2, tp=0.3, U=6.0, mu=2.9), "R0:N13:S1"),
        ("sq2x7_tp_N13m", W.hubbard_cluster(7, 2, tp=0.3, U=6.0, mu=2.9), "R0:N13:S-1"),
        ("neel2x7", W.hubbard_cluster(7, 2, U=5.0, mu=2.2, M=0.2), "R0:N14:S0"),
    ]


@pytest.mark.parametrize("case", range(10))
def test_hv_matches_reference(qed, oracle, fresh, case):
    name, prob, sec = _hv_problems()[case]
    suffix, label = fresh()
    load_both(qed, oracle, prob, suffix, label, fmt="F")
    Hq = qed.Hamiltonian(label, sec)
    Hr = oracle.RefHamiltonian(label, sec)
    assert Hq.dim == Hr.dim
    rng = np.random.default_rng(7 + case)
    x = rng.standard_normal(Hq.dim)
    y0 = rng.standard_normal(Hq.dim)
    y1, y2 = y0.copy(), y0.copy()
    Hq.mult_add(x, y1)
    Hr.mult_add(x, y2)
    assert rel_err(y1, y2) < 1e-13, name
    # diagonal via unit vectors on a few entries
    d = Hq.diag()
    for i in rng.integers(0, Hq.dim, 5):
        e = np.zeros(Hq.dim)
        e[i] = 1.0
        y = np.zeros(Hq.dim)
        Hr.mult_add(e, y)
        assert abs(d[i] - y[i]) < 1e-12


GS_CASES = [
    ("chain8", lambda: W.chain8()),
    ("sq2x3_tp", lambda: W.hubbard_cluster(3, 2, tp=0.3, U=6.0)),
    ("neel2x4", lambda: W.hubbard_cluster(4, 2, U=5.0, mu=1.7, M=0.25)),
    ("plaq8b", lambda: W.plaquette_bath(np.linspace(-1.5, 1.5, 8), np.linspace(0.2, 0.9, 8))),
    ("chain10", lambda: W.hubbard_cluster(10, 1, U=7.0)),
]


@pytest.mark.parametrize("case", range(len(GS_CASES)))
def test_ground_state_energy(qed, oracle, fresh, case):
    name, mk = GS_CASES[case]
    suffix, label = fresh()
    set_both(qed, oracle, GF_method="L")
    load_both(qed, oracle, mk(), suffix, label, fmt="F")
    e1, s1 = qed.ground_state_solve(label)
    e2, s2 = oracle.ground_state(label)
    assert abs(e1 - e2) <= GS_TOL * abs(e2), (name, e1, e2)
    assert s1 == s2


@pytest.mark.parametrize("case", range(len(GS_CASES)))
def test_green_function_band_lanczos(qed, oracle, fresh, case):
    name, mk = GS_CASES[case]
    suffix, label = fresh()
    set_both(qed, oracle, GF_method="L")
    load_both(qed, oracle, mk(), suffix, label, fmt="F")
    z = W.matsubara(256)
    G1 = qed.Green_function(z, label=label)
    G2 = oracle.green_function(label, z)
    assert np.max(np.abs(G1 - G2)) < GF_TOL, name
    if qed.mixing(label) & 4:
        G1d = qed.Green_function(z, spin_down=True, label=label)
        G2d = oracle.green_function(label, z, spin_down=True)
        assert np.max(np.abs(G1d - G2d)) < GF_TOL, name
    assert abs(qed.Potthoff_functional(label) - oracle.potthoff(label)) < 1e-9
    M1 = qed.Green_function_average(label=label)
    M2 = oracle.green_function_average(label)
    assert np.max(np.abs(M1 - M2)) < 1e-8


@pytest.mark.parametrize("case", [0, 1, 2])
def test_green_function_continued_fraction(qed, oracle, fresh, case):
    name, mk = GS_CASES[case]
    suffix, label = fresh()
    set_both(qed, oracle, GF_method="F")
    try:
        load_both(qed, oracle, mk(), suffix, label, fmt="S")
        z = W.matsubara(256)
        G1 = qed.Green_function(z, label=label)
        G2 = oracle.green_function(label, z)
    finally:
        set_both(qed, oracle, GF_method="L")
    assert np.max(np.abs(G1 - G2)) < GF_TOL, name


def test_self_energy_and_hybridization(qed, oracle, fresh):
    suffix, label = fresh()
    set_both(qed, oracle, GF_method="L")
    prob = W.plaquette_bath(np.linspace(-1.5, 1.5, 8), np.linspace(0.2, 0.9, 8))
    load_both(qed, oracle, prob, suffix, label, fmt="F")
    z = W.matsubara(32)
    S1 = qed.self_energy(z, label=label)
    oracle.green_solve(label)  # the reference's self_energy needs a solved GF (src_ed/model_instance.hpp:683-700)
    S2 = oracle.self_energy(label, z)
    assert np.max(np.abs(S1 - S2)) < 1e-6
    H1 = qed.hybridization_function(z, label=label)
    H2 = oracle.hybridization_function(label, z)
    assert np.max(np.abs(H1 - H2)) < 1e-12


def test_apply_dots_device_matches_host_path(qed, oracle, fresh):
    """Fused H.v + Lanczos reductions on device pointers (torch-owned memory)."""
    import torch
    suffix, label = fresh()
    prob = W.hubbard_cluster(4, 2, U=5.0, mu=1.7, M=0.25)
    load_both(qed, oracle, prob, suffix, label, fmt="F")
    H = qed.Hamiltonian(label, prob.sectors)
    Hr = oracle.RefHamiltonian(label, prob.sectors)
    x = np.random.default_rng(3).standard_normal(H.dim)
    xd = torch.tensor(x, device="cuda")
    yd = torch.empty_like(xd)
    dots = torch.zeros(3, dtype=torch.float64, device="cuda")
    H.apply_dots_device(xd.data_ptr(), yd.data_ptr(), dots.data_ptr(), torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    y_ref = np.zeros(H.dim)
    Hr.mult_add(x, y_ref)
    y = yd.cpu().numpy()
    assert rel_err(y, y_ref) < 1e-13
    d = dots.cpu().numpy()
    assert abs(d[0] - x @ y_ref) < 1e-10 * abs(x @ y_ref)
    assert abs(d[1] - y_ref @ y_ref) < 1e-10 * (y_ref @ y_ref)
    assert abs(d[2] - x @ x) < 1e-12 * (x @ x)


def test_apply_dots_device_staged_kernels(qed, oracle, fresh):
    """The fused H.v + reductions on a sector large enough for the staged-row
    kernels (2x7 cluster with t', 3432 x 3432 states): TMA-staged column pass,
    reductions in its epilogue; y, <x,y>, <y,y>, <x,x> against the reference."""
    import torch
    suffix, label = fresh()
    prob = W.hubbard_cluster(7, 2, tp=0.3, U=6.0, mu=2.9)
    load_both(qed, oracle, prob, suffix, label, fmt="F")
    H = qed.Hamiltonian(label, prob.sectors)
    Hr = oracle.RefHamiltonian(label, prob.sectors)
    x = np.random.default_rng(5).standard_normal(H.dim)
    xd = torch.tensor(x, device="cuda")
    yd = torch.empty_like(xd)
    dots = torch.zeros(3, dtype=torch.float64, device="cuda")
    for _ in range(2):  # a second call on the same buffers gives the same result
        H.apply_dots_device(xd.data_ptr(), yd.data_ptr(), dots.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        y_ref = np.zeros(H.dim)
        Hr.mult_add(x, y_ref)
        y = yd.cpu().numpy()
        assert rel_err(y, y_ref) < 1e-13
        d = dots.cpu().numpy()
        assert abs(d[0] - x @ y_ref) < 1e-10 * abs(x @ y_ref)
        assert abs(d[1] - y_ref @ y_ref) < 1e-10 * (y_ref @ y_ref)
        assert abs(d[2] - x @ x) < 1e-12 * (x @ x)
    # the autotuner timed every launch shape on this sector; they wrote the same bits
    rec = [t for t in qed.hv_tuning_report() if (t["dim_up"], t["dim_dn"]) == (3432, 3432)]
    assert rec and all(t["bit_identical"] for t in rec), rec


def test_ground_state_staged_kernels(qed, oracle, fresh):
    """Lanczos ground state of a 924^2-state sector (the staged-row kernels with
    the subtraction list and the fused reductions) against the reference."""
    suffix, label = fresh()
    prob = W.hubbard_cluster(6, 2, tp=0.3, U=6.0, mu=3.0)
    prob.sectors = "R0:N12:S0"
    load_both(qed, oracle, prob, suffix, label, fmt="F")
    e1, s1 = qed.ground_state_solve(label)
    e2, s2 = oracle.ground_state(label)
    assert abs(e1 - e2) <= 1e-10 * abs(e2), (e1, e2)
    assert s1 == s2


def test_lanczos_graphs_replay_the_same_steps(qed, oracle, fresh):
    """The ground-state Lanczos of a 924^2-state sector with its 16-step chunks
    replayed from CUDA graphs gives the bits of the directly launched chunks and
    the reference's energy; so does a 63504-state sector (chain of 10 sites) with
    the graphs' size threshold lowered to include it."""
    def solve(prob, graphs, min_dim=None):
        suffix, label = fresh()
        qed.set_global_parameter("lanczos_graphs", graphs)
        if min_dim is not None:
            qed.set_global_parameter("lanczos_graphs_min_dim", min_dim)
        load_both(qed, oracle, prob, suffix, label, fmt="F")
        try:
            return qed.ground_state_solve(label), label
        finally:
            qed.set_global_parameter("lanczos_graphs", True)
            qed.set_global_parameter("lanczos_graphs_min_dim", 131072)

    prob = W.hubbard_cluster(6, 2, tp=0.3, U=6.0, mu=3.0)
    prob.sectors = "R0:N12:S0"
    (e1, s1), _ = solve(prob, False)
    (e2, s2), label = solve(prob, True)
    e_ref, s_ref = oracle.ground_state(label)
    assert e1 == e2 and s1 == s2 == s_ref, (e1, e2)
    assert abs(e2 - e_ref) <= 1e-10 * abs(e_ref)
    chain = W.hubbard_cluster(10, 1, U=4.0, mu=2.0)
    chain.sectors = "R0:N10:S0"
    (c1, _), _ = solve(chain, False)
    (c2, _), _ = solve(chain, True, min_dim=0)
    assert c1 == c2, (c1, c2)


def test_batched_solves_match_reference(qed, oracle, fresh):
    """Many random clusters (every sector listed, staggered field) solved concurrently."""
    probs = W.random_batch(12, seed=77, geoms=[(2, 2), (2, 3), (2, 4), (8, 1)])
    labels = []
    for p in probs:
        suffix, label = fresh()
        load_both(qed, oracle, p, suffix, label, fmt="F")
        labels.append(label)
    set_both(qed, oracle, GF_method="L")
    e = qed.ground_state_solve_batch(labels, threads=6)
    qed.Green_function_solve_batch(labels, threads=6)
    z = W.matsubara(64)
    # The band Lanczos deflates a vector whose norm falls below accur_deflation
    # (1e-7). Where a norm lands at that threshold the decision follows the last
    # bits of the arithmetic, and the reference's own G moves by O(1e-7) from one
    # process to the next (its OpenMP reductions are not ordered; this library's
    # result is bit-identical across runs and thread counts). One such instance
    # here (a 2x3 cluster whose reference G is 1.6e-7 from the dense-diagonalisation
    # G) is held to 5 * accur_deflation; every other G to 1e-8.
    errs = []
    for p, lab, ei in zip(probs, labels, e):
        e_ref, sec_ref = oracle.ground_state(lab)
        assert abs(ei - e_ref) <= 1e-10 * max(1.0, abs(e_ref)), (p.name, ei, e_ref)
        assert qed.ground_state_solve(lab)[1] == sec_ref
        G1 = qed.Green_function(z, label=lab)
        G2 = oracle.green_function(lab, z)
        errs.append(np.max(np.abs(G1 - G2)))
        if qed.mixing(lab) & 4:
            G1d = qed.Green_function(z, spin_down=True, label=lab)
            G2d = oracle.green_function(lab, z, spin_down=True)
            errs[-1] = max(errs[-1], np.max(np.abs(G1d - G2d)))
    errs = np.array(errs)
    assert np.max(errs) < 5e-7, errs
    assert np.sum(errs >= 1e-8) <= 1, errs


def test_async_batch_queue(qed, oracle, fresh):
    """The asynchronous work queue: two batches (ground states of one half,
    Green functions of the other) submitted at once run on background threads
    while this thread solves the same problems with the reference; polling
    returns while they run, the results then match the reference (G of random
    clusters to 1e-8 but one instance at the deflation threshold, as in the
    blocking batched test) and the tickets are released."""
    import time
    probs = W.random_batch(10, seed=91, geoms=[(2, 2), (2, 3), (2, 4), (8, 1)])
    labels = []
    for p in probs:
        suffix, label = fresh()
        load_both(qed, oracle, p, suffix, label, fmt="F")
        labels.append(label)
    set_both(qed, oracle, GF_method="L")
    t_gs = qed.batch_submit(labels[:5], qed.QED_BATCH_GROUND_STATE, threads=3)
    t_gf = qed.batch_submit(labels[5:], qed.QED_BATCH_GREEN_FUNCTION, threads=3)
    z = W.matsubara(64)
    ref = [(oracle.ground_state(lab), oracle.green_function(lab, z)) for lab in labels]
    polls = 0
    pending = {t_gs, t_gf}
    while pending:
        for t in list(pending):
            if qed.batch_poll(t):
                pending.discard(t)
        polls += 1
        time.sleep(0.01)
    assert polls >= 1
    for t in (t_gs, t_gf):
        with pytest.raises(qed.QEDError):
            qed.batch_poll(t)
    errs = []
    for lab, ((e_ref, sec_ref), G2) in zip(labels, ref):
        e, sec = qed.ground_state_solve(lab)
        assert abs(e - e_ref) <= 1e-10 * max(1.0, abs(e_ref)) and sec == sec_ref, (lab, e, e_ref)
        errs.append(np.max(np.abs(qed.Green_function(z, label=lab) - G2)))
    errs = np.array(errs)
    assert np.max(errs) < 5e-7, errs
    assert np.sum(errs >= 1e-8) <= 1, errs


# Non-factorized formats ('S' here): sectors below max_dim_full (256) are
# diagonalised densely on both sides (Hamiltonian_Dense), which keeps every
# degenerate ground state of a sector; larger sectors run Lanczos.
DENSE_CASES = [
    # 2x2, N=3, S=1: two-fold degenerate ground state inside the sector
    ("plaq_N3_degenerate", lambda: W.hubbard_cluster(2, 2, U=4.0, mu=1.0, n_up=2, n_dn=1), None),
    ("plaq_multi", lambda: W.hubbard_cluster(2, 2, U=6.0, mu=3.0),
     "R0:N4:S0/R0:N3:S1/R0:N5:S1/R0:N3:S-1/R0:N5:S-1"),
    # ground-state sector above the threshold (Lanczos), N-1 targets below it (dense)
    ("chain8_low", lambda: W.hubbard_cluster(8, 1, U=4.0, mu=0.5, n_up=2, n_dn=2), None),
    ("neel2x3", lambda: W.hubbard_cluster(3, 2, U=5.0, mu=2.0, M=0.2, n_up=2, n_dn=2), None),
]


@pytest.mark.parametrize("case", range(len(DENSE_CASES)))
def test_dense_path_small_sectors(qed, oracle, fresh, case):
    name, mk, sectors = DENSE_CASES[case]
    prob = mk()
    if sectors:
        prob.sectors = sectors
    suffix, label = fresh()
    set_both(qed, oracle, GF_method="L")
    load_both(qed, oracle, prob, suffix, label, fmt="S")
    e1, s1 = qed.ground_state_solve(label)
    e2, s2 = oracle.ground_state(label)
    assert abs(e1 - e2) <= GS_TOL * abs(e2), (name, e1, e2)
    assert s1 == s2
    z = W.matsubara(256)
    G1 = qed.Green_function(z, label=label)
    G2 = oracle.green_function(label, z)
    assert np.max(np.abs(G1 - G2)) < GF_TOL, name
    if qed.mixing(label) & 4:
        G1d = qed.Green_function(z, spin_down=True, label=label)
        G2d = oracle.green_function(label, z, spin_down=True)
        assert np.max(np.abs(G1d - G2d)) < GF_TOL, name
    assert abs(qed.Potthoff_functional(label) - oracle.potthoff(label)) < 1e-9


def test_dense_path_keeps_degenerate_states(qed, oracle, fresh):
    """The same degenerate sector through the factorized format (one Lanczos
    state, a start-vector-dependent vector of the degenerate pair) and through
    'S' (both dense eigenstates at equal weight) gives different Green
    functions; the 'S' one matches the reference in the same format."""
    z = W.matsubara(64)
    G = {}
    for fmt in ("F", "S"):
        suffix, label = fresh()
        set_both(qed, oracle, GF_method="L")
        load_both(qed, oracle, W.hubbard_cluster(2, 2, U=4.0, mu=1.0, n_up=2, n_dn=1), suffix, label, fmt=fmt)
        G[fmt] = qed.Green_function(z, label=label)
        if fmt == "S":
            assert np.max(np.abs(G[fmt] - oracle.green_function(label, z))) < GF_TOL
    assert np.max(np.abs(G["F"] - G["S"])) > 1e-6


@pytest.mark.parametrize("case", [0, 2, 4])
def test_block_lanczos_green_function(qed, oracle, fresh, case):
    """The block form of the band-Lanczos recurrence (p vectors per H.v), forced
    on every sector with p >= 2, against the reference's band Lanczos."""
    name, mk = GS_CASES[case]
    suffix, label = fresh()
    set_both(qed, oracle, GF_method="L")
    qed.set_global_parameter("block_lanczos_min_dim", 2)
    qed.set_global_parameter("block_lanczos_min_p", 2)
    try:
        load_both(qed, oracle, mk(), suffix, label, fmt="F")
        z = W.matsubara(256)
        G1 = qed.Green_function(z, label=label)
        G1d = qed.Green_function(z, spin_down=True, label=label) if qed.mixing(label) & 4 else None
    finally:
        qed.set_global_parameter("block_lanczos_min_dim", 1000)
        qed.set_global_parameter("block_lanczos_min_p", 4)
    G2 = oracle.green_function(label, z)
    assert np.max(np.abs(G1 - G2)) < GF_TOL, name
    if G1d is not None:
        assert np.max(np.abs(G1d - oracle.green_function(label, z, spin_down=True))) < GF_TOL, name


@pytest.mark.parametrize("case", list(range(len(GS_CASES))) + [100])
def test_cluster_averages(qed, oracle, fresh, case):
    """ED::cluster_averages: ground-state average and variance of every operator
    (cluster operators divided by the number of sites, 'mu' with a minus sign)."""
    if case == 100:  # dense path, two-fold degenerate ground state
        name, mk, fmt = "plaq_N3_degenerate", lambda: W.hubbard_cluster(2, 2, U=4.0, mu=1.0, n_up=2, n_dn=1), "S"
    else:
        (name, mk), fmt = GS_CASES[case], "F"
    suffix, label = fresh()
    set_both(qed, oracle, GF_method="L")
    load_both(qed, oracle, mk(), suffix, label, fmt=fmt)
    a1 = qed.cluster_averages(label)
    oracle.ground_state(label)
    a2 = oracle.cluster_averages(label)
    assert [x[0] for x in a1] == [x[0] for x in a2], name
    for (n, v1, s1), (_, v2, s2) in zip(a1, a2):
        assert abs(v1 - v2) < 1e-9 * max(1.0, abs(v2)), (name, n, v1, v2)
        assert abs(s1 - s2) < 1e-8 * max(1.0, abs(s2)), (name, n, s1, s2)


@pytest.mark.parametrize("case", [2, 3])
def test_tr_sigma_inf_and_gf_density(qed, oracle, fresh, case):
    """ED::tr_sigma_inf (self-energy trace extrapolated from |z| ~ 1e5; the
    extrapolation amplifies round-off, hence 1e-6) and ED::Green_function_density."""
    name, mk = GS_CASES[case]
    suffix, label = fresh()
    set_both(qed, oracle, GF_method="L")
    load_both(qed, oracle, mk(), suffix, label, fmt="F")
    qed.Green_function_solve(label)
    oracle.green_solve(label)
    assert abs(qed.Green_function_density(label) - oracle.gf_density(label)) < 1e-8, name
    s1, s2 = qed.tr_sigma_inf(label), oracle.tr_sigma_inf(label)
    assert abs(s1 - s2) < 1e-6 * max(1.0, abs(s2)), (name, s1, s2)


@pytest.mark.parametrize("case,op", [(2, "M"), (2, "t"), (0, "U"), (3, "mu")])
def test_susceptibility(qed, oracle, fresh, case, op):
    """ED::susceptibility and susceptibility_poles (Lehmann representation of
    O|psi> by band Lanczos with one start vector). With a single start vector the
    recurrence stops as soon as its lowest Ritz value (the ground state itself)
    changes by less than 1e-12 between steps, a test that round-off can pass one
    step earlier or later in either code, which moves the unconverged high
    poles: the tolerance is 1e-5 here instead of the 1e-8 of the Green functions,
    and 1e-4 on the poles of residue above 0.05 (the reference's own small poles
    for chain8 / U move by 2e-5 when only its random seed changes; those of
    plaq8b / mu with residue 0.03 by 1e-3 between the two codes)."""
    name, mk = GS_CASES[case]
    suffix, label = fresh()
    set_both(qed, oracle, GF_method="L")
    load_both(qed, oracle, mk(), suffix, label, fmt="F")
    w = np.array([0.3 + 0.05j, 1.0 + 0.1j, 2.5 + 0.2j, 1j, 6.0 + 0.5j])
    c1 = qed.susceptibility(op, w, label=label)
    oracle.ground_state(label)
    c2 = oracle.susceptibility(label, op, w)
    scale = max(1.0, np.max(np.abs(c2)))
    # frequencies at or below the converged part of the spectrum: 1e-5
    assert np.max(np.abs(c1[:4] - c2[:4])) < 1e-5 * scale, (name, op)
    # 6 + 0.5i sits among the unconverged high poles, which move with the step
    # at which the Ritz test stops (observed: 1.3e-3 for plaq8b / mu on B200)
    assert abs(c1[4] - c2[4]) < 5e-3 * max(1.0, abs(c2[4])), (name, op, c1[4], c2[4])
    p1 = qed.susceptibility_poles(op, label=label)
    p2 = oracle.susceptibility_poles(label, op)
    big1 = [x for x in p1 if x[1] > 0.05]
    big2 = [x for x in p2 if x[1] > 0.05]
    assert len(big1) == len(big2), (name, op)
    for (e1, r1), (e2, r2) in zip(sorted(big1), sorted(big2)):
        assert abs(e1 - e2) < 1e-4 and abs(r1 - r2) < 1e-4 * max(1.0, r2), (name, op, e1, e2, r1, r2)


def test_fidelity(qed, oracle, fresh):
    """ED::fidelity between two instances of one model at nearby parameters: the
    overlap of ground states does not depend on their signs or normalisation
    conventions beyond those of the reference (both Lanczos vectors, weight 1)."""
    mk = lambda U: W.hubbard_cluster(4, 2, U=U, mu=1.7, M=0.25, name="fid")
    labels = []
    for U in (5.0, 5.3):
        suffix, label = fresh()
        load_both(qed, oracle, mk(U), "_fid" + suffix, label, fmt="F")
        labels.append(label)
    f1 = qed.fidelity(*labels)
    f2 = oracle.fidelity(*labels)
    assert abs(f1 - f2) < 1e-9, (f1, f2)
    assert abs(qed.fidelity(labels[0], labels[0]) - oracle.fidelity(labels[0], labels[0])) < 1e-9


def _uncorrelated(p):
    p.operators.pop("U")
    p.params.pop("U")
    return p


UNCORRELATED = [
    ("free2x3_neel", lambda: _uncorrelated(W.hubbard_cluster(3, 2, U=4.0, mu=0.7, M=0.2, name="free23"))),
    ("free_chain6", lambda: _uncorrelated(W.hubbard_cluster(6, 1, U=4.0, mu=0.4, name="free6"))),
    ("free_plaq8b", lambda: _uncorrelated(W.plaquette_bath(np.linspace(-1.5, 1.5, 8), np.linspace(0.2, 0.9, 8),
                                                           name="freepb"))),
]


@pytest.mark.parametrize("case", range(len(UNCORRELATED)))
def test_uncorrelated_one_body_path(qed, oracle, fresh, case):
    """Instances without an interaction operator: one_body_solve (ground-state
    energy from the occupied one-body levels, the Q-matrix of the one-body
    problem, averages from <c+ c>)."""
    name, mk = UNCORRELATED[case]
    suffix, label = fresh()
    set_both(qed, oracle, GF_method="L")
    load_both(qed, oracle, mk(), suffix, label, fmt="F")
    e1, s1 = qed.ground_state_solve(label)
    e2, s2 = oracle.ground_state(label)
    assert s1 == s2 == "uncorrelated"
    assert abs(e1 - e2) <= 1e-12 * max(1.0, abs(e2)), (name, e1, e2)
    z = W.matsubara(64)
    assert np.max(np.abs(qed.Green_function(z, label=label) - oracle.green_function(label, z))) < 1e-12
    if qed.mixing(label) & 4:
        assert np.max(np.abs(qed.Green_function(z, spin_down=True, label=label)
                             - oracle.green_function(label, z, spin_down=True))) < 1e-12
    assert abs(qed.Potthoff_functional(label) - oracle.potthoff(label)) < 1e-12
    assert np.max(np.abs(qed.Green_function_average(label=label) - oracle.green_function_average(label))) < 1e-12
    a1, a2 = qed.cluster_averages(label), oracle.cluster_averages(label)
    assert [x[0] for x in a1] == [x[0] for x in a2]
    for (n, v1, s1_), (_, v2, s2_) in zip(a1, a2):
        assert abs(v1 - v2) < 1e-12, (name, n, v1, v2)
        assert np.isnan(s1_) and np.isnan(s2_)
