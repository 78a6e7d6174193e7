"""CPU tests of the oracle itself: the numpy restatement (oracle/port.py) against
the compiled reference (oracle/ref.py), analytic known answers, and the
committed golden fixtures (tests/golden/, made by tests/golden/make_golden.py
from the reference)."""
import math
import os

import numpy as np
import pytest

from oracle import port
from pyqcm_b200 import workloads as W
from tests.helpers import rel_err

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("L,N", [(4, 2), (8, 4), (10, 3), (12, 6)])
def test_halfbasis_port_vs_reference(oracle, L, N):
    assert np.array_equal(port.halfbasis(L, N), oracle.halfbasis(L, N))
    B = port.halfbasis(L, N)
    assert [port.rank(int(b)) for b in B] == list(range(len(B)))


@pytest.mark.parametrize("L,nu,nd,a", [(5, 2, 3, 1), (5, 2, 3, 8), (6, 3, 3, 0), (6, 3, 3, 11)])
def test_destroy_signs_port_vs_reference(oracle, L, nu, nd, a):
    tgt, ph = oracle.destroy_table(L, nu, nd, a)
    spin, orb = (1, a - L) if a >= L else (0, a)
    psi = np.arange(1, len(tgt) + 1, dtype=float)
    y = port.cdag(psi, L, nu, nd, -1, spin, orb)
    for I in range(len(tgt)):
        if tgt[I] >= 0:
            assert y[tgt[I]] == (-1) ** (ph[I] % 2) * psi[I]
    assert np.count_nonzero(y) == np.count_nonzero(tgt >= 0)


SMALL = [
    ("chain6", lambda: W.hubbard_cluster(6, 1, U=4.0)),
    ("sq2x3_tp", lambda: W.hubbard_cluster(3, 2, tp=0.3, U=6.0)),
    ("neel2x3", lambda: W.hubbard_cluster(3, 2, U=5.0, mu=1.7, M=0.25)),
    ("dimer4b", lambda: _dimer_bath()),
]


def _dimer_bath():
    p = W.ClusterProblem("dimer4b", 2, 4)
    L = 6
    both = lambda el: el + [(r + L, c + L, v) for (r, c, v) in el]
    p.operators["t"] = ("one-body", both([(0, 1, 1.0)]))
    p.operators["U"] = ("interaction", [(0, L, 1.0), (1, 1 + L, 1.0)])
    p.operators["mu"] = ("one-body", both([(0, 0, -1.0), (1, 1, -1.0)]))
    p.params = {"t": -1.0, "U": 4.0, "mu": 2.0}
    for b in range(4):
        p.operators[f"e{b}"] = ("one-body", both([(2 + b, 2 + b, 1.0)]))
        p.operators[f"v{b}"] = ("one-body", both([(b // 2, 2 + b, 1.0)]))
        p.params[f"e{b}"] = [-1.0, 1.0, -0.5, 0.5][b]
        p.params[f"v{b}"] = [0.5, 0.4, 0.3, 0.6][b]
    p.sectors = "R0:N6:S0"
    return p


@pytest.mark.parametrize("case", range(len(SMALL)))
def test_hv_port_vs_reference(oracle, fresh, case):
    name, mk = SMALL[case]
    prob = mk()
    suffix, label = fresh()
    oracle.load_problem(prob, label, model_name=name + suffix, fmt="F")
    N, S = port.parse_sector(prob.sectors)
    nu, nd = (N + S) // 2, (N - S) // 2
    H, _, _ = port.sector_hamiltonian(prob, nu, nd)
    Hr = oracle.RefHamiltonian(label, prob.sectors)
    x = np.random.default_rng(case).standard_normal(H.shape[0])
    y = np.zeros(H.shape[0])
    Hr.mult_add(x, y)
    assert rel_err(H @ x, y) < 1e-13


@pytest.mark.parametrize("case", range(len(SMALL)))
@pytest.mark.parametrize("method", ["L", "F"])
def test_solve_port_vs_reference(oracle, fresh, case, method):
    name, mk = SMALL[case]
    prob = mk()
    suffix, label = fresh()
    oracle.set_param("GF_method", method)
    try:
        oracle.load_problem(prob, label, model_name=name + suffix, fmt="F" if method == "L" else "S")
        e_ref, _ = oracle.ground_state(label)
        z = W.matsubara(64)
        G_ref = oracle.green_function(label, z)
    finally:
        oracle.set_param("GF_method", "L")
    sol = port.solve(prob, gf_method=method)
    assert abs(sol["E0"] - e_ref) <= 1e-10 * abs(e_ref)
    G = port.green_function(sol, z)
    assert np.max(np.abs(G - G_ref)) < 1e-8


def test_two_site_hubbard_closed_form(oracle, fresh):
    """Half-filled Hubbard dimer: E0 = U/2 - sqrt((U/2)^2 + 4 t^2) at mu = 0."""
    t, U = -1.0, 3.0
    p = W.hubbard_cluster(2, 1, t=t, U=U, mu=0.0)
    suffix, label = fresh()
    oracle.load_problem(p, label, model_name="dimer" + suffix, fmt="F")
    e, _ = oracle.ground_state(label)
    exact = U / 2 - math.sqrt((U / 2) ** 2 + 4 * t * t)
    assert abs(e - exact) < 1e-12
    assert abs(port.solve(p)["E0"] - exact) < 1e-12


def test_noninteracting_limit_resolvent(oracle, fresh):
    """U -> 0: the cluster G(z) is the one-body resolvent (z - t)^-1."""
    p = W.hubbard_cluster(6, 1, t=-1.0, U=1e-9, mu=0.0)
    suffix, label = fresh()
    oracle.load_problem(p, label, model_name="free" + suffix, fmt="F")
    z = W.matsubara(32)
    G = oracle.green_function(label, z)
    T = np.zeros((6, 6))
    for i in range(5):
        T[i, i + 1] = T[i + 1, i] = -1.0
    exact = np.array([np.linalg.inv(w * np.eye(6) - T) for w in z])
    assert np.max(np.abs(G - exact)) < 1e-8


def test_golden_fixtures_reproduce(oracle, fresh):
    """The committed fixtures were made by the reference; re-running it here
    (or on the GPU box, where the prebuilt oracle travels) must give them back."""
    path = os.path.join(GOLDEN, "small_cases.npz")
    if not os.path.exists(path):
        pytest.skip("fixtures not generated")
    g = np.load(path, allow_pickle=False)
    names = [str(n) for n in g["names"]]
    for i, name in enumerate(names):
        if not name.startswith(("chain8", "sq2x3")):
            continue
        prob = W.chain8() if name.startswith("chain8") else W.hubbard_cluster(3, 2, tp=0.3, U=6.0)
        method = "F" if name.endswith("_F") else "L"
        suffix, label = fresh()
        oracle.set_param("GF_method", method)
        try:
            oracle.load_problem(prob, label, model_name=name + suffix, fmt="S" if method == "F" else "F")
            e, _ = oracle.ground_state(label)
            G = oracle.green_function(label, W.matsubara(256))
        finally:
            oracle.set_param("GF_method", "L")
        n = int(g["dims"][i])
        assert abs(e - g["E0"][i]) <= 1e-10 * abs(e)
        assert np.max(np.abs(G - g["G"][i][:, :n, :n])) < 1e-8


def test_c2v_record_pins_the_oracle(oracle, fresh):
    """The reference's own diagonalization record (tests/test_diagonalization/
    S_format.ref: 2x2 plaquette + 8 bath orbitals with C2v generators, solved in the
    symmetry-adapted basis, CSR format): the compiled oracle reproduces its ground-state
    energy (6 significant digits in the record) and each irrep's Green function built
    from the record's 14-digit poles, at off-axis frequencies, to 1e-7."""
    from tests.helpers import C2V_Z, c2v_golden, c2v_irrep_gf, c2v_problem, project_irreps
    gold = c2v_golden()
    suffix, label = fresh()
    oracle.set_param("GF_method", "L")
    oracle.load_problem(c2v_problem(gold, True), label, model_name="c2v" + suffix, fmt="S")
    E, sec = oracle.ground_state(label)
    assert abs(E - gold["gs"]["energy"]) < 5.1e-5, E
    assert sec == gold["gs"]["sector"]
    G = oracle.green_function(label, C2V_Z)
    assert np.max(np.abs(project_irreps(G) - c2v_irrep_gf(gold, C2V_Z))) < 1e-7
