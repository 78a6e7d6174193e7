"""CPU tests of the cluster point group (pyqcm_b200/csrc/symmetry.*) against the
reference's own symmetry_group and ED_mixed_basis (compiled in the oracle): group
order, character phases, symmetric orbitals, orbit representatives with phases and
lengths, the representative basis of a sector, and the reference's error messages
for bad generators. Host logic only: nothing here touches a GPU."""
from math import comb

import numpy as np
import pytest

from tests.helpers import c2v_golden

# (n_sites, n_bath, generators in pyqcm's 1-based form, bath_irrep)
GROUPS = {
    "c2v_8b_record": None,  # filled from the reference's record
    "chain6_mirror": (6, 0, [[6, 5, 4, 3, 2, 1]], False),
    "plaquette_c4": (4, 0, [[2, 4, 1, 3]], False),
    "ring3_c3": (3, 0, [[2, 3, 1]], False),
    "sq2x3_c2v": (6, 0, [[3, 2, 1, 6, 5, 4], [4, 5, 6, 1, 2, 3]], False),
    "dimer_bath_swap": (2, 2, [[2, 1, 4, 3]], False),
    "chain4_bath_irrep": (4, 2, [[4, 3, 2, 1, 0, 1]], True),
}


def _group(name):
    if name == "c2v_8b_record":
        m = c2v_golden()["model"]
        return m["n_sites"], m["n_bath"], m["generators"], m["bath_irrep"]
    return GROUPS[name]


def _sector_states(n_orb, n_up, n_dn):
    def strings(n):
        return [b for b in range(1 << n_orb) if bin(b).count("1") == n]
    up = np.array(strings(n_up), dtype=np.uint64)
    dn = np.array(strings(n_dn), dtype=np.uint64)
    return (up[None, :] | (dn[:, None] << np.uint64(32))).reshape(-1)  # sorted: dn major, up minor


@pytest.mark.parametrize("name", list(GROUPS))
def test_group_tables_match_the_reference(oracle, name):
    import pyqcm_b200 as qed
    ns, nb, gens, bi = _group(name)
    mine = qed.symmetry_group(ns, nb, gens, bi)
    ref = oracle.symmetry_group(ns, nb, gens, bi)
    assert mine["g"] == ref["g"]
    assert np.array_equal(mine["phi"], ref["phi"])
    assert np.array_equal(mine["site_irrep_dim"], ref["site_irrep_dim"])
    assert np.max(np.abs(mine["S"] - ref["S"])) < 1e-14


@pytest.mark.parametrize("name", list(GROUPS))
def test_representatives_match_the_reference(oracle, name):
    import pyqcm_b200 as qed
    ns, nb, gens, bi = _group(name)
    n_orb = ns + nb
    g = qed.symmetry_group(ns, nb, gens, bi)["g"]
    n_up, n_dn = n_orb // 2, (n_orb + 1) // 2
    states = _sector_states(n_orb, n_up, n_dn)
    if len(states) > 200000:
        states = np.random.default_rng(7).choice(states, 200000, replace=False)
    for r in range(g):
        rep, ph, ln = qed.symmetry_representatives(ns, nb, gens, bi, r, states)
        rrep, rph, rln = oracle.representatives(ns, nb, gens, bi, r, states)
        assert np.array_equal(ln, rln), (name, r)
        live = ln > 0
        assert np.array_equal(rep[live], rrep[live]), (name, r)
        assert np.array_equal(ph[live], rph[live]), (name, r)


@pytest.mark.parametrize("name,sector", [("c2v_8b_record", "R0:N12:S0"), ("c2v_8b_record", "R3:N11:S1"),
                                         ("sq2x3_c2v", "R2:N6:S0"), ("plaquette_c4", "R1:N4:S0"),
                                         ("ring3_c3", "R2:N3:S1"), ("chain4_bath_irrep", "R1:N6:S0")])
def test_representative_basis_matches_the_reference(oracle, name, sector):
    """The symmetry-adapted basis of a sector: every state of the (N_up, N_dn)
    sector that is its orbit's representative with a nonzero projection, in
    ascending order (ED_mixed_basis, src_ed/ED_basis.cpp:185-385). Enumerating the
    factorized sector in its own order (down string major) gives them sorted."""
    import pyqcm_b200 as qed
    ns, nb, gens, bi = _group(name)
    n_orb = ns + nb
    r, N, S = (int(t[1:]) for t in sector.split(":"))
    states = _sector_states(n_orb, (N + S) // 2, (N - S) // 2)
    rep, _, ln = qed.symmetry_representatives(ns, nb, gens, bi, r, states)
    mine = states[(ln > 0) & (rep == states)]
    ref = oracle.mixed_basis(ns, nb, gens, bi, sector)
    assert np.array_equal(mine, ref)


@pytest.mark.parametrize("name,N,S", [("c2v_8b_record", 12, 0), ("sq2x3_c2v", 5, 1), ("chain6_mirror", 6, 0)])
def test_irrep_bases_partition_the_sector(name, N, S):
    """For real characters the irrep bases together span the sector: their
    dimensions add up to the factorized dimension C(n, N_up) C(n, N_dn)."""
    import pyqcm_b200 as qed
    ns, nb, gens, bi = _group(name)
    n_orb = ns + nb
    g = qed.symmetry_group(ns, nb, gens, bi)["g"]
    states = _sector_states(n_orb, (N + S) // 2, (N - S) // 2)
    total = 0
    for r in range(g):
        rep, _, ln = qed.symmetry_representatives(ns, nb, gens, bi, r, states)
        total += int(np.count_nonzero((ln > 0) & (rep == states)))
    assert total == comb(n_orb, (N + S) // 2) * comb(n_orb, (N - S) // 2)


@pytest.mark.parametrize("gens,msg", [([[2, 1, 3], [1, 3, 2]], "do not commute"),
                                      ([[1, 1, 3]], "is not valid"),
                                      ([[2, 1, 3]] * 5, "exceeds the limit")])
def test_bad_generators_raise_the_reference_messages(oracle, gens, msg):
    import pyqcm_b200 as qed
    with pytest.raises(qed.QEDError, match=msg):
        qed.symmetry_group(3, 0, gens, False)
    with pytest.raises(oracle.OracleError, match=msg):
        oracle.symmetry_group(3, 0, gens, False)


def _port_gens(gens, n_sites, bath_irrep):
    return [[v - 1 if (i < n_sites or not bath_irrep) else v for i, v in enumerate(g)] for g in gens]


@pytest.mark.parametrize("name", ["c2v_8b_record", "plaquette_c4", "chain4_bath_irrep", "dimer_bath_swap"])
def test_symmetry_port_matches_the_reference(oracle, name):
    """The numpy restatement (oracle/port_sym.py) of the group and of the
    representative map against the compiled reference."""
    from oracle import port_sym
    ns, nb, gens, bi = _group(name)
    G = port_sym.group(ns, nb, _port_gens(gens, ns, bi), bi)
    ref = oracle.symmetry_group(ns, nb, gens, bi)
    assert G["g"] == ref["g"] and np.array_equal(G["phi"], ref["phi"])
    n_orb = ns + nb
    states = _sector_states(n_orb, n_orb // 2, (n_orb + 1) // 2)
    states = np.random.default_rng(3).choice(states, min(len(states), 3000), replace=False)
    for r in range(G["g"]):
        rrep, rph, rln = oracle.representatives(ns, nb, gens, bi, r, states)
        for b, a, p, n in zip(states, rrep, rph, rln):
            rep, ph, ln = port_sym.representative(G, int(b), r)
            assert ln == n and (n == 0 or (rep == a and ph == p))


@pytest.mark.parametrize("case,sectors", [
    ("sq2x3_c2v_hubbard", ["R0:N6:S0", "R1:N6:S0", "R3:N5:S1"]),
    ("c2v_8b_record", ["R0:N3:S1", "R2:N3:S1"]),
])
def test_mixed_basis_hamiltonian_port_matches_reference_csr(oracle, fresh, case, sectors):
    """H x in the symmetry-adapted basis: the numpy restatement (one-body elements
    reaching orbit representatives with sign, character phase and
    sqrt(len_I / len_J)) against the reference's own CSR Hamiltonian, to 1e-13."""
    from oracle import port_sym
    from pyqcm_b200 import workloads as W
    from tests.helpers import c2v_golden, c2v_problem
    if case == "c2v_8b_record":
        prob = c2v_problem(c2v_golden(), True)
    else:
        prob = W.hubbard_cluster(3, 2, tp=0.3, U=6.0, mu=2.5)
        prob.generators = [[3, 2, 1, 6, 5, 4], [4, 5, 6, 1, 2, 3]]
    suffix, label = fresh()
    oracle.load_problem(prob, label, model_name="sym" + suffix, fmt="S")
    G = port_sym.group(prob.n_sites, prob.n_bath, _port_gens(prob.generators, prob.n_sites, prob.bath_irrep),
                       prob.bath_irrep)
    for sec in sectors:
        H, basis = port_sym.mixed_hamiltonian(prob, G, sec)
        R = oracle.RefHamiltonian(label, sec, csr=True)
        assert R.dim == H.shape[0]
        x = np.random.default_rng(11).standard_normal(R.dim)
        y = np.zeros(R.dim)
        R.mult_add(x, y)
        assert np.max(np.abs(y - H @ x)) <= 1e-13 * max(1.0, np.max(np.abs(y))), sec


def test_irrep_green_functions_port_matches_reference(oracle, fresh):
    """Per-irrep Green functions in the symmetry-adapted basis (numpy restatement:
    destruction operators of symmetric orbitals between irrep bases, target irreps
    by the irrep product, dense Lehmann sums) against the compiled reference's
    site-basis Green function projected on each symmetric orbital, 2x3 cluster with
    C2v generators, ground state in its lowest irrep: to 1e-10."""
    from oracle import port_sym
    from pyqcm_b200 import workloads as W
    prob = W.hubbard_cluster(3, 2, tp=0.3, U=6.0, mu=2.5)
    prob.generators = [[3, 2, 1, 6, 5, 4], [4, 5, 6, 1, 2, 3]]
    G = port_sym.group(6, 0, [[v - 1 for v in g] for g in prob.generators], False)
    lows = [np.linalg.eigvalsh(port_sym.mixed_hamiltonian(prob, G, f"R{r}:N6:S0")[0].toarray())[0] for r in range(4)]
    prob.sectors = f"R{int(np.argmin(lows))}:N6:S0"
    suffix, label = fresh()
    oracle.set_param("GF_method", "L")
    oracle.load_problem(prob, label, model_name="irrgf" + suffix, fmt="S")
    e_ref, _ = oracle.ground_state(label)
    z = np.array([0.3j, 1j, 2.5j, -1 + 0.4j])
    Gs = oracle.green_function(label, z)
    rows, irreps = port_sym.symmetric_orbitals(G, 6)
    assert np.max(np.abs(rows - oracle.symmetry_group(6, 0, prob.generators, False)["S"].real)) < 1e-14
    for row, rho in zip(rows, irreps):
        gp, e0 = port_sym.irrep_green_function(prob, G, prob.sectors, row, rho, z)
        assert abs(e0 - e_ref) < 1e-10
        assert np.max(np.abs(gp - np.einsum("a,zab,b->z", row, Gs, row))) < 1e-10


def test_trivial_group_and_model_generators_errors(oracle):
    """No generators: the trivial group (g = 1, one orbital per site in irrep 0), as
    the reference builds it. A model created with invalid generators fails with the
    reference's message, through ED::new_model on both sides."""
    import pyqcm_b200 as qed
    mine = qed.symmetry_group(3, 1, None, False)
    ref = oracle.symmetry_group(3, 1, None, False)
    assert mine["g"] == ref["g"] == 1
    assert np.array_equal(mine["site_irrep_dim"], ref["site_irrep_dim"])
    assert np.max(np.abs(mine["S"] - ref["S"])) < 1e-15
    with pytest.raises(qed.QEDError, match="is not valid"):
        qed.new_model("badgen_host", 3, 0, [[1, 1, 2]], False)
    with pytest.raises(oracle.OracleError, match="is not valid"):
        oracle.new_model("badgen_host", 3, 0, [[1, 1, 2]], False)
