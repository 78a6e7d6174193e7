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
