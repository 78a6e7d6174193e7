"""CPU tests of the C ABI boundary: the library loads, exports every symbol the
header declares, and its host-side model logic mirrors the reference's error
behaviour. No kernel is launched here."""
import ctypes
import os
import re

import numpy as np
import pytest

from pyqcm_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "qed_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(qed_[a-zA-Z_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(qed):
    L = ctypes.CDLL(qed.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 30
    missing = [s for s in syms if not hasattr(L, s)]
    assert not missing, missing


def test_model_and_instance_host_logic(qed, fresh):
    suffix, label = fresh()
    prob = W.chain8()
    qed.load_problem(prob, label, model_name="cpu" + suffix)
    assert qed.Green_function_dimension(label) == 8
    assert qed.mixing(label) == 0
    # staggered field makes the two spins different (mixing up_down = 4)
    suffix, label = fresh()
    qed.load_problem(W.hubbard_cluster(4, 2, U=4.0, M=0.1), label, model_name="cpu" + suffix)
    assert qed.mixing(label) == 4


def test_errors_follow_reference_conventions(qed, fresh):
    suffix, label = fresh()
    with pytest.raises(qed.QEDError) as e:
        qed.new_model_instance("no_such_model" + suffix, {"t": 1.0}, "R0:N2:S0", label)
    assert e.value.code == 1 and "not defined" in str(e.value)
    qed.new_model("m" + suffix, 4, 0)
    qed.new_operator("m" + suffix, "t", "one-body", [(0, 1, 1.0), (4, 5, 1.0)])
    qed.new_operator("m" + suffix, "U", "interaction", [(i, i + 4, 1.0) for i in range(4)])
    with pytest.raises(qed.QEDError) as e:
        qed.new_model_instance("m" + suffix, {"t": -1.0, "U": 2.0}, "R0:N3:S0", label)
    assert "not valid" in str(e.value)
    # a spin-flip one-body term leaves the spin-factorized solver's scope
    qed.new_model("sf" + suffix, 4, 0)
    qed.new_operator("sf" + suffix, "t", "one-body", [(0, 1, 1.0), (4, 5, 1.0)])
    qed.new_operator("sf" + suffix, "sf", "one-body", [(0, 5, 1.0)])
    with pytest.raises(qed.QEDError) as e:
        qed.new_model_instance("sf" + suffix, {"t": -1.0, "sf": 0.5}, "R0:N4:S0", label + 1)
    assert e.value.code == 6
    with pytest.raises(qed.QEDError) as e:
        qed.new_operator("m" + suffix, "an", "anomalous", [(0, 5, 1.0)])
    assert e.value.code == 6
    with pytest.raises(qed.QEDError):
        qed.set_global_parameter("no_such_option", 1.0)
    with pytest.raises(qed.QEDError) as e:
        qed.ground_state_solve(987654)
    assert e.value.code == 1


def test_matrix_continued_fraction_options(qed, fresh):
    """GF_method 'M' (matrix continued fractions from block Lanczos) is
    accepted; combining the electron and hole fractions (combine_mcf, with 'M'
    or 'L') is refused with the unsupported status when the instance is made,
    as is 'M' for a model with generators once it is solved."""
    suffix, label = fresh()
    qed.new_model("mcf" + suffix, 4, 0)
    qed.new_operator("mcf" + suffix, "t", "one-body", [(0, 1, 1.0), (4, 5, 1.0)])
    qed.new_operator("mcf" + suffix, "U", "interaction", [(i, i + 4, 1.0) for i in range(4)])
    try:
        qed.set_global_parameter("GF_method", "M")
        qed.new_model_instance("mcf" + suffix, {"t": -1.0, "U": 2.0}, "R0:N4:S0", label)
        qed.set_global_parameter("combine_mcf", True)
        for gf in ("M", "L"):
            qed.set_global_parameter("GF_method", gf)
            with pytest.raises(qed.QEDError) as e:
                qed.new_model_instance("mcf" + suffix, {"t": -1.0, "U": 2.0}, "R0:N4:S0", label + 1)
            assert e.value.code == qed.QED_ERR_UNSUPPORTED and "combine_mcf" in str(e.value)
    finally:
        qed.set_global_parameter("combine_mcf", False)
        qed.set_global_parameter("GF_method", "L")
    from tests.helpers import c2v_golden, c2v_problem
    prob = c2v_problem(c2v_golden(), True)
    qed.set_global_parameter("GF_method", "M")
    try:
        qed.load_problem(prob, label + 2, model_name="c2v_mcf" + suffix)
        with pytest.raises(qed.QEDError) as e:
            qed.ground_state_solve(label + 2)
        assert e.value.code == qed.QED_ERR_UNSUPPORTED and "'M'" in str(e.value)
    finally:
        qed.set_global_parameter("GF_method", "L")


def test_async_batch_queue_host_logic(qed, fresh):
    """qed_batch_submit / poll / wait: unknown labels and a bad kind fail at
    submission, unknown tickets at poll; a submitted batch finishes (here, with
    no device, with the no-device status, which the wait returns once and then
    releases the ticket)."""
    suffix, label = fresh()
    with pytest.raises(qed.QEDError) as e:
        qed.batch_submit([987655], qed.QED_BATCH_GROUND_STATE)
    assert e.value.code == qed.QED_ERR_ARGUMENT
    qed.new_model("ab" + suffix, 4, 0)
    qed.new_operator("ab" + suffix, "t", "one-body", [(0, 1, 1.0), (4, 5, 1.0), (1, 2, 1.0), (5, 6, 1.0)])
    qed.new_operator("ab" + suffix, "U", "interaction", [(i, i + 4, 1.0) for i in range(4)])
    qed.new_model_instance("ab" + suffix, {"t": -1.0, "U": 2.0}, "R0:N4:S0", label)
    with pytest.raises(qed.QEDError) as e:
        qed.batch_submit([label], 7)
    assert e.value.code == qed.QED_ERR_ARGUMENT
    t = qed.batch_submit([label], qed.QED_BATCH_GREEN_FUNCTION, threads=2)
    assert t > 0
    try:
        assert qed.batch_wait(t, timeout=600)
    except qed.QEDError as err:  # no GPU here: the batch's own status comes back
        assert err.code == qed.QED_ERR_NO_DEVICE, err
    with pytest.raises(qed.QEDError) as e:
        qed.batch_poll(t)
    assert e.value.code == qed.QED_ERR_ARGUMENT


def test_unknown_label_and_options(qed):
    qed.set_global_parameter("accur_lanczos", 1e-12)
    assert qed.get_global_double("accur_lanczos") == 1e-12
    qed.set_global_parameter("kgrid_side", 32)  # lattice-layer option is accepted


def test_models_with_generators_load_and_refuse_what_is_not_covered():
    """A cluster model with symmetry generators (g > 1) loads with its group
    (sector strings may name irreps below g) and is solved in the
    symmetry-adapted basis; what that path does not cover is refused with the
    unsupported status before any device work: continued-fraction Green
    functions (GF_method 'F') and, below, groups with complex characters."""
    import pyqcm_b200 as qed
    from tests.helpers import c2v_golden, c2v_problem
    prob = c2v_problem(c2v_golden(), True)
    qed.set_global_parameter("GF_method", "F")
    try:
        qed.load_problem(prob, 4101, model_name="c2v_host")
        for fn in (qed.ground_state_solve, qed.Green_function_solve):
            with pytest.raises(qed.QEDError) as err:
                fn(4101)
            assert err.value.code == qed.QED_ERR_UNSUPPORTED
            assert "continued-fraction" in str(err.value)
    finally:
        qed.set_global_parameter("GF_method", "L")
    qed.new_model_instance("c2v_host", prob.params, "R3:N11:S1", 4102)
    with pytest.raises(qed.QEDError, match="not valid"):
        qed.new_model_instance("c2v_host", prob.params, "R4:N12:S0", 4103)


def test_complex_character_groups_are_refused_by_the_mixed_hamiltonian():
    """A generator of order 4 (C4 on a plaquette) gives the group complex
    characters, for which the reference switches to a complex Hilbert space; the
    real symmetry-adapted Hamiltonian refuses such models with the unsupported
    status (before any device work) instead of returning real-phase products."""
    import pyqcm_b200 as qed
    qed.new_model("c4_plaquette_host", 4, 0, [[2, 4, 1, 3]])
    hop = [(0, 1, -1.0), (1, 3, -1.0), (3, 2, -1.0), (0, 2, -1.0)]
    hop += [(a + 4, b + 4, v) for a, b, v in hop]
    qed.new_operator("c4_plaquette_host", "t", "one-body", hop)
    qed.new_operator("c4_plaquette_host", "U", "interaction", [(i, i + 4, 1.0) for i in range(4)])
    qed.new_model_instance("c4_plaquette_host", {"t": 1.0, "U": 4.0}, "R1:N4:S0", 4201)
    with pytest.raises(qed.QEDError) as err:
        qed.MixedHamiltonian(4201, "R1:N4:S0")
    assert err.value.code == qed.QED_ERR_UNSUPPORTED
    assert "complex" in str(err.value)
    with pytest.raises(qed.QEDError) as err:
        qed.ground_state_solve(4201)
    assert err.value.code == qed.QED_ERR_UNSUPPORTED
    assert "complex" in str(err.value)
