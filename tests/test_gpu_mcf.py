"""Matrix continued fractions (GF_method 'M'): block Lanczos on the start block
c_i^{-+}|GS> of every cluster site, then G(z) = W^T F_0(z) W from the floors,
against the reference's own build_mcf (src_ed/model_instance.hpp:847-946) run
by the compiled oracle on the same problem, for both forms of the off-diagonal
blocks (block_Lanczos_QR false: polar factor, the default; true: QR).

Tolerances: G(i w_n) within 1e-8 absolute on 64 Matsubara frequencies (beta =
50), as the Lehmann and scalar continued-fraction paths; the integrated Green
function (W_h^T W_h, from the start block's QR only) within 1e-10; and the same
G within 1e-8 of this solver's own Lehmann (band-Lanczos Q-matrix) G.
"""
import numpy as np
import pytest

from pyqcm_b200 import workloads as W
from tests.helpers import load_both, set_both

pytestmark = pytest.mark.gpu

CASES = [
    ("chain8", lambda: W.chain8()),
    ("sq2x3_tp", lambda: W.hubbard_cluster(3, 2, tp=0.3, U=6.0)),
    ("neel2x4", lambda: W.hubbard_cluster(4, 2, U=5.0, mu=1.7, M=0.25)),
    ("plaq8b", lambda: W.plaquette_bath(np.linspace(-1.5, 1.5, 8), np.linspace(0.2, 0.9, 8))),
]


def _both(qed, oracle, qr):
    set_both(qed, oracle, GF_method="M")
    qed.set_global_parameter("block_Lanczos_QR", qr)
    oracle.set_param("block_Lanczos_QR", qr)


def _reset(qed, oracle):
    set_both(qed, oracle, GF_method="L")
    qed.set_global_parameter("block_Lanczos_QR", False)
    oracle.set_param("block_Lanczos_QR", False)


@pytest.mark.parametrize("qr", [False, True])
@pytest.mark.parametrize("case", range(len(CASES)))
def test_mcf_green_function_matches_reference(qed, oracle, fresh, case, qr):
    name, mk = CASES[case]
    suffix, label = fresh()
    z = W.matsubara(64)
    try:
        _both(qed, oracle, qr)
        load_both(qed, oracle, mk(), suffix, label, fmt="F")
        G1 = qed.Green_function(z, label=label)
        G2 = oracle.green_function(label, z)
        M1 = qed.Green_function_average(label=label)
        M2 = oracle.green_function_average(label)
        spin_down = bool(qed.mixing(label) & 4)
        if spin_down:
            G1d = qed.Green_function(z, spin_down=True, label=label)
            G2d = oracle.green_function(label, z, spin_down=True)
    finally:
        _reset(qed, oracle)
    assert np.max(np.abs(G1 - G2)) < 1e-8, (name, np.max(np.abs(G1 - G2)))
    assert np.max(np.abs(M1 - M2)) < 1e-10, name
    if spin_down:
        assert np.max(np.abs(G1d - G2d)) < 1e-8, name
    # the same G from this solver's Lehmann path
    suffix2, label2 = fresh()
    qed.load_problem(mk(), label2, model_name=name + "_L" + suffix2, fmt="F")
    GL = qed.Green_function(z, label=label2)
    assert np.max(np.abs(G1 - GL)) < 1e-8, name


def test_mcf_on_a_sector_of_the_staged_kernels(qed, fresh):
    """A 2x7 cluster with t' (target sectors of 3432 x 3003 states, p = 14):
    the block H.v of the matrix continued fraction runs on the staged kernels;
    its G agrees with this solver's Lehmann G (pinned to the reference
    elsewhere) within 1e-8, for both off-diagonal block forms."""
    z = W.matsubara(64)
    prob = W.hubbard_cluster(7, 2, tp=0.3, U=6.0, mu=2.9)
    suffix, label = fresh()
    qed.load_problem(prob, label, model_name="mcf2x7_L" + suffix, fmt="F")
    GL = qed.Green_function(z, label=label)
    for qr in (False, True):
        suffix, label = fresh()
        qed.set_global_parameter("GF_method", "M")
        qed.set_global_parameter("block_Lanczos_QR", qr)
        try:
            qed.load_problem(prob, label, model_name=f"mcf2x7_{qr}" + suffix, fmt="F")
            G = qed.Green_function(z, label=label)
        finally:
            qed.set_global_parameter("GF_method", "L")
            qed.set_global_parameter("block_Lanczos_QR", False)
        assert np.max(np.abs(G - GL)) < 1e-8, (qr, np.max(np.abs(G - GL)))
