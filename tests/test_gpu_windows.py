"""GPU parity of the window H.v kernels (winhv.hpp) against the reference.

Sectors are taken through the window kernels (option hv_windows, off by
default) by lowering hv_windows_min_dim;
the H.v (host and device entries, with the fused reductions) is compared with
the compiled reference's Hamiltonian_Factorized::mult_add within 1e-13 relative
(FP64 round-off of another summation order), the Lanczos ground state within
1e-10. The process-wide window launch count shows that the window kernels, not
the staged ones, ran.
"""
import numpy as np
import pytest

from pyqcm_b200 import workloads as W
from tests.helpers import load_both, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture
def windows_everywhere(qed):
    qed.set_global_parameter("hv_windows", True)
    qed.set_global_parameter("hv_windows_min_dim", 0)
    yield
    qed.set_global_parameter("hv_windows", False)
    qed.set_global_parameter("hv_windows_min_dim", 1 << 22)


CASES = [
    # 4x4 with t': three windows; equal and unequal spin dimensions (560, 1820)
    ("sq4x4_N6", lambda: W.square4x4(), "R0:N6:S0"),
    ("sq4x4_N7", lambda: W.square4x4(), "R0:N7:S1"),
    ("sq4x4_N7m", lambda: W.square4x4(), "R0:N7:S-1"),
    # 4x3 with t' at half filling: two windows, 924 x 924
    ("sq4x3_tp", lambda: W.hubbard_cluster(4, 3, tp=0.3, U=6.0, mu=3.0), "R0:N12:S0"),
    # 5x2 ladder with a Neel field (spin-dependent diagonal): two windows, 252 x 252
    ("neel5x2", lambda: W.hubbard_cluster(5, 2, U=5.0, mu=2.2, M=0.25), "R0:N10:S0"),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_window_hv_matches_reference(qed, oracle, fresh, windows_everywhere, case):
    import torch
    name, make, sec = CASES[case]
    prob = make()
    prob.sectors = sec
    suffix, label = fresh()
    load_both(qed, oracle, prob, suffix, label, fmt="F")
    H = qed.Hamiltonian(label, sec)
    Hr = oracle.RefHamiltonian(label, sec)
    rng = np.random.default_rng(case + 40)
    x = rng.standard_normal(H.dim)
    y_ref = rng.standard_normal(H.dim)
    y = y_ref.copy()
    Hr.mult_add(x, y_ref)
    H.mult_add(x, y)  # the host entry keeps its copy-overlapped pipeline of the staged passes
    assert rel_err(y, y_ref) < 1e-13, name
    n1 = qed.window_launches()
    # device entry with the fused reductions <x,y>, <y,y>, <x,x>: the window kernels
    hx = np.zeros(H.dim)
    Hr.mult_add(x, hx)
    xd = torch.tensor(x, device="cuda")
    yd = torch.empty_like(xd)
    dots = torch.zeros(3, dtype=torch.float64, device="cuda")
    for _ in range(2):
        H.apply_dots_device(xd.data_ptr(), yd.data_ptr(), dots.data_ptr(), torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert rel_err(yd.cpu().numpy(), hx) < 1e-13, name
        d = dots.cpu().numpy()
        assert abs(d[0] - x @ hx) < 1e-10 * abs(x @ hx)
        assert abs(d[1] - hx @ hx) < 1e-10 * (hx @ hx)
        assert abs(d[2] - x @ x) < 1e-12 * (x @ x)
    assert qed.window_launches() >= n1 + 2, "the window kernels did not run"


def test_window_ground_state_matches_reference(qed, oracle, fresh, windows_everywhere):
    """Lanczos ground state through the window kernels (the subtraction list and
    the reductions in the up-spin pass) against the reference's own Lanczos."""
    prob = W.hubbard_cluster(4, 3, tp=0.3, U=6.0, mu=3.0)
    prob.sectors = "R0:N12:S0"
    suffix, label = fresh()
    load_both(qed, oracle, prob, suffix, label, fmt="F")
    n0 = qed.window_launches()
    e1, _ = qed.ground_state_solve(label)
    e2, _ = oracle.ground_state(label)
    assert qed.window_launches() > n0
    assert abs(e1 - e2) < 1e-10 * abs(e2), (e1, e2)


def test_window_and_staged_kernels_agree(qed, oracle, fresh):
    """The same 4x4 sector (N_up = N_dn = 4, 1820^2 states) through the window
    kernels and through the staged kernels (device entry): H x within 1e-13
    relative."""
    prob = W.square4x4()
    prob.sectors = "R0:N8:S0"
    suffix, label = fresh()
    load_both(qed, oracle, prob, suffix, label, fmt="F")
    x = np.random.default_rng(3).standard_normal(1820 * 1820)
    ys = []
    for use in (True, False):
        qed.set_global_parameter("hv_windows", use)
        qed.set_global_parameter("hv_windows_min_dim", 0)
        try:
            import torch
            n0 = qed.window_launches()
            H = qed.Hamiltonian(label, prob.sectors)
            xd = torch.tensor(x, device="cuda")
            yd = torch.empty_like(xd)
            H.apply_device(xd.data_ptr(), yd.data_ptr(), torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            assert (qed.window_launches() > n0) == use
            ys.append(yd.cpu().numpy())
        finally:
            qed.set_global_parameter("hv_windows", False)
            qed.set_global_parameter("hv_windows_min_dim", 1 << 22)
    assert rel_err(ys[0], ys[1]) < 1e-13
