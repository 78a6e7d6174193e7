"""Spin tables built on the host (small tables, option host_table_max_dim) equal
the device-built ones bit for bit: the same strings, hop entries, bank-ordered
and packed copies and diagonal, hence the same H x and the same Lanczos energy
to the last bit. Checked by building every case both ways."""
import numpy as np
import pytest

from pyqcm_b200 import workloads as W
from tests.helpers import load_both

pytestmark = pytest.mark.gpu

CASES = [
    ("chain8", W.chain8(), "R0:N8:S0"),
    ("sq2x3_tp", W.hubbard_cluster(3, 2, tp=0.3, U=6.0), "R0:N6:S0"),
    ("neel2x4", W.hubbard_cluster(4, 2, U=5.0, mu=1.7, M=0.25), "R0:N8:S0"),
    ("plaq8b", W.plaquette_bath(np.linspace(-1.5, 1.5, 8), np.linspace(0.2, 0.9, 8)), "R0:N12:S0"),
    # spin tables of 3432 / 3003 strings: bank-ordered and packed copies (staged kernels)
    ("sq2x7_tp_N13", W.hubbard_cluster(7, 2, tp=0.3, U=6.0, mu=2.9), "R0:N13:S1"),
]


@pytest.mark.parametrize("case", range(len(CASES)))
def test_host_tables_equal_device_tables(qed, oracle, fresh, case):
    import torch
    name, prob, sec = CASES[case]
    prob.sectors = sec
    ys, es = [], []
    for limit in (1 << 20, 0):  # host build, then device build
        qed.set_global_parameter("host_table_max_dim", limit)
        try:
            suffix, label = fresh()
            load_both(qed, oracle, prob, suffix, label, fmt="F")
            H = qed.Hamiltonian(label, sec)
            x = torch.tensor(np.random.default_rng(7).standard_normal(H.dim), device="cuda")
            y = torch.empty_like(x)
            H.apply_device(x.data_ptr(), y.data_ptr(), torch.cuda.current_stream().cuda_stream)
            torch.cuda.synchronize()
            ys.append(y.cpu().numpy())
            es.append(qed.ground_state_solve(label)[0])
        finally:
            qed.set_global_parameter("host_table_max_dim", 4096)
    assert np.array_equal(ys[0], ys[1]), name
    assert es[0] == es[1], (name, es)
