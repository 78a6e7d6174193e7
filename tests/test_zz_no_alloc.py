"""The no-allocation H.v entry point against the allocating one.

qed_hamiltonian_apply_dots_device_noalloc serves callers that cannot allocate
device memory when they call in (their device memory belongs to another
runtime's pool, or they cannot afford cudaMalloc's implicit synchronisation).
It must give the same y = H x and the same (<x,y>, <y,y>, <x,x>) as
qed_hamiltonian_apply_dots_device, call after call: its scratch is one fixed
array shared by all calls, so a second call must not see stale partial sums.
Tolerances: y within 1e-13 relative (identical kernels, same launch shape),
the dot products within 1e-12 relative.

This file is collected last so that a run stopping at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from pyqcm_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_entry_two_calls(qed, fresh):
    import torch

    L = qed.lib()
    f = L.qed_hamiltonian_apply_dots_device_noalloc
    f.argtypes = [C.c_void_p] * 5
    f.restype = C.c_int
    suffix, label = fresh()
    prob = W.hubbard_cluster(4, 2, U=5.0, mu=1.7, M=0.25)  # dim 4900, both spins differ
    qed.load_problem(prob, label, model_name="noalloc" + suffix)
    H = qed.Hamiltonian(label, prob.sectors)
    stream = torch.cuda.current_stream().cuda_stream
    rng = np.random.default_rng(11)
    for call in range(2):
        x = torch.tensor(rng.standard_normal(H.dim), device="cuda")
        y_ref = torch.full_like(x, np.nan)
        y_new = torch.full_like(x, np.nan)
        d_ref = torch.full((3,), np.nan, dtype=torch.float64, device="cuda")
        d_new = torch.full((3,), np.nan, dtype=torch.float64, device="cuda")
        H.apply_dots_device(x.data_ptr(), y_ref.data_ptr(), d_ref.data_ptr(), stream)
        rc = f(H._h, C.c_void_p(x.data_ptr()), C.c_void_p(y_new.data_ptr()), C.c_void_p(d_new.data_ptr()),
               C.c_void_p(stream))
        assert rc == 0, qed.QEDError(rc, "no-alloc entry failed")
        torch.cuda.synchronize()
        a, b = y_ref.cpu().numpy(), y_new.cpu().numpy()
        assert np.all(np.isfinite(b))
        assert np.max(np.abs(a - b)) <= 1e-13 * np.max(np.abs(a)), call
        da, db = d_ref.cpu().numpy(), d_new.cpu().numpy()
        assert np.all(np.abs(da - db) <= 1e-12 * np.abs(da)), (call, da, db)
        # and against the host path
        assert abs(db[2] - float((x * x).sum())) <= 1e-12 * abs(db[2])
