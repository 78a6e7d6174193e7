"""Instance checkpoints in the reference's HDF5 layout (write_instance_to_hdf5 /
read_instance_from_hdf5): a solved instance written to a file and read into a
fresh instance of the same model gives the same Green function, average and
density without a new solve; the file's Q-matrix is the reference's own."""
import numpy as np
import pytest

from pyqcm_b200 import workloads as W
from tests.helpers import load_both, set_both

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case,method", [("chain8", "L"), ("neel2x4", "L"), ("chain8", "F")])
def test_checkpoint_round_trip(qed, oracle, fresh, tmp_path, case, method):
    from pyqcm_b200 import hdf5 as H
    mk = {"chain8": W.chain8, "neel2x4": lambda: W.hubbard_cluster(4, 2, U=5.0, mu=1.7, M=0.25)}[case]
    set_both(qed, oracle, GF_method=method)
    try:
        suffix, label = fresh()
        prob = mk()
        load_both(qed, oracle, prob, suffix, label, fmt="F" if method == "L" else "S")
        z = W.matsubara(64)
        G = qed.Green_function(z, label=label)
        e0, sec = qed.ground_state_solve(label)
        path = str(tmp_path / "ckpt.h5")
        qed.write_instance_to_hdf5(path, "cluster_0", label)
        root = H.read_file(path).group("cluster_0")
        assert root.attrs["GF_format"] == ("bl" if method == "L" else "cf")
        assert root.attrs["GS_energy"] == e0 and root.attrs["GS_sectors"] == sec
        assert root.attrs["nstates"] >= 1 and "params" in root
        # a fresh instance of the same model: nothing solved, then the file
        label2 = label + 50000
        qed.new_model_instance(prob.name + suffix, prob.params, prob.sectors, label2)
        qed.read_instance_from_hdf5(path, "cluster_0", label2)
        G2 = qed.Green_function(z, label=label2)
        assert np.max(np.abs(G2 - G)) < 1e-13
        for sd in ((False, True) if qed.mixing(label) & 4 else (False,)):
            assert np.max(np.abs(qed.Green_function_average(spin_down=sd, label=label2)
                                 - qed.Green_function_average(spin_down=sd, label=label))) < 1e-14
        assert qed.ground_state_solve(label2) == (e0, sec)
        if method == "L" and root.attrs["nstates"] == 1:  # the reference's Q-matrix of the same instance
            e_ref, v_ref = oracle.qmatrix(label)
            b = root.group("state_0").group("gf").group("block_0")
            e = b.dataset("e")
            v = b.group("v").dataset("data").reshape(int(b.attrs["M"]), int(b.attrs["L"])).T
            # (the unconverged top of the spectrum may hold a pole more or less:
            # compare the Lehmann sums, as the Green-function parity tests do)
            Gq = lambda ee, vv, w: (vv / (w - ee)) @ vv.conj().T
            for w in (0.3j, 1.7j):
                assert np.max(np.abs(Gq(e, v, w) - Gq(e_ref, v_ref, w))) < 1e-8
        qed.erase_model_instance(label2)
    finally:
        set_both(qed, oracle, GF_method="L")
