"""Generates the golden fixtures in tests/golden/ by running the reference's own
ED (the compiled oracle, oracle/_ref) on the synthetic workloads.

    python tests/golden/make_golden.py            # small cases (seconds)
    python tests/golden/make_golden.py --big      # 4x4 ground state (about 1.5 h on one core)
    python tests/golden/make_golden.py --sq4x3    # 4x3 ground state + Green function (minutes)

Fixtures:
  small_cases.npz : names, E0, G (256 Matsubara points, beta = 50) for
                    chain8 (band Lanczos and continued fraction), 2x3 with t',
                    2x4 with a Neel field (both spins), plaquette + 8 bath, chain10
  sq4x4_gs.json   : ground-state energy and sector of the 4x4 cluster (t'=0.3, U=8)
  sq4x3_gf.npz    : 4x3 cluster (t'=0.3, U=8, half filling, dim 853776): E0, Potthoff
                    functional and G on 64 Matsubara points (band Lanczos, p = 12)
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref  # noqa: E402
from pyqcm_b200 import workloads as W  # noqa: E402


def small():
    cases = [
        ("chain8_L", W.chain8(), "L"),
        ("chain8_F", W.chain8(), "F"),
        ("sq2x3_tp_L", W.hubbard_cluster(3, 2, tp=0.3, U=6.0), "L"),
        ("neel2x4_L", W.hubbard_cluster(4, 2, U=5.0, mu=1.7, M=0.25), "L"),
        ("plaq8b_L", W.plaquette_bath(np.linspace(-1.5, 1.5, 8), np.linspace(0.2, 0.9, 8)), "L"),
        ("chain10_L", W.hubbard_cluster(10, 1, U=7.0), "L"),
    ]
    z = W.matsubara(256)
    names, E0, G, Gd, omega = [], [], [], [], []
    for k, (name, prob, method) in enumerate(cases):
        ref.set_param("GF_method", method)
        ref.load_problem(prob, 500 + k, model_name="golden_" + name, fmt="S" if method == "F" else "F")
        e, _ = ref.ground_state(500 + k)
        names.append(name)
        E0.append(e)
        G.append(ref.green_function(500 + k, z))
        Gd.append(ref.green_function(500 + k, z, spin_down=True) if ref.mixing(500 + k) & 4
                  else np.zeros_like(G[-1]))
        omega.append(ref.potthoff(500 + k))
        print(f"{name}: E0 = {e:.15g}")
    ref.set_param("GF_method", "L")
    n = max(g.shape[1] for g in G)
    pad = lambda g: np.pad(g, ((0, 0), (0, n - g.shape[1]), (0, n - g.shape[2])))
    np.savez_compressed(os.path.join(HERE, "small_cases.npz"), names=np.array(names), E0=np.array(E0),
                        G=np.array([pad(g) for g in G]), G_down=np.array([pad(g) for g in Gd]),
                        dims=np.array([g.shape[1] for g in G]), omega=np.array(omega), z=z)


def big():
    prob = W.square4x4()
    ref.set_param("GF_method", "L")
    ref.load_problem(prob, 600, model_name="golden_sq4x4", fmt="F")
    t = time.time()
    e, sec = ref.ground_state(600)
    out = dict(workload="4x4 Hubbard, open, t=-1, t'=0.3, U=8, mu=4, R0:N16:S0", E0=e, sector=sec,
               seconds=time.time() - t, threads=1)
    with open(os.path.join(HERE, "sq4x4_gs.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(out)


def sq4x3():
    prob = W.hubbard_cluster(4, 3, t=-1.0, tp=0.3, U=8.0, mu=4.0, name="sq4x3")
    ref.set_param("GF_method", "L")
    ref.load_problem(prob, 700, model_name="golden_sq4x3", fmt="F")
    t = time.time()
    e, sec = ref.ground_state(700)
    z = W.matsubara(64)
    G = ref.green_function(700, z)
    om = ref.potthoff(700)
    np.savez_compressed(os.path.join(HERE, "sq4x3_gf.npz"), E0=e, sector=sec, G=G, z=z, omega=om,
                        seconds=time.time() - t)
    print(e, sec, om, time.time() - t)


if __name__ == "__main__":
    if "--big" in sys.argv:
        big()
    elif "--sq4x3" in sys.argv:
        sq4x3()
    else:
        small()
