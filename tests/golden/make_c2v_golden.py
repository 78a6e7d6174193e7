"""Generates tests/golden/c2v_8b.json from the reference's own diagonalization test
record tests/test_diagonalization/S_format.ref: a 2x2 plaquette with 8 bath orbitals
and the C2v symmetry generators of model_2x2_2C_8b_C2v_L (cluster 'clus'), solved by
the reference in its CSR format with the symmetry-adapted (mixed) basis.

Written out: the cluster model (sites, bath, generators as pyqcm takes them:
1-based sites, bath entries as irrep phases because bath_irrep=True), its operators
(0-based orbitals, spin down at i + 12, as ED::new_operator takes them), the
instance parameters that reach the ED solver (U and mu of the lattice acting on the
four correlated sites, the cluster parameters eb*_1 / tb*_1 under their cluster
names), the target sector, and the reference's results: the ground-state energy
(6 significant digits in the record) and, per irrep of the cluster's site orbitals,
the Lehmann poles (e_i, v_i) of the spin-up Green function in the symmetric-orbital
basis (14 digits).

The lattice operators that are not set in the record (tc, D, hx) are zero and the
ones acting only on the uncorrelated cluster (e, tpd, tpp, tppp, Ud) do not reach
this cluster's ED instance, so they are not written.

    python tests/golden/make_c2v_golden.py
"""
import ast
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
from oracle.refpath import reference_file  # noqa: E402

REF = reference_file("tests/test_diagonalization/S_format.ref")


def _call_args(line):
    call = ast.parse(line.strip()).body[0].value
    args = [ast.literal_eval(a) for a in call.args]
    kw = {k.arg: ast.literal_eval(k.value) for k in call.keywords}
    return args, kw


def main():
    lines = open(REF).read().splitlines()
    model, operators, params = None, {}, {}
    for ln in lines:
        if ln.startswith("new_cluster_model('clus',"):
            args, kw = _call_args(ln)
            model = {"name": args[0], "n_sites": args[1], "n_bath": args[2],
                     "generators": kw["generators"], "bath_irrep": bool(kw["bath_irrep"])}
        elif ln.startswith("new_cluster_operator('clus',"):
            args, _ = _call_args(ln)
            _, name, typ, elems = args
            if typ != "one-body":
                continue  # the anomalous sb* operators are not set in the record
            operators[name] = (typ, [(r - 1, c - 1, float(v)) for (r, c, v) in elems])
        elif ln.startswith("set_parameter("):
            args, _ = _call_args(ln)
            params[args[0]] = float(args[1])
    n_orb = model["n_sites"] + model["n_bath"]
    ns = model["n_sites"]
    # lattice operators acting on the correlated cluster's sites
    operators["U"] = ("interaction", [(i, i + n_orb, 1.0) for i in range(ns)])
    operators["mu"] = ("one-body", [(i, i, -1.0) for i in range(ns)] +
                       [(i + n_orb, i + n_orb, -1.0) for i in range(ns)])
    inst = {"U": params["U"], "mu": params["mu"]}
    for k, v in params.items():
        if k.endswith("_1"):
            inst[k[:-2]] = v

    gs = None
    blocks = []
    i = 0
    while i < len(lines):
        ln = lines[i]
        if ln.startswith("GS_energy:") and gs is None:
            t = ln.split()
            gs = {"energy": float(t[1]), "sector": t[3]}
        if ln.startswith("w\t") and len(blocks) < 4:
            _, L, M = ln.split()
            L, M = int(L), int(M)
            e, v = [], []
            for row in lines[i + 1:i + 1 + M]:
                a, b = row.split()
                e.append(float(a))
                v.append(float(b))
            blocks.append({"L": L, "M": M, "e": e, "v": v})
            i += M
        i += 1
    out = {"source": "tests/test_diagonalization/S_format.ref (reference)",
           "model": model, "operators": operators, "params": inst,
           "sectors": "R0:N12:S0", "gs": gs, "irrep_poles": blocks}
    with open(os.path.join(HERE, "c2v_8b.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("GS", gs, "blocks", [b["M"] for b in blocks], "ops", sorted(operators), inst)


if __name__ == "__main__":
    main()
