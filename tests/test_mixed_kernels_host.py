"""The mixed-basis kernels' own source (k_mixed_mark, k_mixed_rows, k_mixed_diag
and their device helpers in pyqcm_b200/csrc/mixed.cu), compiled for the host with
one-thread launch shims and run sequentially: the basis and every stored matrix
element against the numpy restatement of the reference (oracle/port_sym.py). This
checks the kernels' index arithmetic (colex ranks, factorized-index map, fermion
signs, phases, orbit-length ratios) without a GPU."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle import port_sym
from pyqcm_b200 import workloads as W
from tests.helpers import c2v_golden, c2v_problem

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "pyqcm_b200", "csrc")
HERE = os.path.join(ROOT, "tests", "host_emulation")

SHIM = r'''
#include <cstdint>
#include <cmath>
#include <cstdio>
#include <vector>
#define __global__
#define __device__
#define __forceinline__ inline
#define __restrict__
#include "symmetry.cuh"
struct D3 { unsigned x; };
static D3 blockIdx{0}, blockDim{1}, gridDim{1}, threadIdx{0};
static uint32_t c_mbinom[33][33];
inline int __ffs(uint32_t x) { return __builtin_ffs(x); }
inline int __popcll(uint64_t x) { return __builtin_popcountll(x); }
using std::sqrt;
namespace qed {
'''


def _grab(src, start):
    i = src.index(start)
    depth, j, seen = 0, i, False
    while True:
        c = src[j]
        if c == "{":
            depth += 1
            seen = True
        elif c == "}":
            depth -= 1
            if seen and depth == 0:
                return src[i:j + 1]
        j += 1


@pytest.fixture(scope="module")
def emulator(tmp_path_factory):
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    src = open(os.path.join(CSRC, "mixed.cu")).read()
    k = src.index("struct OffTerms {")
    parts = [src[k:src.index("};", k) + 2],
             _grab(src, "__device__ __forceinline__ uint32_t colex_rank"),
             _grab(src, "__device__ __forceinline__ uint64_t orb_mask"),
             _grab(src, "__global__ void k_mixed_mark"),
             _grab(src, "template <bool fill>\n__global__ void k_mixed_rows"),
             _grab(src, "__global__ void k_mixed_diag")]
    d = tmp_path_factory.mktemp("mixed_emu")
    (d / "kernels_host.hpp").write_text(SHIM + "\n\n".join(parts) + "\n}\n")
    exe = d / "emu"
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", str(d), "-I", CSRC, "-I", os.path.join(ROOT, "include"),
                    "-I", cuda_inc, os.path.join(HERE, "mixed_rows_main.cpp"), os.path.join(CSRC, "symmetry.cpp"),
                    "-o", str(exe)], check=True, capture_output=True)
    return str(exe)


def _terms(prob):
    n = prob.n_orb
    mk = lambda i: (1 << (i - n + 32)) if i >= n else (1 << i)
    off, diag = {}, {}
    for name, val in prob.params.items():
        if name not in prob.operators:
            continue
        typ, el = prob.operators[name]
        for (r, c, v) in el:
            if typ == "interaction":
                r, c = min(r, c), max(r, c)
                diag[mk(r) + mk(c)] = diag.get(mk(r) + mk(c), 0.0) + val * v
            elif r == c:
                diag[mk(r)] = diag.get(mk(r), 0.0) + val * v
            elif r < c:
                off[(r, c)] = off.get((r, c), 0.0) + val * v
                off[(c, r)] = off.get((c, r), 0.0) + val * v
    return off, diag


def _sq2x3():
    p = W.hubbard_cluster(3, 2, tp=0.3, U=6.0, mu=2.5)
    p.generators = [[3, 2, 1, 6, 5, 4], [4, 5, 6, 1, 2, 3]]
    return p


def _chain4():
    p = W.hubbard_cluster(4, 1, U=4.0)
    p.generators = [[4, 3, 2, 1]]
    return p


@pytest.mark.parametrize("case,sector", [("sq2x3", "R0:N6:S0"), ("sq2x3", "R1:N6:S0"), ("sq2x3", "R3:N5:S1"),
                                         ("record", "R0:N3:S1"), ("record", "R3:N4:S0"),
                                         ("chain4", "R1:N4:S0"), ("chain4", "R1:N3:S1")])
def test_mixed_kernels_on_the_host_match_the_restatement(emulator, case, sector):
    prob = {"sq2x3": _sq2x3, "chain4": _chain4, "record": lambda: c2v_problem(c2v_golden(), True)}[case]()
    r, N, S = (int(t[1:]) for t in sector.split(":"))
    gens0 = [[v - 1 if (i < prob.n_sites or not prob.bath_irrep) else v for i, v in enumerate(g)]
             for g in prob.generators]
    off, diag = _terms(prob)
    lines = [f"{prob.n_sites} {prob.n_bath} {int(prob.bath_irrep)} {len(gens0)}"]
    lines += [" ".join(map(str, g)) for g in gens0]
    lines.append(f"{r} {(N + S) // 2} {(N - S) // 2}")
    lines.append(str(len(off)))
    lines += [f"{a} {b} {v!r}" for (a, b), v in sorted(off.items())]
    lines.append(str(len(diag)))
    lines += [f"{m} {v!r}" for m, v in sorted(diag.items())]
    out = subprocess.run([emulator], input="\n".join(lines), capture_output=True, text=True,
                         check=True).stdout.split("\n")
    D = int(out[0])
    states = np.array([int(s.split()[0]) for s in out[1:1 + D]], dtype=np.uint64)
    A = np.diag([float(s.split()[1]) for s in out[1:1 + D]])
    for s in out[1 + D:]:
        if s.strip():
            J, K, v = s.split()
            A[int(J), int(K)] += float(v)
    G = port_sym.group(prob.n_sites, prob.n_bath, gens0, prob.bath_irrep)
    Hp, basis = port_sym.mixed_hamiltonian(prob, G, sector)
    assert np.array_equal(states, basis)
    assert np.max(np.abs(A - Hp.toarray())) < 1e-13


@pytest.fixture(scope="module")
def cdag_emulator(tmp_path_factory):
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    src = open(os.path.join(CSRC, "mixed.cu")).read()
    k = src.index("struct OffTerms {")
    parts = [src[k:src.index("};", k) + 2],
             _grab(src, "__device__ __forceinline__ uint32_t colex_rank"),
             _grab(src, "__device__ __forceinline__ uint64_t orb_mask"),
             _grab(src, "__global__ void k_mixed_mark"),
             src[src.index("struct OrbCoef {"):src.index("};", src.index("struct OrbCoef {")) + 2],
             _grab(src, "__device__ __forceinline__ int32_t mixed_index"),
             _grab(src, "__global__ void k_mixed_create"),
             _grab(src, "__global__ void k_mixed_destroy")]
    d = tmp_path_factory.mktemp("mixed_cdag_emu")
    (d / "kernels_host.hpp").write_text(SHIM + "\n\n".join(parts) + "\n}\n")
    exe = d / "emu"
    cuda_inc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "include")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", str(d), "-I", CSRC, "-I", os.path.join(ROOT, "include"),
                    "-I", cuda_inc, os.path.join(HERE, "mixed_cdag_main.cpp"), os.path.join(CSRC, "symmetry.cpp"),
                    "-o", str(exe)], check=True, capture_output=True)
    return str(exe)


@pytest.mark.parametrize("case,sector", [("record", "R0:N4:S0"), ("record", "R2:N5:S1"), ("sq2x3", "R0:N6:S0"),
                                         ("sq2x3", "R3:N5:S-1")])
def test_mixed_cdag_kernels_on_the_host_match_the_restatement(cdag_emulator, case, sector):
    """c and c+ of every symmetric orbital, both spins, on a random vector of the
    sector: the device gathers (creation over target states, destruction over
    the orbits of the target states) against the restatement's destruction
    matrices (oracle/port_sym.destroy_matrix, pinned to the reference)."""
    prob = {"sq2x3": _sq2x3, "record": lambda: c2v_problem(c2v_golden(), True)}[case]()
    r0, N, S = (int(t[1:]) for t in sector.split(":"))
    gens0 = [[v - 1 if (i < prob.n_sites or not prob.bath_irrep) else v for i, v in enumerate(g)]
             for g in prob.generators]
    G = port_sym.group(prob.n_sites, prob.n_bath, gens0, prob.bath_irrep)
    _, B0 = port_sym.mixed_hamiltonian(prob, G, sector)
    psi = np.random.default_rng(r0 + 7 * N).standard_normal(len(B0))
    rows, irr = port_sym.symmetric_orbitals(G, prob.n_sites)
    checked = 0
    for k, (s_row, r_orb) in enumerate(zip(rows, irr)):
        for spin in (0, 1):
            for pm in (1, -1):
                rt = port_sym.shift_irrep(G, r0, pm, r_orb)
                ds = -1 if spin else 1
                tsec = f"R{rt}:N{N + pm}:S{S + pm * ds}"
                _, Bt = port_sym.mixed_hamiltonian(prob, G, tsec)
                if len(Bt) == 0:
                    continue
                if pm == 1:
                    ref = port_sym.destroy_matrix(G, s_row, spin, Bt, rt, B0, r0).T @ psi
                else:
                    ref = port_sym.destroy_matrix(G, s_row, spin, B0, r0, Bt, rt) @ psi
                nu, nd = (N + S) // 2, (N - S) // 2
                lines = [f"{prob.n_sites} {prob.n_bath} {int(prob.bath_irrep)} {len(gens0)}"]
                lines += [" ".join(map(str, g)) for g in gens0]
                lines.append(f"{r0} {nu} {nd} {rt} {pm} {spin}")
                lines.append(" ".join(repr(float(c)) for c in s_row))
                lines.append(" ".join(repr(float(x)) for x in psi))
                out = subprocess.run([cdag_emulator], input="\n".join(lines), capture_output=True, text=True,
                                     check=True).stdout.split("\n")
                ds_, dt_ = (int(t) for t in out[0].split())
                assert ds_ == len(B0) and dt_ == len(Bt)
                st = np.array([int(s.split()[0]) for s in out[1:1 + dt_]], dtype=np.uint64)
                phi = np.array([float(s.split()[1]) for s in out[1:1 + dt_]])
                assert np.array_equal(st, Bt)
                assert np.max(np.abs(phi - ref)) <= 1e-13 * max(1.0, np.max(np.abs(ref))), (k, spin, pm)
                checked += 1
    assert checked >= 4
