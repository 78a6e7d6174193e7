"""pyqcm_b200 -- B200 (sm_100a) exact-diagonalization solver for pyqcm's cluster path.

This module mirrors the reference's ED API (namespace ED, src_ed/qcm_ED.hpp:23-340,
as exposed to Python by src_python/qcm_ED_wrap.hpp) on top of the C ABI in
include/qed_b200.h. Every call goes through the CUDA library
pyqcm_b200/libqed_b200.so; there is no CPU fallback: if the library or a GPU is
missing, the calls raise QEDError.

Differences from the reference's Python binding, all deliberate:
  * operator matrix elements are 0-based (the C++ ED API convention);
  * Green_function / self_energy / hybridization_function accept an array of
    frequencies and evaluate all of them in one GPU launch.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

__all__ = [
    "QEDError", "lib", "set_global_parameter", "new_model", "new_operator", "new_model_instance",
    "erase_model_instance", "mixing", "ground_state_solve", "Green_function_solve",
    "Green_function_dimension", "Green_function", "self_energy", "hybridization_function",
    "Green_function_average", "Potthoff_functional", "qmatrix", "cf_coefficients",
    "ground_state_vector", "Hamiltonian", "halfbasis", "halfbasis_rank", "destroy_table",
    "load_problem",
]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqed_b200.so")

QED_OK = 0
QED_ERR_ARGUMENT = 1
QED_ERR_UNSUPPORTED = 6
QED_ERR_NO_DEVICE = 7
_CODES = {1: "argument", 2: "lanczos", 3: "qmatrix", 4: "cuda", 5: "memory", 6: "unsupported",
          7: "no-device", 8: "internal"}


class QEDError(RuntimeError):
    """Error raised by the solver; .code is the C-ABI status (include/qed_b200.h)."""

    def __init__(self, code, msg):
        super().__init__(f"[{_CODES.get(code, code)}] {msg}")
        self.code = code


_lib = None


def lib():
    """Loads the CUDA library (built by python -m pyqcm_b200.build)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise QEDError(7, f"CUDA extension not built: {LIB_PATH} (run python -m pyqcm_b200.build)")
    L = C.CDLL(LIB_PATH)
    dp = C.POINTER(C.c_double)
    ip = C.POINTER(C.c_int)
    lp = C.POINTER(C.c_long)
    up = C.POINTER(C.c_uint)
    sig = {
        "qed_last_error": [C.c_char_p, C.c_int],
        "qed_hv_tuning_report": [C.c_char_p, C.c_int],
        "qed_window_plan": [C.c_int, C.c_int, C.c_int, ip, ip, dp, dp, dp, ip],
        "qed_window_compile": [C.c_int, C.c_int, C.c_int, C.c_int, ip, ip, C.c_char_p, C.c_int, ip],
        "qed_window_launches": [C.POINTER(C.c_longlong)],
        "qed_spin_table_host": [C.c_int, C.c_int, dp, dp, C.c_int, up, C.POINTER(C.c_ubyte), dp, up, C.c_long,
                                ip, dp, ip],
        "qed_init": [C.c_int],
        "qed_set_global_int": [C.c_char_p, C.c_long],
        "qed_set_global_double": [C.c_char_p, C.c_double],
        "qed_set_global_char": [C.c_char_p, C.c_char],
        "qed_set_global_bool": [C.c_char_p, C.c_int],
        "qed_get_global_double": [C.c_char_p, dp],
        "qed_new_model": [C.c_char_p, C.c_int, C.c_int],
        "qed_new_operator": [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, ip, ip, dp],
        "qed_new_model_instance": [C.c_char_p, C.c_int, C.POINTER(C.c_char_p), dp, C.c_char_p, C.c_int],
        "qed_erase_model_instance": [C.c_int],
        "qed_mixing": [C.c_int, ip],
        "qed_ground_state_solve": [C.c_int, dp, C.c_char_p, C.c_int],
        "qed_Green_function_solve": [C.c_int],
        "qed_Green_function_dimension": [C.c_int, ip],
        "qed_Green_function": [C.c_int, C.c_int, C.c_int, dp, dp],
        "qed_self_energy": [C.c_int, C.c_int, C.c_int, dp, dp],
        "qed_hybridization_function": [C.c_int, C.c_int, C.c_int, dp, dp],
        "qed_Green_function_average": [C.c_int, C.c_int, dp],
        "qed_Green_function_average_dimension": [C.c_int, ip],
        "qed_Potthoff_functional": [C.c_int, dp],
        "qed_cluster_averages": [C.c_int, C.c_int, ip, dp, dp, C.c_char_p, C.c_int],
        "qed_model_size": [C.c_char_p, ip, ip, ip],
        "qed_operator_exists": [C.c_char_p, C.c_char_p, ip],
        "qed_matrix_elements": [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, C.c_int, ip, ip, ip, dp],
        "qed_complex_HS": [C.c_int, ip],
        "qed_Green_function_density": [C.c_int, dp],
        "qed_hopping_matrix": [C.c_int, C.c_int, dp],
        "qed_hopping_matrix_full": [C.c_int, C.c_int, C.c_int, ip, dp],
        "qed_interactions": [C.c_int, C.c_int, ip, ip, ip, dp],
        "qed_tr_sigma_inf": [C.c_int, dp],
        "qed_susceptibility": [C.c_int, C.c_char_p, C.c_int, dp, dp],
        "qed_fidelity": [C.c_int, C.c_int, dp],
        "qed_susceptibility_poles": [C.c_int, C.c_char_p, C.c_int, ip, dp, dp],
        "qed_qmatrix": [C.c_int, C.c_int, ip, ip, dp, dp],
        "qed_cf_coefficients": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, ip, dp, dp],
        "qed_instance_states": [C.c_int, ip, dp, C.c_char_p, C.c_int, ip, ip],
        "qed_instance_parameters": [C.c_int, C.c_int, ip, C.c_char_p, C.c_int, dp],
        "qed_instance_state": [C.c_int, C.c_int, C.c_char_p, C.c_int, dp, dp],
        "qed_instance_state_qmatrix": [C.c_int, C.c_int, C.c_int, C.c_int, ip, ip, dp, dp],
        "qed_instance_state_cf": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, ip, dp, dp],
        "qed_instance_load_begin": [C.c_int, C.c_double, C.c_int, C.c_int],
        "qed_instance_load_state": [C.c_int, C.c_char_p, C.c_double, C.c_double, ip],
        "qed_instance_load_qmatrix": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, dp, dp],
        "qed_instance_load_cf": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, dp, dp],
        "qed_instance_load_end": [C.c_int],
        "qed_ground_state_vector": [C.c_int, lp, dp],
        "qed_hamiltonian_create": [C.c_int, C.c_char_p, C.POINTER(C.c_void_p), lp],
        "qed_hamiltonian_mult_add": [C.c_void_p, dp, dp],
        "qed_hamiltonian_apply_device": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
        "qed_hamiltonian_apply_dots_device": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
        "qed_hamiltonian_diag": [C.c_void_p, dp],
        "qed_hamiltonian_destroy": [C.c_void_p],
        "qed_halfbasis": [C.c_int, C.c_int, up, lp],
        "qed_halfbasis_rank": [C.c_int, C.c_int, C.c_long, up, up],
        "qed_destroy_table": [C.c_int, C.c_int, C.c_int, C.c_int, lp, ip],
        "qed_new_model_generators": [C.c_char_p, C.c_int, C.c_int, C.c_int, ip, C.c_int],
        "qed_mixed_hamiltonian_create": [C.c_int, C.c_char_p, C.POINTER(C.c_void_p), lp],
        "qed_mixed_hamiltonian_states": [C.c_void_p, C.POINTER(C.c_uint64)],
        "qed_mixed_hamiltonian_mult_add": [C.c_void_p, dp, dp],
        "qed_mixed_hamiltonian_apply_device": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
        "qed_mixed_hamiltonian_ground_state": [C.c_void_p, dp, ip],
        "qed_mixed_hamiltonian_ground_state_vector": [C.c_void_p, dp, dp],
        "qed_mixed_hamiltonian_nnz": [C.c_void_p, lp],
        "qed_mixed_hamiltonian_destroy": [C.c_void_p],
        "qed_symmetry_group": [C.c_int, C.c_int, C.c_int, ip, C.c_int, ip, ip, dp, dp, ip],
        "qed_symmetry_representatives": [C.c_int, C.c_int, C.c_int, ip, C.c_int, C.c_int, C.c_long,
                                         C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), ip, ip],
        "qed_sef_integrand_grid": [C.c_int, C.c_int, C.c_int, dp, C.c_int, ip, ip, ip, dp, C.c_int, dp,
                                   C.c_int, C.c_int, C.c_int, dp],
        "qed_cpt_projected_green_function": [C.c_int, C.c_int, C.c_int, dp, C.c_int, ip, ip, ip, dp, C.c_int,
                                             dp, C.c_int, C.c_int, C.c_int, C.c_double, dp],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    _lib = L
    return L


def _check(rc):
    if rc != QED_OK:
        buf = C.create_string_buffer(8192)
        lib().qed_last_error(buf, 8192)
        raise QEDError(rc, buf.value.decode(errors="replace"))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def init(device: int = 0):
    _check(lib().qed_init(device))


# ---- options ----------------------------------------------------------------

def set_global_parameter(name: str, value=None):
    """set_global_parameter (src_python/qcm_ED_wrap.hpp:296-315): None sets a bool to True."""
    L, n = lib(), name.encode()
    if value is None or isinstance(value, bool):
        _check(L.qed_set_global_bool(n, 1 if value is None else int(value)))
    elif isinstance(value, (int, np.integer)):
        _check(L.qed_set_global_int(n, int(value)))
    elif isinstance(value, float):
        _check(L.qed_set_global_double(n, value))
    elif isinstance(value, str) and len(value) == 1:
        _check(L.qed_set_global_char(n, value.encode()))
    else:
        raise TypeError(f"unknown type of global_parameter: {value!r}")


def get_global_double(name: str) -> float:
    v = C.c_double()
    _check(lib().qed_get_global_double(name.encode(), C.byref(v)))
    return v.value


# ---- models and instances ---------------------------------------------------

def new_model(name: str, n_sites: int, n_bath: int = 0, generators=None, bath_irrep: bool = False):
    """ED::new_model. generators: pyqcm's symmetry generators (1-based sites); a
    model with a nontrivial group has its sector Hamiltonians in the
    symmetry-adapted basis (MixedHamiltonian) but no ground-state solve yet."""
    if not generators:
        _check(lib().qed_new_model(name.encode(), n_sites, n_bath))
        return
    ng, flat = _generators_abi(n_sites, n_bath, generators, bath_irrep)
    _check(lib().qed_new_model_generators(name.encode(), n_sites, n_bath, ng,
                                          flat.ctypes.data_as(C.POINTER(C.c_int)), int(bool(bath_irrep))))


def new_operator(model: str, op: str, typ: str, elements):
    """elements: iterable of 0-based (r, c, v)."""
    el = list(elements)
    n = len(el)
    r = (C.c_int * max(n, 1))(*[int(e[0]) for e in el])
    c = (C.c_int * max(n, 1))(*[int(e[1]) for e in el])
    v = (C.c_double * max(n, 1))(*[float(e[2]) for e in el])
    _check(lib().qed_new_operator(model.encode(), op.encode(), typ.encode(), n, r, c, v))


def new_model_instance(model: str, values: dict, sectors: str, label: int = 0):
    names = list(values)
    arr = (C.c_char_p * max(len(names), 1))(*[k.encode() for k in names])
    vals = (C.c_double * max(len(names), 1))(*[float(values[k]) for k in names])
    _check(lib().qed_new_model_instance(model.encode(), len(names), arr, vals, sectors.encode(), label))


def load_problem(prob, label: int = 0, model_name: str | None = None, fmt: str | None = None):
    """Defines the model (with its operators) of a workloads.ClusterProblem and an instance.

    fmt, if given, is set as the Hamiltonian_format option first ('F' factorized:
    Lanczos in every sector; 'S', 'E', 'O', 'N': sectors below max_dim_full are
    diagonalised densely, as in the reference). The format is latched by the
    model's first instance."""
    if fmt is not None:
        set_global_parameter("Hamiltonian_format", fmt)
    mname = model_name or prob.name
    new_model(mname, prob.n_sites, prob.n_bath, getattr(prob, "generators", None),
              getattr(prob, "bath_irrep", False))
    for op, (typ, el) in prob.operators.items():
        new_operator(mname, op, typ, el)
    new_model_instance(mname, prob.params, prob.sectors, label)


def erase_model_instance(label: int):
    _check(lib().qed_erase_model_instance(label))


def mixing(label: int = 0) -> int:
    m = C.c_int()
    _check(lib().qed_mixing(label, C.byref(m)))
    return m.value


def ground_state_solve(label: int = 0):
    """Returns (ground-state energy, sector string), like ED::ground_state_solve."""
    E = C.c_double()
    buf = C.create_string_buffer(1024)
    _check(lib().qed_ground_state_solve(label, C.byref(E), buf, 1024))
    return E.value, buf.value.decode()


def Green_function_solve(label: int = 0):
    _check(lib().qed_Green_function_solve(label))


def ground_state_solve_batch(labels, threads: int = 0):
    """Ground states of many instances at once, on `threads` host threads with one
    CUDA stream each (0 = all hardware threads). Returns the energies."""
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    e = np.zeros(len(lab))
    L = lib()
    L.qed_ground_state_solve_batch.argtypes = [C.POINTER(C.c_int), C.c_int, C.c_int, C.POINTER(C.c_double)]
    L.qed_ground_state_solve_batch.restype = C.c_int
    _check(L.qed_ground_state_solve_batch(lab.ctypes.data_as(C.POINTER(C.c_int)), len(lab), threads, _dp(e)))
    return e


def Green_function_solve_batch(labels, threads: int = 0):
    """Green_function_solve for many instances at once (see ground_state_solve_batch)."""
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    L = lib()
    L.qed_Green_function_solve_batch.argtypes = [C.POINTER(C.c_int), C.c_int, C.c_int]
    L.qed_Green_function_solve_batch.restype = C.c_int
    _check(L.qed_Green_function_solve_batch(lab.ctypes.data_as(C.POINTER(C.c_int)), len(lab), threads))


QED_BATCH_GROUND_STATE = 1
QED_BATCH_GREEN_FUNCTION = 2


def batch_submit(labels, what: int = QED_BATCH_GREEN_FUNCTION, threads: int = 0) -> int:
    """Hands the ground states (what = QED_BATCH_GROUND_STATE) or Green functions
    (QED_BATCH_GREEN_FUNCTION) of `labels` to a background thread and returns a
    ticket at once (qed_batch_submit)."""
    lab = np.ascontiguousarray(labels, dtype=np.int32)
    t = C.c_longlong()
    L = lib()
    L.qed_batch_submit.argtypes = [C.POINTER(C.c_int), C.c_int, C.c_int, C.c_int, C.POINTER(C.c_longlong)]
    L.qed_batch_submit.restype = C.c_int
    _check(L.qed_batch_submit(lab.ctypes.data_as(C.POINTER(C.c_int)), len(lab), what, threads, C.byref(t)))
    return t.value


def batch_poll(ticket: int) -> bool:
    """True once the batch has finished (its failure, if any, is raised then and
    the ticket released); False while it runs."""
    d = C.c_int()
    L = lib()
    L.qed_batch_poll.argtypes = [C.c_longlong, C.POINTER(C.c_int)]
    L.qed_batch_poll.restype = C.c_int
    _check(L.qed_batch_poll(ticket, C.byref(d)))
    return bool(d.value)


def batch_wait(ticket: int, timeout: float | None = None) -> bool:
    """Waits for the batch (at most `timeout` seconds if given); as batch_poll."""
    d = C.c_int()
    L = lib()
    L.qed_batch_wait.argtypes = [C.c_longlong, C.c_int, C.POINTER(C.c_int)]
    L.qed_batch_wait.restype = C.c_int
    _check(L.qed_batch_wait(ticket, -1 if timeout is None else int(timeout * 1000), C.byref(d)))
    return bool(d.value)


def Green_function_dimension(label: int = 0) -> int:
    d = C.c_int()
    _check(lib().qed_Green_function_dimension(label, C.byref(d)))
    return d.value


def _zbatch(fn, z, spin_down, label):
    scalar = np.ndim(z) == 0
    zz = np.ascontiguousarray(np.atleast_1d(np.asarray(z, dtype=np.complex128)))
    n = Green_function_dimension(label)
    out = np.zeros((len(zz), n, n), dtype=np.complex128)
    _check(fn(label, int(spin_down), len(zz), _dp(zz.view(np.float64)), _dp(out.view(np.float64))))
    out = out.transpose(0, 2, 1)  # column-major blocks -> [k, row, col]
    return out[0].copy() if scalar else out.copy()


def Green_function(z, spin_down: bool = False, label: int = 0):
    """G(z) (n x n) for a scalar z, or (nz, n, n) for an array of frequencies."""
    return _zbatch(lib().qed_Green_function, z, spin_down, label)


def self_energy(z, spin_down: bool = False, label: int = 0):
    return _zbatch(lib().qed_self_energy, z, spin_down, label)


def hybridization_function(z, spin_down: bool = False, label: int = 0):
    return _zbatch(lib().qed_hybridization_function, z, spin_down, label)


def Green_function_average(spin_down: bool = False, label: int = 0):
    d = C.c_int()
    _check(lib().qed_Green_function_average_dimension(label, C.byref(d)))
    n = d.value
    out = np.zeros((n, n), dtype=np.complex128)
    _check(lib().qed_Green_function_average(label, int(spin_down), _dp(out.view(np.float64))))
    return out.T.copy()


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _dpp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def model_size(model: str):
    """ED::model_size: (n_sites, n_bath, number of group elements)."""
    a, b, c = C.c_int(), C.c_int(), C.c_int()
    _check(lib().qed_model_size(model.encode(), C.byref(a), C.byref(b), C.byref(c)))
    return a.value, b.value, c.value


def exists(model: str, op: str) -> bool:
    """ED::exists: whether the model defines the operator."""
    f = C.c_int()
    _check(lib().qed_operator_exists(model.encode(), op.encode(), C.byref(f)))
    return bool(f.value)


def matrix_elements(model: str, op: str):
    """ED::matrix_elements: (type, [(r, c, v), ...]) of an operator, 0-based orbitals."""
    cap = 1 << 14
    r, c, v = np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros(cap)
    n = C.c_int()
    t = C.create_string_buffer(64)
    _check(lib().qed_matrix_elements(model.encode(), op.encode(), t, len(t), cap, C.byref(n), _ip(r), _ip(c), _dpp(v)))
    return t.value.decode(), [(int(r[i]), int(c[i]), float(v[i])) for i in range(n.value)]


def complex_HS(label: int = 0) -> bool:
    f = C.c_int()
    _check(lib().qed_complex_HS(label, C.byref(f)))
    return bool(f.value)


def Green_function_density(label: int = 0) -> float:
    d = C.c_double()
    _check(lib().qed_Green_function_density(label, C.byref(d)))
    return d.value


def _square_complex(nrow, call):
    out = np.zeros((nrow, nrow), dtype=np.complex128)
    buf = np.zeros(2 * nrow * nrow)
    call(_dpp(buf))
    out[:] = (buf[0::2] + 1j * buf[1::2]).reshape(nrow, nrow).T  # column-major
    return out


def hopping_matrix(spin_down: bool = False, label: int = 0):
    """ED::hopping_matrix: the cluster one-body matrix (n_sites x n_sites, complex)."""
    n = Green_function_dimension(label)
    return _square_complex(n, lambda p: _check(lib().qed_hopping_matrix(label, int(spin_down), p)))


def hopping_matrix_full(spin_down: bool = False, diag: bool = False, label: int = 0):
    """ED::hopping_matrix_full: cluster + bath one-body matrix ((n_sites + n_bath)^2, complex)."""
    d = C.c_int()
    _check(lib().qed_hopping_matrix_full(label, int(spin_down), int(diag), C.byref(d), None))
    return _square_complex(d.value, lambda p: _check(lib().qed_hopping_matrix_full(label, int(spin_down), int(diag),
                                                                                   C.byref(d), p)))


def interactions(label: int = 0):
    """ED::interactions: [(r, c, v * value), ...] of the instance's interaction operators."""
    cap = 1 << 14
    r, c, v = np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros(cap)
    n = C.c_int()
    _check(lib().qed_interactions(label, cap, C.byref(n), _ip(r), _ip(c), _dpp(v)))
    return [(int(r[i]), int(c[i]), float(v[i])) for i in range(n.value)]


def tr_sigma_inf(label: int = 0) -> float:
    """ED::tr_sigma_inf: trace of the self-energy at infinite frequency."""
    d = C.c_double()
    _check(lib().qed_tr_sigma_inf(label, C.byref(d)))
    return d.value


def susceptibility(op: str, w, label: int = 0):
    """ED::susceptibility: dynamical susceptibility of operator op at the complex frequencies w."""
    w = np.ascontiguousarray(np.atleast_1d(np.asarray(w, dtype=np.complex128)))
    chi = np.zeros(len(w), dtype=np.complex128)
    _check(lib().qed_susceptibility(label, op.encode(), len(w), _dpp(w.view(np.float64)), _dpp(chi.view(np.float64))))
    return chi


def susceptibility_poles(op: str, label: int = 0):
    """ED::susceptibility_poles: [(pole, residue), ...]."""
    cap = 1 << 14
    e, r = np.zeros(cap), np.zeros(cap)
    n = C.c_int()
    _check(lib().qed_susceptibility_poles(label, op.encode(), cap, C.byref(n), _dpp(e), _dpp(r)))
    return [(float(e[i]), float(r[i])) for i in range(n.value)]


def fidelity(label1: int, label2: int) -> float:
    """ED::fidelity: sum over same-sector state pairs of w1 w2 |<psi1|psi2>|^2."""
    d = C.c_double()
    _check(lib().qed_fidelity(label1, label2, C.byref(d)))
    return d.value


def cluster_averages(label: int = 0):
    """ED::cluster_averages: [(operator name, average, variance), ...] in name order."""
    cap = 256
    n = C.c_int(0)
    ave = np.zeros(cap)
    var = np.zeros(cap)
    buf = C.create_string_buffer(1 << 16)
    _check(lib().qed_cluster_averages(label, cap, C.byref(n), ave.ctypes.data_as(C.POINTER(C.c_double)),
                                      var.ctypes.data_as(C.POINTER(C.c_double)), buf, len(buf)))
    names = buf.value.decode().split("\n")[: n.value]
    return [(names[i], float(ave[i]), float(var[i])) for i in range(n.value)]


def Potthoff_functional(label: int = 0) -> float:
    w = C.c_double()
    _check(lib().qed_Potthoff_functional(label, C.byref(w)))
    return w.value


def sef_integrand_grid(V0, r, c, R, v, w, nk, spin_down: bool = False, label: int = 0):
    """Per frequency w[i]: 1/Nk sum_k log|det(V(k) G(i w[i]) - 1)| on the k grid nk
    (see qed_sef_integrand_grid). V0: k-independent part of V (dim x dim);
    (r, c, R, v): inter-cluster elements, R in superlattice coordinates."""
    V0 = np.asfortranarray(V0, dtype=np.complex128)
    dim = V0.shape[0]
    n = len(r)
    ri = np.ascontiguousarray(r, dtype=np.int32)
    ci = np.ascontiguousarray(c, dtype=np.int32)
    Ri = np.ascontiguousarray(np.reshape(R, (-1, 3)), dtype=np.int32) if n else np.zeros((1, 3), np.int32)
    vv = np.ascontiguousarray(v, dtype=np.complex128) if n else np.zeros(1, np.complex128)
    ww = np.ascontiguousarray(w, dtype=np.float64)
    nk = tuple(int(x) for x in nk) + (1,) * (3 - len(tuple(nk)))
    out = np.zeros(len(ww))
    v0 = V0.ravel(order="F").view(np.float64)
    _check(lib().qed_sef_integrand_grid(label, int(spin_down), dim, _dp(v0), n, _ip(ri if n else np.zeros(1, np.int32)),
                                        _ip(ci if n else np.zeros(1, np.int32)), _ip(Ri), _dp(vv.view(np.float64)),
                                        len(ww), _dp(ww), nk[0], nk[1], nk[2], _dp(out)))
    return out


def cpt_projected_green_function(V0, r, c, R, v, w, nk, offset=0.5, spin_down: bool = False, label: int = 0):
    """Per frequency w[i]: grid average of G (1 - V(k) G)^{-1} (see
    qed_cpt_projected_green_function); V0: (nw, dim, dim) k-independent parts."""
    V0 = np.asarray(V0, dtype=np.complex128)
    nw, dim = V0.shape[0], V0.shape[1]
    v0 = np.ascontiguousarray(np.transpose(V0, (0, 2, 1))).view(np.float64)  # column-major blocks
    n = len(r)
    ri = np.ascontiguousarray(r if n else [0], dtype=np.int32)
    ci = np.ascontiguousarray(c if n else [0], dtype=np.int32)
    Ri = np.ascontiguousarray(np.reshape(R, (-1, 3)) if n else np.zeros((1, 3)), dtype=np.int32)
    vv = np.ascontiguousarray(v if n else [0.0], dtype=np.complex128)
    ww = np.ascontiguousarray(w, dtype=np.float64)
    nk = tuple(int(x) for x in nk) + (1,) * (3 - len(tuple(nk)))
    out = np.zeros(2 * dim * dim * nw)
    _check(lib().qed_cpt_projected_green_function(label, int(spin_down), dim, _dp(v0), n, _ip(ri), _ip(ci), _ip(Ri),
                                                  _dp(vv.view(np.float64)), nw, _dp(ww), nk[0], nk[1], nk[2],
                                                  float(offset), _dp(out)))
    return (out[0::2] + 1j * out[1::2]).reshape(nw, dim, dim).transpose(0, 2, 1)


def qmatrix(spin_down: bool = False, label: int = 0, capacity: int = 1 << 16):
    """Lehmann representation: (poles e[M], residues V as an L x M complex matrix)."""
    M = C.c_int(capacity)
    L = C.c_int(0)
    n = Green_function_dimension(label)
    e = np.zeros(capacity)
    v = np.zeros((capacity * n, 2))
    _check(lib().qed_qmatrix(label, int(spin_down), C.byref(M), C.byref(L), _dp(e), _dp(v)))
    m, l = M.value, L.value
    vv = (v[: m * l, 0] + 1j * v[: m * l, 1]).reshape(m, l).T
    return e[:m].copy(), vv.copy()


def cf_coefficients(o1: int, o2: int, pm: int, spin_down: bool = False, label: int = 0, capacity=4096):
    n = C.c_int(capacity)
    a = np.zeros(capacity)
    b = np.zeros(capacity)
    _check(lib().qed_cf_coefficients(label, int(spin_down), o1, o2, pm, C.byref(n), _dp(a), _dp(b)))
    return a[: n.value].copy(), b[: n.value].copy()


def ground_state_vector(label: int = 0):
    d = C.c_long()
    _check(lib().qed_ground_state_vector(label, C.byref(d), None))
    psi = np.zeros(d.value)
    _check(lib().qed_ground_state_vector(label, C.byref(d), _dp(psi)))
    return psi


# ---- plugin point and basis -------------------------------------------------

class MixedHamiltonian:
    """Device Hamiltonian of one sector of a model with point-group generators, in
    the symmetry-adapted basis (the reference's CSR format over ED_mixed_basis)."""

    def __init__(self, label: int, sector: str):
        h = C.c_void_p()
        d = C.c_long()
        _check(lib().qed_mixed_hamiltonian_create(label, sector.encode(), C.byref(h), C.byref(d)))
        self.h = h
        self.dim = d.value

    def states(self):
        out = np.zeros(self.dim, dtype=np.uint64)
        _check(lib().qed_mixed_hamiltonian_states(self.h, out.ctypes.data_as(C.POINTER(C.c_uint64))))
        return out

    @property
    def nnz(self) -> int:
        n = C.c_long()
        _check(lib().qed_mixed_hamiltonian_nnz(self.h, C.byref(n)))
        return n.value

    def mult_add(self, x, y):
        """y += H x (host float64 arrays)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert y.dtype == np.float64 and y.flags.c_contiguous and len(y) == self.dim
        _check(lib().qed_mixed_hamiltonian_mult_add(self.h, _dp(x), _dp(y)))

    def ground_state_energy(self):
        """(lowest eigenvalue, Lanczos iterations) of the sector."""
        e = C.c_double()
        it = C.c_int()
        _check(lib().qed_mixed_hamiltonian_ground_state(self.h, C.byref(e), C.byref(it)))
        return e.value, it.value

    def ground_state(self):
        """(lowest eigenvalue, its eigenvector in the order of states())."""
        e = C.c_double()
        psi = np.zeros(self.dim)
        _check(lib().qed_mixed_hamiltonian_ground_state_vector(self.h, C.byref(e), _dp(psi)))
        return e.value, psi

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.qed_mixed_hamiltonian_destroy(self.h)
            self.h = None


class Hamiltonian:
    """Device Hamiltonian of one sector (Hamiltonian<double> plugin point)."""

    def __init__(self, label: int, sector: str):
        h = C.c_void_p()
        d = C.c_long()
        _check(lib().qed_hamiltonian_create(label, sector.encode(), C.byref(h), C.byref(d)))
        self._h = h
        self.dim = d.value

    def mult_add(self, x, y):
        """y += H x on host arrays (Hamiltonian::mult_add)."""
        x = np.ascontiguousarray(x, dtype=np.float64)
        if not (y.dtype == np.float64 and y.flags.c_contiguous and y.size == self.dim):
            raise ValueError("y must be a contiguous float64 array of the sector dimension")
        _check(lib().qed_hamiltonian_mult_add(self._h, _dp(x), _dp(y)))

    def apply_device(self, x_ptr: int, y_ptr: int, stream: int = 0):
        """y = H x on device pointers (e.g. torch tensors' data_ptr()), enqueued on the
        cudaStream_t handle `stream` (0 = legacy default stream, torch's default)."""
        _check(lib().qed_hamiltonian_apply_device(self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr),
                                                  C.c_void_p(stream)))

    def apply_dots_device(self, x_ptr: int, y_ptr: int, dots_ptr: int, stream: int = 0):
        """y = H x and dots = (<x,y>, <y,y>, <x,x>) on device pointers, in one pass."""
        _check(lib().qed_hamiltonian_apply_dots_device(self._h, C.c_void_p(x_ptr), C.c_void_p(y_ptr),
                                                       C.c_void_p(dots_ptr), C.c_void_p(stream)))

    def diag(self):
        d = np.zeros(self.dim)
        _check(lib().qed_hamiltonian_diag(self._h, _dp(d)))
        return d

    def close(self):
        if getattr(self, "_h", None):
            lib().qed_hamiltonian_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def halfbasis(L: int, N: int):
    d = C.c_long()
    _check(lib().qed_halfbasis(L, N, None, C.byref(d)))
    out = np.zeros(d.value, dtype=np.uint32)
    _check(lib().qed_halfbasis(L, N, out.ctypes.data_as(C.POINTER(C.c_uint)), C.byref(d)))
    return out


def halfbasis_rank(L: int, N: int, strings):
    s = np.ascontiguousarray(strings, dtype=np.uint32)
    r = np.zeros(len(s), dtype=np.uint32)
    _check(lib().qed_halfbasis_rank(L, N, len(s), s.ctypes.data_as(C.POINTER(C.c_uint)),
                                    r.ctypes.data_as(C.POINTER(C.c_uint))))
    return r


def _generators_abi(n_sites, n_bath, generators, bath_irrep):
    """pyqcm's generators (1-based sites; bath entries 1-based orbitals, or irrep
    phases with bath_irrep) -> ED::new_model's 0-based rows, as the reference's
    Python binding converts them (src_python/qcm_ED_wrap.hpp:145-163)."""
    n_orb = n_sites + n_bath
    rows = [list(map(int, g)) for g in (generators or [])]
    for j, g in enumerate(rows):
        if len(g) != n_orb:
            raise QEDError(1, f"generator {j + 1} should have {n_orb} elements")
        for i in range(n_orb):
            if i < n_sites or not bath_irrep:
                g[i] -= 1
    flat = np.ascontiguousarray(np.array(rows, dtype=np.int32).reshape(-1))
    return len(rows), flat


def symmetry_group(n_sites: int, n_bath: int = 0, generators=None, bath_irrep: bool = False):
    """The cluster point group of pyqcm's generators: dict with the order g, the
    character phases phi (g x g, units of 2 pi / g), the symmetric site orbitals S
    (rows, irreps in order) and site_irrep_dim."""
    ng, flat = _generators_abi(n_sites, n_bath, generators, bath_irrep)
    g = C.c_int()
    phi = np.zeros(256, dtype=np.int32)
    sre = np.zeros(n_sites * n_sites)
    sim = np.zeros(n_sites * n_sites)
    dims = np.zeros(16, dtype=np.int32)
    ip = C.POINTER(C.c_int)
    _check(lib().qed_symmetry_group(n_sites, n_bath, ng, flat.ctypes.data_as(ip), int(bool(bath_irrep)),
                                    C.byref(g), phi.ctypes.data_as(ip), _dp(sre), _dp(sim),
                                    dims.ctypes.data_as(ip)))
    n = g.value
    return {"g": n, "phi": phi[:n * n].reshape(n, n).copy(),
            "S": (sre + 1j * sim).reshape(n_sites, n_sites), "site_irrep_dim": dims[:n].copy()}


def symmetry_representatives(n_sites: int, n_bath: int, generators, bath_irrep: bool, irrep: int, states):
    """symmetry_group::Representative of each 64-bit state (spin up in the low
    word): (representative, phase in units of pi/g, orbit length; 0 = null)."""
    ng, flat = _generators_abi(n_sites, n_bath, generators, bath_irrep)
    st = np.ascontiguousarray(states, dtype=np.uint64)
    rep = np.zeros(len(st), dtype=np.uint64)
    ph = np.zeros(len(st), dtype=np.int32)
    ln = np.zeros(len(st), dtype=np.int32)
    ip = C.POINTER(C.c_int)
    up = C.POINTER(C.c_uint64)
    _check(lib().qed_symmetry_representatives(n_sites, n_bath, ng, flat.ctypes.data_as(ip), int(bool(bath_irrep)),
                                              irrep, len(st), st.ctypes.data_as(up), rep.ctypes.data_as(up),
                                              ph.ctypes.data_as(ip), ln.ctypes.data_as(ip)))
    return rep, ph, ln


def destroy_table(L: int, n_up: int, n_dn: int, a: int):
    from math import comb
    dim = comb(L, n_up) * comb(L, n_dn)
    tgt = np.zeros(dim, dtype=np.int64)
    ph = np.zeros(dim, dtype=np.int32)
    _check(lib().qed_destroy_table(L, n_up, n_dn, a, tgt.ctypes.data_as(C.POINTER(C.c_long)),
                                   ph.ctypes.data_as(C.POINTER(C.c_int))))
    return tgt, ph


def hv_tuning_report():
    """Launch shapes chosen by the H.v autotuner so far (list of dicts: dim_up,
    dim_dn, choice, bit_identical -- every candidate wrote the same bits of
    H x --, ms per candidate)."""
    import json
    n = lib().qed_hv_tuning_report(None, 0)
    buf = C.create_string_buffer(n + 1)
    lib().qed_hv_tuning_report(buf, n + 1)
    return json.loads(buf.value.decode() or "[]")


def window_plan(L: int, N: int, pd, ps, amp, x):
    """The window form of one spin's hop operator applied on the host
    (qed_window_plan): returns (number of windows, y); 0 windows and y = None when
    the pairs pd[q] <- ps[q] do not fit windows of eight consecutive sites."""
    pd = np.ascontiguousarray(pd, dtype=np.int32)
    ps = np.ascontiguousarray(ps, dtype=np.int32)
    amp = np.ascontiguousarray(amp, dtype=np.float64)
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.zeros_like(x)
    nw = C.c_int()
    _check(lib().qed_window_plan(L, N, len(pd), _ip(pd), _ip(ps), _dp(amp), _dp(x), _dp(y), C.byref(nw)))
    return nw.value, (y if nw.value else None)


def window_compile(L: int, n_up: int, n_dn: int, pd, ps):
    """Compiles the window H.v kernels for a sector whose spins hop on pairs
    pd[q] <- ps[q] (NVRTC, no device needed); returns (ok, log with the ptxas
    register and spill lines)."""
    pd = np.ascontiguousarray(pd, dtype=np.int32)
    ps = np.ascontiguousarray(ps, dtype=np.int32)
    buf = C.create_string_buffer(1 << 16)
    ok = C.c_int()
    _check(lib().qed_window_compile(L, n_up, n_dn, len(pd), _ip(pd), _ip(ps), buf, len(buf), C.byref(ok)))
    return bool(ok.value), buf.value.decode(errors="replace")


def spin_table_host(L: int, N: int, t, vsame, bank_order: bool = False) -> dict:
    """One spin's tables as the solver builds them (qed_spin_table_host, host
    only): strings, hop counts, diagonal, ELL entries (rank << 8 | value slot,
    shape (width, dim)) and the value slots."""
    from math import comb
    t = np.ascontiguousarray(t, dtype=np.float64)
    vsame = np.ascontiguousarray(vsame, dtype=np.float64)
    dim = comb(L, N)
    bits = np.zeros(dim, np.uint32)
    cnt = np.zeros(dim, np.uint8)
    diag = np.zeros(dim)
    cap = 256 * dim
    ell = np.zeros(cap, np.uint32)
    vals = np.zeros(258)
    w = C.c_int()
    nv = C.c_int()
    _check(lib().qed_spin_table_host(L, N, _dp(t), _dp(vsame), int(bank_order),
                                     bits.ctypes.data_as(C.POINTER(C.c_uint)), cnt.ctypes.data_as(C.POINTER(C.c_ubyte)),
                                     _dp(diag), ell.ctypes.data_as(C.POINTER(C.c_uint)), cap, C.byref(w),
                                     _dp(vals), C.byref(nv)))
    return {"bits": bits, "cnt": cnt, "diag": diag, "ell": ell[:w.value * dim].reshape(w.value, dim),
            "vals": vals[:nv.value], "width": w.value}


def window_launches() -> int:
    """H.v calls that ran the window kernels so far in this process."""
    n = C.c_longlong()
    _check(lib().qed_window_launches(C.byref(n)))
    return n.value


# ------------------------------------------------------------ instance checkpoints --

_GF_FORMATS = ("bl", "cf", "mcf")


def write_instance_to_hdf5(filename: str, group: str, label: int = 0):
    """qcm.write_instance_to_hdf5 (src_python/qcm_ED_wrap.hpp:364-369 -> ED::write_instance_hdf5,
    src_ed/qcm_ED.cpp:373-389): solves the instance's Green function if needed and
    writes it to `group` of the HDF5 file (created if absent, the group replaced if
    present) in the reference's layout: attributes GS_energy, GS_sectors, GF_format,
    mixing, complex_HS, nstates; group params; one group state_i per state (sec,
    energy, weight, gf_format; gf and, with spin asymmetry, gf_down holding a
    Q-matrix set or a continued-fraction set). The file is written by
    pyqcm_b200.hdf5 (no HDF5 library needed)."""
    from . import hdf5
    L = lib()
    n, e0, fmt, mix = C.c_int(), C.c_double(), C.c_int(), C.c_int()
    gs = C.create_string_buffer(4096)
    _check(L.qed_instance_states(label, C.byref(n), C.byref(e0), gs, 4096, C.byref(fmt), C.byref(mix)))
    cap, npar = 4096, C.c_int()
    names = C.create_string_buffer(1 << 16)
    vals = np.zeros(cap)
    _check(L.qed_instance_parameters(label, cap, C.byref(npar), names, 1 << 16, _dp(vals)))
    pnames = names.value.decode().split("\n")[:npar.value]
    nsites = Green_function_dimension(label)
    f = hdf5.File(filename, "a")
    f.root.unlink(group)
    g = f.root.create_group(group)
    g.attrs.update({"GS_energy": e0.value, "GS_sectors": gs.value.decode(), "GF_format": _GF_FORMATS[fmt.value],
                    "mixing": mix.value, "complex_HS": 0})
    pg = g.create_group("params")
    for k, v in zip(pnames, vals):
        pg.attrs[k] = float(v)
    g.attrs["nstates"] = n.value
    for i in range(n.value):
        sec = C.create_string_buffer(256)
        en, w = C.c_double(), C.c_double()
        _check(L.qed_instance_state(label, i, sec, 256, C.byref(en), C.byref(w)))
        sg = g.create_group(f"state_{i}")
        sg.attrs.update({"sec": sec.value.decode(), "energy": en.value, "weight": w.value,
                         "gf_format": _GF_FORMATS[fmt.value]})
        for sd in ((0, 1) if mix.value & 4 else (0,)):
            gg = sg.create_group("gf_down" if sd else "gf")
            if fmt.value == 0:  # Q_matrix_set::write_hdf5 (src_ed/Q_matrix_set.hpp:187-194), one block
                Lr, M = C.c_int(), C.c_int()
                _check(L.qed_instance_state_qmatrix(label, i, sd, 0, C.byref(Lr), C.byref(M), None, None))
                e = np.zeros(M.value)
                v = np.zeros(Lr.value * M.value)
                _check(L.qed_instance_state_qmatrix(label, i, sd, M.value, C.byref(Lr), C.byref(M), _dp(e), _dp(v)))
                gg.attrs["nblocks"] = 1
                bg = gg.create_group("block_0")
                bg.attrs.update({"L": Lr.value, "M": M.value})
                bg.create_dataset("e", e)
                vg = bg.create_group("v")
                vg.attrs.update({"r": Lr.value, "c": M.value})
                vg.create_dataset("data", v)
            else:  # continued_fraction_set::write_hdf5 (src_ed/continued_fraction_set.cpp:136-153)
                gg.attrs["is_complex"] = 0
                for a in range(nsites):
                    for b in range(a + 1):
                        cg = gg.create_group(f"r0_a{a}_b{b}")
                        for part, pm in (("e", 1), ("h", -1)):
                            nl = C.c_int()
                            _check(L.qed_instance_state_cf(label, i, sd, a, b, pm, 0, C.byref(nl), None, None))
                            ca, cb = np.zeros(nl.value), np.zeros(nl.value)
                            _check(L.qed_instance_state_cf(label, i, sd, a, b, pm, nl.value, C.byref(nl), _dp(ca),
                                                           _dp(cb)))
                            pgp = cg.create_group(part)
                            pgp.create_dataset("a", ca)
                            pgp.create_dataset("b", cb)
    f.close()


def read_instance_from_hdf5(filename: str, group: str, label: int = 0):
    """qcm.read_instance_from_hdf5 (src_python/qcm_ED_wrap.hpp:371-376 -> ED::read_instance_hdf5,
    src_ed/qcm_ED.cpp:392-403, model_instance::read_hdf5): replaces the states of
    instance `label` by those of `group`, which then counts as solved (Green
    function, its average and density from the file). As the reference does, a
    parameter value in the file that differs from the instance's by more than
    1e-4 only prints a warning."""
    from . import hdf5
    L = lib()
    g = hdf5.File(filename, "r").root.group(group)
    fmt = _GF_FORMATS.index(g.attrs["GF_format"])
    mix = int(g.attrs["mixing"])
    cap, npar = 4096, C.c_int()
    names = C.create_string_buffer(1 << 16)
    vals = np.zeros(cap)
    _check(L.qed_instance_parameters(label, cap, C.byref(npar), names, 1 << 16, _dp(vals)))
    current = dict(zip(names.value.decode().split("\n")[:npar.value], vals))
    stored = g.group("params").attrs if "params" in g else {}
    for k, v in current.items():
        if k in stored and abs(float(stored[k]) - v) > 1e-4:
            print(f"WARNING : The value of {k} from the HDF5 solution ({stored[k]}) differs from the expected "
                  f"value ({v}).")
    nsites = Green_function_dimension(label)
    _check(L.qed_instance_load_begin(label, float(g.attrs["GS_energy"]), fmt, mix))
    for i in range(int(g.attrs["nstates"])):
        sg = g.group(f"state_{i}")
        idx = C.c_int()
        _check(L.qed_instance_load_state(label, sg.attrs["sec"].encode(), float(sg.attrs["energy"]),
                                         float(sg.attrs["weight"]), C.byref(idx)))
        for sd, gname in ((0, "gf"), (1, "gf_down")):
            if gname not in sg:
                continue
            gg = sg.group(gname)
            if fmt == 0:
                if int(gg.attrs["nblocks"]) != 1:
                    raise QEDError(QED_ERR_UNSUPPORTED, "Q-matrix sets of more than one block (point groups)")
                bg = gg.group("block_0")
                e = np.ascontiguousarray(bg.dataset("e"), dtype=np.float64)
                v = np.ascontiguousarray(bg.group("v").dataset("data"), dtype=np.float64)
                _check(L.qed_instance_load_qmatrix(label, idx.value, sd, int(bg.attrs["L"]), int(bg.attrs["M"]),
                                                   _dp(e), _dp(v)))
            else:
                for a in range(nsites):
                    for b in range(a + 1):
                        cg = gg.group(f"r0_a{a}_b{b}")
                        for part, pm in (("e", 1), ("h", -1)):
                            ca = np.ascontiguousarray(cg.group(part).dataset("a"), dtype=np.float64)
                            cb = np.ascontiguousarray(cg.group(part).dataset("b"), dtype=np.float64)
                            _check(L.qed_instance_load_cf(label, idx.value, sd, a, b, pm, len(ca), _dp(ca), _dp(cb)))
    _check(L.qed_instance_load_end(label))
