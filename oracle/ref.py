"""CPU oracle: ctypes access to the reference's own ED library.

TEST INFRASTRUCTURE ONLY -- imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference arm, never by the product package.

The library (oracle/_ref/libqcm_ed_ref.so) is the reference's src_ed + src_util
compiled from its sources by oracle/ref_build/Makefile, with the flat C layer
oracle/ref_build/ref_capi.cpp on top of namespace ED (src_ed/qcm_ED.hpp:23-340).
The reference keeps its models and instances in process-global maps
(src_ed/qcm_ED.cpp:25-26), so one process holds one oracle state; tests that
need a clean slate use fresh model names / instance labels.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libqcm_ed_ref.so")

_lib = None


class OracleError(RuntimeError):
    pass


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise OracleError(f"oracle library not built: {LIB_PATH} (run make -C oracle/ref_build)")
        # RTLD_DEEPBIND: resolve the oracle's LAPACK/BLAS calls in its own
        # OpenBLAS, not in libraries already loaded into the process (torch's
        # libtorch_cpu exports an incompatible zgetrf_, for instance).
        L = C.CDLL(LIB_PATH, mode=os.RTLD_LOCAL | os.RTLD_DEEPBIND)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        lp = C.POINTER(C.c_long)
        sig = {
            "ref_last_error": [C.c_char_p, C.c_int],
            "ref_init": [],
            "ref_set_int": [C.c_char_p, C.c_long],
            "ref_set_double": [C.c_char_p, C.c_double],
            "ref_set_char": [C.c_char_p, C.c_char],
            "ref_set_bool": [C.c_char_p, C.c_int],
            "ref_new_model": [C.c_char_p, C.c_int, C.c_int],
            "ref_new_model_gen": [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_int],
            "ref_symmetry_group": [C.c_int, C.c_int, C.c_int, ip, C.c_int, ip, ip, dp, dp, ip],
            "ref_representatives": [C.c_int, C.c_int, C.c_int, ip, C.c_int, C.c_int, C.c_long,
                                    C.POINTER(C.c_uint64), C.POINTER(C.c_uint64), ip, ip],
            "ref_mixed_basis": [C.c_int, C.c_int, C.c_int, ip, C.c_int, C.c_char_p, C.POINTER(C.c_uint64), lp],
            "ref_new_operator": [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int, ip, ip, dp],
            "ref_new_instance": [C.c_char_p, C.c_int, C.POINTER(C.c_char_p), dp, C.c_char_p, C.c_int, C.c_char],
            "ref_erase_instance": [C.c_int],
            "ref_ground_state": [C.c_int, dp, C.c_char_p, C.c_int],
            "ref_green_solve": [C.c_int],
            "ref_gf_dim": [C.c_int],
            "ref_mixing": [C.c_int],
            "ref_green_function": [C.c_int, C.c_int, C.c_int, dp, dp],
            "ref_self_energy": [C.c_int, C.c_int, C.c_int, dp, dp],
            "ref_hybridization_function": [C.c_int, C.c_int, C.c_int, dp, dp],
            "ref_green_function_average": [C.c_int, C.c_int, dp],
            "ref_potthoff": [C.c_int, dp],
            "ref_qmatrix": [C.c_int, C.c_int, ip, ip, dp, dp],
            "ref_cf_coeffs": [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, ip, dp, dp],
            "ref_gs_vector": [C.c_int, lp, dp, dp],
            "ref_halfbasis": [C.c_int, C.c_int, C.POINTER(C.c_uint), lp],
            "ref_destroy_table": [C.c_int, C.c_int, C.c_int, C.c_int, lp, ip],
            "ref_hv_apply": [C.c_void_p, dp, dp],
            "ref_hv_bench": [C.c_void_p, C.c_int, dp],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        cpp = C.POINTER(C.c_char_p)
        sig.update({
            "ref_qcm_great_reset": [],
            "ref_qcm_add_cluster": [lp, C.c_int, lp, C.c_int, C.c_int],
            "ref_qcm_add_system": [C.c_char_p, C.c_int],
            "ref_qcm_lattice_model": [C.c_char_p, C.c_int, lp, lp],
            "ref_qcm_hopping_operator": [C.c_char_p, lp, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int],
            "ref_qcm_interaction_operator": [C.c_char_p, lp, C.c_double, C.c_int, C.c_int, C.c_char_p],
            "ref_qcm_density_wave": [C.c_char_p, C.c_char_p, dp, lp, C.c_double, C.c_int, C.c_double],
            "ref_qcm_set_target_sectors": [C.c_int, cpp],
            "ref_qcm_set_parameters": [C.c_int, cpp, dp, C.c_int, cpp, dp, cpp],
            "ref_qcm_set_parameter": [C.c_char_p, C.c_double],
            "ref_qcm_new_model_instance": [C.c_int],
            "ref_qcm_erase_instance": [C.c_int],
            "ref_qcm_dims": [ip, ip, ip],
            "ref_qcm_set_wavevector_grid": [C.c_int, C.c_int, C.c_int],
            "ref_qcm_frequency_grid": [C.c_int, dp, dp],
            "ref_qcm_potthoff": [C.c_int, dp],
            "ref_qcm_cluster_hopping": [C.c_int, C.c_int, C.c_int, ip, dp],
            "ref_qcm_V_superdual": [C.c_int, C.c_int, C.c_double, C.c_double, dp, ip, dp],
            "ref_qcm_cluster_gf": [C.c_int, C.c_int, C.c_double, C.c_double, ip, dp],
            "ref_qcm_ed_label": [C.c_int, C.c_int],
            "ref_qcm_cdmft_variational_set": [C.c_int, cpp],
            "ref_qcm_cdmft_host": [C.c_int, C.c_int, dp, dp],
            "ref_qcm_get_cdmft_host": [C.c_int, C.c_int, C.c_int, C.c_int, ip, dp],
            "ref_qcm_cdmft_distance": [C.c_int, C.c_int, dp, C.c_int, dp],
        })
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        L.ref_hv_create.argtypes = [C.c_int, C.c_char_p, lp]
        L.ref_hv_create.restype = C.c_void_p
        L.ref_hv_create_csr.argtypes = [C.c_int, C.c_char_p, lp]
        L.ref_hv_create_csr.restype = C.c_void_p
        L.ref_hv_destroy.argtypes = [C.c_void_p]
        L.ref_hv_destroy.restype = None
        if L.ref_init() != 0:
            raise OracleError("ref_init failed")
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        buf = C.create_string_buffer(4096)
        lib().ref_last_error(buf, 4096)
        raise OracleError(buf.value.decode())


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def set_param(name: str, value):
    L = lib()
    n = name.encode()
    if isinstance(value, bool):
        _check(L.ref_set_bool(n, int(value)))
    elif isinstance(value, int):
        _check(L.ref_set_int(n, value))
    elif isinstance(value, float):
        _check(L.ref_set_double(n, value))
    elif isinstance(value, str) and len(value) == 1:
        _check(L.ref_set_char(n, value.encode()))
    else:
        raise TypeError(value)


def new_model(name, n_sites, n_bath, generators=None, bath_irrep=False):
    """generators: pyqcm's form (1-based sites; see ref_new_model_gen)."""
    if not generators:
        _check(lib().ref_new_model(name.encode(), n_sites, n_bath))
        return
    flat = [int(v) for row in generators for v in row]
    arr = (C.c_int * len(flat))(*flat)
    _check(lib().ref_new_model_gen(name.encode(), n_sites, n_bath, len(generators), arr, int(bath_irrep)))


def new_operator(model, op, typ, elements):
    n = len(elements)
    r = (C.c_int * n)(*[int(e[0]) for e in elements])
    c = (C.c_int * n)(*[int(e[1]) for e in elements])
    v = (C.c_double * n)(*[float(e[2]) for e in elements])
    _check(lib().ref_new_operator(model.encode(), op.encode(), typ.encode(), n, r, c, v))


def new_instance(model, params: dict, sectors: str, label: int, fmt: str = "F"):
    """fmt: Hamiltonian_format of this instance ('F' factorized, 'S' CSR)."""
    names = list(params)
    arr = (C.c_char_p * len(names))(*[k.encode() for k in names])
    vals = (C.c_double * len(names))(*[float(params[k]) for k in names])
    _check(lib().ref_new_instance(model.encode(), len(names), arr, vals, sectors.encode(), label,
                                  fmt.encode()))


def load_problem(prob, label: int, model_name: str | None = None, fmt: str = "F"):
    """Defines model + operators (once per model name) and an instance.

    The reference's continued-fraction builder dereferences the Hamiltonian's
    mixed basis, which its factorized format never sets
    (src_ed/model_instance.cpp:52 with Hamiltonian_Factorized); use fmt='S'
    for GF_method 'F'."""
    mname = model_name or prob.name
    new_model(mname, prob.n_sites, prob.n_bath, getattr(prob, "generators", None),
              getattr(prob, "bath_irrep", False))
    for op, (typ, el) in prob.operators.items():
        new_operator(mname, op, typ, el)
    new_instance(mname, prob.params, prob.sectors, label, fmt)


def ground_state(label):
    E = C.c_double()
    buf = C.create_string_buffer(256)
    _check(lib().ref_ground_state(label, C.byref(E), buf, 256))
    return E.value, buf.value.decode()


def green_solve(label):
    _check(lib().ref_green_solve(label))


def gf_dim(label):
    return lib().ref_gf_dim(label)


def mixing(label):
    return lib().ref_mixing(label)


def _zcall(fn, label, z, spin_down, n):
    z = np.ascontiguousarray(np.atleast_1d(np.asarray(z, dtype=np.complex128)))
    out = np.zeros((len(z), n, n), dtype=np.complex128)
    _check(fn(label, int(spin_down), len(z), _dp(z.view(np.float64)), _dp(out.view(np.float64))))
    # column-major n x n blocks -> [k, row, col]
    return out.transpose(0, 2, 1).copy()


def green_function(label, z, spin_down=False):
    return _zcall(lib().ref_green_function, label, z, spin_down, gf_dim(label))


def self_energy(label, z, spin_down=False):
    return _zcall(lib().ref_self_energy, label, z, spin_down, gf_dim(label))


def hybridization_function(label, z, spin_down=False):
    return _zcall(lib().ref_hybridization_function, label, z, spin_down, gf_dim(label))


def green_function_average(label, spin_down=False):
    d = C.c_int()
    _check(lib().ref_green_function_average_dim(label, int(spin_down), C.byref(d)))
    n = d.value
    out = np.zeros((n, n), dtype=np.complex128)
    _check(lib().ref_green_function_average(label, int(spin_down), _dp(out.view(np.float64))))
    return out.T.copy()


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def model_size(model):
    a, b, c = C.c_int(), C.c_int(), C.c_int()
    _check(lib().ref_model_size(model.encode(), C.byref(a), C.byref(b), C.byref(c)))
    return a.value, b.value, c.value


def exists(model, op):
    f = C.c_int()
    _check(lib().ref_exists(model.encode(), op.encode(), C.byref(f)))
    return bool(f.value)


def matrix_elements(model, op):
    cap = 1 << 14
    r, c, v = np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros(cap)
    n = C.c_int()
    t = C.create_string_buffer(64)
    _check(lib().ref_matrix_elements(model.encode(), op.encode(), t, len(t), cap, C.byref(n), _ip(r), _ip(c), _dp(v)))
    return t.value.decode(), [(int(r[i]), int(c[i]), float(v[i])) for i in range(n.value)]


def gf_density(label):
    d = C.c_double()
    _check(lib().ref_gf_density(label, C.byref(d)))
    return d.value


def _square(fn, *args):
    d = C.c_int()
    _check(fn(*args, C.byref(d), None))
    buf = np.zeros(2 * d.value * d.value)
    _check(fn(*args, C.byref(d), _dp(buf)))
    return (buf[0::2] + 1j * buf[1::2]).reshape(d.value, d.value).T.copy()


def hopping_matrix(label, spin_down=False):
    return _square(lib().ref_hopping_matrix, label, int(spin_down))


def hopping_matrix_full(label, spin_down=False, diag=False):
    return _square(lib().ref_hopping_matrix_full, label, int(spin_down), int(diag))


def interactions(label):
    cap = 1 << 14
    r, c, v = np.zeros(cap, np.int32), np.zeros(cap, np.int32), np.zeros(cap)
    n = C.c_int()
    _check(lib().ref_interactions(label, cap, C.byref(n), _ip(r), _ip(c), _dp(v)))
    return [(int(r[i]), int(c[i]), float(v[i])) for i in range(n.value)]


def tr_sigma_inf(label):
    d = C.c_double()
    _check(lib().ref_tr_sigma_inf(label, C.byref(d)))
    return d.value


def susceptibility(label, op, w):
    w = np.ascontiguousarray(np.atleast_1d(np.asarray(w, dtype=np.complex128)))
    chi = np.zeros(len(w), dtype=np.complex128)
    _check(lib().ref_susceptibility(label, op.encode(), len(w), _dp(w.view(np.float64)), _dp(chi.view(np.float64))))
    return chi


def susceptibility_poles(label, op):
    cap = 1 << 14
    e, r = np.zeros(cap), np.zeros(cap)
    n = C.c_int()
    _check(lib().ref_susceptibility_poles(label, op.encode(), cap, C.byref(n), _dp(e), _dp(r)))
    return [(float(e[i]), float(r[i])) for i in range(n.value)]


def fidelity(l1, l2):
    d = C.c_double()
    _check(lib().ref_fidelity(l1, l2, C.byref(d)))
    return d.value


def cluster_averages(label):
    """ED::cluster_averages: [(operator name, average, variance), ...]."""
    cap = 256
    n = C.c_int(0)
    ave = np.zeros(cap)
    var = np.zeros(cap)
    buf = C.create_string_buffer(1 << 16)
    _check(lib().ref_cluster_averages(label, cap, C.byref(n), _dp(ave), _dp(var), buf, len(buf)))
    names = buf.value.decode().split("\n")[: n.value]
    return [(names[i], float(ave[i]), float(var[i])) for i in range(n.value)]


def potthoff(label):
    w = C.c_double()
    _check(lib().ref_potthoff(label, C.byref(w)))
    return w.value


def qmatrix(label, spin_down=False, capacity=1 << 16):
    M = C.c_int(capacity)
    L = C.c_int(0)
    e = np.zeros(capacity)
    v = np.zeros((capacity * 64, 2))
    _check(lib().ref_qmatrix(label, int(spin_down), C.byref(M), C.byref(L), _dp(e), _dp(v)))
    m, l = M.value, L.value
    vv = (v[: m * l, 0] + 1j * v[: m * l, 1]).reshape(m, l).T  # column-major L x M
    return e[:m].copy(), vv.copy()


def cf_coeffs(label, o1, o2, pm, spin_down=False, capacity=4096):
    n = C.c_int(capacity)
    a = np.zeros(capacity)
    b = np.zeros(capacity)
    _check(lib().ref_cf_coeffs(label, int(spin_down), o1, o2, pm, C.byref(n), _dp(a), _dp(b)))
    return a[: n.value].copy(), b[: n.value].copy()


def gs_vector(label):
    d = C.c_long()
    E = C.c_double()
    _check(lib().ref_gs_vector(label, C.byref(d), C.byref(E), None))
    psi = np.zeros(d.value)
    _check(lib().ref_gs_vector(label, C.byref(d), C.byref(E), _dp(psi)))
    return E.value, psi


def halfbasis(L, N):
    d = C.c_long()
    _check(lib().ref_halfbasis(L, N, None, C.byref(d)))
    out = np.zeros(d.value, dtype=np.uint32)
    _check(lib().ref_halfbasis(L, N, out.ctypes.data_as(C.POINTER(C.c_uint)), C.byref(d)))
    return out


def destroy_table(L, n_up, n_dn, a):
    dim = len(halfbasis(L, n_up)) * len(halfbasis(L, n_dn))
    tgt = np.zeros(dim, dtype=np.int64)
    ph = np.zeros(dim, dtype=np.int32)
    _check(lib().ref_destroy_table(L, n_up, n_dn, a, tgt.ctypes.data_as(C.POINTER(C.c_long)),
                                   ph.ctypes.data_as(C.POINTER(C.c_int))))
    return tgt, ph


class RefHamiltonian:
    """y += H x through the reference's factorized Hamiltonian, for one sector
    (csr=True: its CSR Hamiltonian, in the symmetry-adapted basis of a model with
    generators)."""

    def __init__(self, label, sector: str, csr: bool = False):
        d = C.c_long()
        fn = lib().ref_hv_create_csr if csr else lib().ref_hv_create
        self.h = fn(label, sector.encode(), C.byref(d))
        if not self.h:
            _check(1)
        self.dim = d.value

    def mult_add(self, x, y):
        x = np.ascontiguousarray(x, dtype=np.float64)
        assert y.dtype == np.float64 and y.flags.c_contiguous
        _check(lib().ref_hv_apply(self.h, _dp(x), _dp(y)))

    def bench(self, reps):
        s = C.c_double()
        _check(lib().ref_hv_bench(self.h, reps, C.byref(s)))
        return s.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().ref_hv_destroy(self.h)
            self.h = None


# ------------------------------------------------------------ lattice layer --
# The reference's lattice layer (namespace QCM, src_qcm) holds ONE lattice model
# per process (src_qcm/QCM.cpp:34); load_lattice starts from QCM::great_reset,
# which also clears the ED models and instances (src_qcm/QCM.cpp:81-92).

def _strs(xs):
    return (C.c_char_p * max(1, len(xs)))(*[x.encode() for x in xs])


def _longs(xs):
    xs = [int(v) for v in xs]
    return (C.c_long * max(1, len(xs)))(*xs)


def load_lattice(prob, label: int = 0, cluster_name: str = "clus"):
    """Builds `prob` (a workloads.LatticeProblem) the way pyqcm does
    (cluster_model -> cluster -> lattice_model -> operators -> set_target_sectors
    -> set_parameters, pyqcm/__init__.py:107-600) and creates instance `label`."""
    L = lib()
    _check(L.ref_qcm_great_reset())
    new_model(cluster_name, prob.n_sites, getattr(prob, "n_bath", 0))
    for op, (typ, el) in getattr(prob, "cluster_operators", {}).items():
        new_operator(cluster_name, op, typ, el)
    pos = [c for s in prob.sites for c in s]
    _check(L.ref_qcm_add_cluster(_longs([0, 0, 0]), prob.n_sites, _longs(pos), -1, 0))
    _check(L.ref_qcm_add_system(cluster_name.encode(), 0))
    sl = [c for v in prob.superlattice for c in v]
    _check(L.ref_qcm_lattice_model(prob.name.encode(), len(prob.superlattice), _longs(sl), None))
    for name in prob.interactions:
        _check(L.ref_qcm_interaction_operator(name.encode(), None, 1.0, 1, 1, b"Hubbard"))
    for name, link, amp in prob.hoppings:
        _check(L.ref_qcm_hopping_operator(name.encode(), _longs(link), float(amp), 1, 1, 1, 0))
    for name, typ, Q in prob.density_waves:
        q = np.asarray(Q, dtype=np.float64)
        _check(L.ref_qcm_density_wave(name.encode(), typ.encode(), _dp(q), None, 1.0, 0, 0.0))
    _check(L.ref_qcm_set_target_sectors(1, _strs([prob.sectors])))
    names = list(prob.params)
    vals = np.array([prob.params[k] for k in names], dtype=np.float64)
    en = [e[0] for e in prob.equiv]
    em = np.array([e[1] for e in prob.equiv] or [0.0], dtype=np.float64)
    er = [e[2] for e in prob.equiv]
    _check(L.ref_qcm_set_parameters(len(names), _strs(names), _dp(vals), len(en), _strs(en), _dp(em), _strs(er)))
    _check(L.ref_qcm_new_model_instance(label))


def lattice_new_instance(label: int, **values):
    """Sets independent parameters, then creates lattice instance `label`."""
    for k, v in values.items():
        _check(lib().ref_qcm_set_parameter(k.encode(), float(v)))
    _check(lib().ref_qcm_new_model_instance(label))


def lattice_dims():
    m, d, n = C.c_int(), C.c_int(), C.c_int()
    _check(lib().ref_qcm_dims(C.byref(m), C.byref(d), C.byref(n)))
    return m.value, d.value, n.value


def set_grids(freqs, weights, nk):
    f = np.ascontiguousarray(freqs, dtype=np.float64)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    _check(lib().ref_qcm_frequency_grid(len(f), _dp(f), _dp(w)))
    nk = tuple(nk) + (1,) * (3 - len(tuple(nk)))
    _check(lib().ref_qcm_set_wavevector_grid(*[int(v) for v in nk]))


def lattice_potthoff(label: int) -> float:
    om = C.c_double()
    _check(lib().ref_qcm_potthoff(label, C.byref(om)))
    return om.value


def _cmat(fn, *args):
    d = C.c_int()
    _check(fn(*args, C.byref(d), None))
    out = np.zeros(2 * d.value * d.value)
    _check(fn(*args, C.byref(d), _dp(out)))
    n = d.value
    return (out[0::2] + 1j * out[1::2]).reshape(n, n, order="F")


def lattice_cluster_hopping(label: int, spin_down=False, clus=0):
    return _cmat(lib().ref_qcm_cluster_hopping, label, clus, int(spin_down))


def lattice_V(label: int, w: complex, k, spin_down=False):
    """V(k) at frequency w for k in the superdual basis (fractions of the reduced zone)."""
    kk = np.zeros(3)
    kk[:len(k)] = k
    return _cmat(lib().ref_qcm_V_superdual, label, int(spin_down), w.real, w.imag, _dp(kk))


def lattice_cluster_gf(label: int, w: complex, spin_down=False):
    return _cmat(lib().ref_qcm_cluster_gf, label, int(spin_down), w.real, w.imag)


def lattice_ed_label(label: int, s: int = 0) -> int:
    return lib().ref_qcm_ed_label(label, s)


def cdmft_variational_set(names):
    _check(lib().ref_qcm_cdmft_variational_set(len(names), _strs(names)))


def cdmft_host(label, freqs, weights):
    f = np.ascontiguousarray(freqs, dtype=np.float64)
    w = np.ascontiguousarray(weights, dtype=np.float64)
    _check(lib().ref_qcm_cdmft_host(label, len(f), _dp(f), _dp(w)))


def get_cdmft_host(label, iw, spin_down=False, clus=0):
    return _cmat(lib().ref_qcm_get_cdmft_host, label, int(spin_down), iw, clus)


def cdmft_distance(label, p, clus=0):
    v = np.ascontiguousarray(p, dtype=np.float64)
    d = C.c_double()
    _check(lib().ref_qcm_cdmft_distance(label, len(v), _dp(v), clus, C.byref(d)))
    return d.value


def _gen0(n_sites, n_bath, generators, bath_irrep):
    """pyqcm's 1-based generators -> ED::new_model's 0-based rows (flat int array)."""
    n_orb = n_sites + n_bath
    rows = [list(map(int, g)) for g in (generators or [])]
    for g in rows:
        for i in range(n_orb):
            if i < n_sites or not bath_irrep:
                g[i] -= 1
    flat = [v for g in rows for v in g]
    return len(rows), (C.c_int * max(len(flat), 1))(*flat)


def symmetry_group(n_sites, n_bath, generators, bath_irrep=False):
    ng, arr = _gen0(n_sites, n_bath, generators, bath_irrep)
    g = C.c_int()
    phi = (C.c_int * 256)()
    sre = np.zeros(n_sites * n_sites)
    sim = np.zeros(n_sites * n_sites)
    dims = (C.c_int * 16)()
    _check(lib().ref_symmetry_group(n_sites, n_bath, ng, arr, int(bool(bath_irrep)), C.byref(g), phi, _dp(sre),
                                    _dp(sim), dims))
    n = g.value
    return {"g": n, "phi": np.array(phi[:n * n]).reshape(n, n), "S": (sre + 1j * sim).reshape(n_sites, n_sites),
            "site_irrep_dim": np.array(dims[:n])}


def representatives(n_sites, n_bath, generators, bath_irrep, irrep, states):
    ng, arr = _gen0(n_sites, n_bath, generators, bath_irrep)
    st = np.ascontiguousarray(states, dtype=np.uint64)
    rep = np.zeros(len(st), dtype=np.uint64)
    ph = np.zeros(len(st), dtype=np.int32)
    ln = np.zeros(len(st), dtype=np.int32)
    u64 = C.POINTER(C.c_uint64)
    ip = C.POINTER(C.c_int)
    _check(lib().ref_representatives(n_sites, n_bath, ng, arr, int(bool(bath_irrep)), irrep, len(st),
                                     st.ctypes.data_as(u64), rep.ctypes.data_as(u64), ph.ctypes.data_as(ip),
                                     ln.ctypes.data_as(ip)))
    return rep, ph, ln


def mixed_basis(n_sites, n_bath, generators, bath_irrep, sector):
    ng, arr = _gen0(n_sites, n_bath, generators, bath_irrep)
    d = C.c_long()
    _check(lib().ref_mixed_basis(n_sites, n_bath, ng, arr, int(bool(bath_irrep)), sector.encode(), None, C.byref(d)))
    out = np.zeros(d.value, dtype=np.uint64)
    _check(lib().ref_mixed_basis(n_sites, n_bath, ng, arr, int(bool(bath_irrep)), sector.encode(),
                                 out.ctypes.data_as(C.POINTER(C.c_uint64)), C.byref(d)))
    return out
