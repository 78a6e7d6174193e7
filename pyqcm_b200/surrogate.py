"""Surrogate of the Potthoff functional for VCA: a multilayer perceptron
(n_in -> W -> W -> W -> 1, GELU) with BF16 tensor-core products, FP32
accumulation and Adam, all in this package's CUDA library (pyqcm_b200/csrc/mlp.cu).
It is trained on Omega values computed by the GPU ED and proposes starting
points for the ED Newton-Raphson search, which then verifies and refines them."""
from __future__ import annotations

import ctypes as C

import numpy as np

import pyqcm_b200 as qed


def _lib():
    L = qed.lib()
    if not getattr(L, "_mlp_sigs", False):
        vp = C.c_void_p
        fp = C.POINTER(C.c_float)
        sig = {
            "qed_mlp_create": [C.c_int, C.c_int, C.c_ulonglong, C.POINTER(C.c_void_p)],
            "qed_mlp_last_error": [C.c_char_p, C.c_int],
            "qed_mlp_num_params": [vp, C.POINTER(C.c_long)],
            "qed_mlp_layout": [vp, C.POINTER(C.c_long)],
            "qed_mlp_get_params": [vp, fp],
            "qed_mlp_set_params": [vp, fp],
            "qed_mlp_forward": [vp, C.c_int, fp, fp],
            "qed_mlp_gradients": [vp, C.c_int, fp, fp, fp, fp],
            "qed_mlp_train": [vp, C.c_int, fp, fp, C.c_int, C.c_int, C.c_float, C.c_ulonglong, fp],
            "qed_mlp_tensor_product": [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint16), C.POINTER(C.c_uint16), fp],
        }
        for k, a in sig.items():
            getattr(L, k).argtypes = a
            getattr(L, k).restype = C.c_int
        L.qed_mlp_destroy.argtypes = [vp]
        L.qed_mlp_destroy.restype = None
        L._mlp_sigs = True
    return L


def _check(rc):
    if rc != 0:
        buf = C.create_string_buffer(4096)
        _lib().qed_mlp_last_error(buf, 4096)
        raise qed.QEDError(rc, buf.value.decode(errors="replace"))


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def to_bf16_bits(a) -> np.ndarray:
    """BF16 bit patterns of a float array (round to nearest even), as uint16."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    r = ((u >> 16) & 1) + 0x7FFF
    return ((u + r) >> 16).astype(np.uint16)


def from_bf16_bits(b) -> np.ndarray:
    return (np.asarray(b, dtype=np.uint32) << 16).view(np.float32)


def tensor_product(a_bits, b_bits) -> np.ndarray:
    """C = A B^T on the surrogate's tcgen05 kernel; A (M x K) and B (N x K) as BF16
    bit patterns (uint16), C in FP32."""
    a_bits = np.ascontiguousarray(a_bits, dtype=np.uint16)
    b_bits = np.ascontiguousarray(b_bits, dtype=np.uint16)
    M, K = a_bits.shape
    N = b_bits.shape[0]
    c = np.empty((M, N), dtype=np.float32)
    u16 = C.POINTER(C.c_uint16)
    _check(_lib().qed_mlp_tensor_product(M, N, K, a_bits.ctypes.data_as(u16), b_bits.ctypes.data_as(u16), _fp(c)))
    return c


class MLP:
    """The surrogate network on the GPU (one CUDA stream of its own)."""

    def __init__(self, n_in: int = 4, width: int = 256, seed: int = 0):
        self.n_in = n_in
        self.width = width
        h = C.c_void_p()
        _check(_lib().qed_mlp_create(n_in, width, seed, C.byref(h)))
        self._h = h
        n = C.c_long()
        _check(_lib().qed_mlp_num_params(h, C.byref(n)))
        self.n_params = n.value
        off = (C.c_long * 9)()
        _check(_lib().qed_mlp_layout(h, off))
        self.offsets = list(off)[:8]
        self.k_in = off[8]

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            _lib().qed_mlp_destroy(h)
            self._h = None

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.n_params, dtype=np.float32)
        _check(_lib().qed_mlp_get_params(self._h, _fp(out)))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.n_params:
            raise ValueError("parameter vector of the wrong size")
        _check(_lib().qed_mlp_set_params(self._h, _fp(p)))

    def blocks(self, p=None):
        """(W1, b1, W2, b2, W3, b3, w4, b4) views of a parameter vector."""
        p = self.get_params() if p is None else p
        W, k = self.width, self.k_in
        shapes = [(W, k), (W,), (W, W), (W,), (W, W), (W,), (W,), (1,)]
        return [p[o:o + int(np.prod(s))].reshape(s) for o, s in zip(self.offsets, shapes)]

    def __call__(self, x) -> np.ndarray:
        x = np.ascontiguousarray(np.atleast_2d(x), dtype=np.float32)
        y = np.zeros(len(x), dtype=np.float32)
        _check(_lib().qed_mlp_forward(self._h, len(x), _fp(x), _fp(y)))
        return y

    def gradients(self, x, t):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(self.n_params, dtype=np.float32)
        loss = C.c_float()
        _check(_lib().qed_mlp_gradients(self._h, len(x), _fp(x), _fp(t), _fp(g), C.byref(loss)))
        return g, loss.value

    def train(self, x, t, epochs: int, batch: int = 256, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        losses = np.zeros(epochs, dtype=np.float32)
        _check(_lib().qed_mlp_train(self._h, len(x), _fp(x), _fp(t), epochs, batch, lr, seed, _fp(losses)))
        return losses
