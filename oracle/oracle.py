"""ctypes wrapper of the CPU oracle (liboracle.so). TEST INFRASTRUCTURE ONLY.

Used by tests/, by `__graft_entry__.smoke()` as the checker, and by bench.py's CPU baseline and
reference arm. The product path never imports this module.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")

_lib = None


def build() -> str:
    """Compile liboracle.so with gcc (make)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        sig = [vp, C.c_int, C.c_int, vp, C.c_int64, vp, C.c_int64, vp, vp, C.c_int]
        for name in ("oracle_matvec", "oracle_farmul", "oracle_nearmul"):
            getattr(L, name).argtypes = sig
            getattr(L, name).restype = C.c_int
        L.oracle_last_error.restype = C.c_char_p
        L.oracle_toeplitz_apply.argtypes = [vp, vp, vp, vp, C.c_int]
        L.oracle_dft.argtypes = [vp, vp, C.c_int]
        L.oracle_max_threads.restype = C.c_int
        _lib = L
    return _lib


def max_threads() -> int:
    return int(lib().oracle_max_threads())


def _call(name, core, x, mode=0, alpha=None, beta=None, y=None, nthreads=0, desc=None):
    from h2factory_b200.core import flatten  # noqa: WPS433 (package registered by the caller)

    if desc is None:
        desc, keep = flatten(core)
    else:
        desc, keep = desc
    nrow, ncol = core.size
    nout, nin = (nrow, ncol) if mode == 0 else (ncol, nrow)
    x = np.asfortranarray(x, dtype=core.dtype)
    nrhs = 1 if x.ndim == 1 else x.shape[1]
    if y is None:
        y = np.zeros((nout,) if x.ndim == 1 else (nout, nrhs), dtype=core.dtype, order="F")
    else:
        y = np.asfortranarray(y, dtype=core.dtype).copy(order="F")
    ab = None
    if alpha is not None or beta is not None:
        a = complex(1 if alpha is None else alpha)
        b = complex(0 if beta is None else beta)
        ab = ((C.c_double * 2)(a.real, a.imag), (C.c_double * 2)(b.real, b.imag))
    st = getattr(lib(), name)(C.byref(desc), mode, nrhs, x.ctypes.data, nin, y.ctypes.data, nout,
                              C.cast(ab[0], C.c_void_p) if ab else None,
                              C.cast(ab[1], C.c_void_p) if ab else None, nthreads)
    if st != 0:
        raise RuntimeError(f"oracle status {st}: {lib().oracle_last_error().decode()}")
    del keep
    return y


def matvec(core, x, mode=0, alpha=None, beta=None, y=None, nthreads=0, desc=None):
    """mul!(y, op(A), x[, α, β]) on the CPU (op: 0 forward, 1 transpose, 2 adjoint)."""
    return _call("oracle_matvec", core, x, mode, alpha, beta, y, nthreads, desc)


def farmul(core, x, mode=0, alpha=None, beta=None, y=None, nthreads=0, desc=None):
    """farmul!(y, op(A), x[, α, β]) on the CPU."""
    return _call("oracle_farmul", core, x, mode, alpha, beta, y, nthreads, desc)


def nearmul(core, x, mode=0, alpha=None, beta=None, y=None, nthreads=0, desc=None):
    """nearmul!(y, op(A), x[, α, β]) on the CPU."""
    return _call("oracle_nearmul", core, x, mode, alpha, beta, y, nthreads, desc)


def toeplitz_apply(khat: np.ndarray, x: np.ndarray, adjoint: bool = False) -> np.ndarray:
    """The standalone Toeplitz operator (ext/H2Toeplitz/H2Toeplitz.jl:19-47)."""
    ts = khat.shape + (1,) * (3 - khat.ndim)
    s = np.array([(t + 1) // 2 for t in ts], np.int32)
    k = np.asfortranarray(khat, np.complex128).ravel(order="F")
    xx = np.ascontiguousarray(x, np.complex128)
    y = np.zeros(int(np.prod(s)), np.complex128)
    lib().oracle_toeplitz_apply(s.ctypes.data, k.ctypes.data, xx.ctypes.data, y.ctypes.data,
                                int(adjoint))
    return y


def dft(a: np.ndarray, inverse: bool = False) -> np.ndarray:
    """fft / ifft of a column-major complex array with AbstractFFTs conventions."""
    n = np.array(list(a.shape) + [1] * (3 - a.ndim), np.int32)
    buf = np.asfortranarray(a, np.complex128).ravel(order="F").copy()
    lib().oracle_dft(buf.ctypes.data, n.ctypes.data, int(inverse))
    return buf.reshape(a.shape, order="F")
