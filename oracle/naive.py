"""ctypes binding of the naive-DFT C restatement (oracle/naive_rhs.c) -- test only."""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "libnaive_rhs.so")
_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        _lib = ctypes.CDLL(_SO)
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.naive_rhs_nonlinear.argtypes = [ctypes.c_int] * 3 + [dp, dp, dp, dp]
        _lib.naive_c2r_field.argtypes = [ctypes.c_int] * 3 + [dp, dp]
        _lib.naive_r2c_field.argtypes = [ctypes.c_int] * 3 + [dp, dp]
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def rhs_nonlinear(uh, nx, ny, nz, alpha=(1.0, 1.0, 1.0), nu=0.0, Q=0.0, Pin=0.1,
                  kcut=2.5, bandlim=False, spherical=False):
    uh = np.ascontiguousarray(uh, np.complex128)
    out = np.empty_like(uh)
    prm = np.array([*alpha, nu, Q, Pin, kcut, float(bandlim), float(spherical)])
    eb = np.zeros(1)
    lib().naive_rhs_nonlinear(nx, ny, nz, _ptr(prm), _ptr(uh.view(np.float64)),
                              _ptr(out.view(np.float64)), _ptr(eb))
    return out, float(eb[0])


def c2r(F, nx, ny, nz):
    F = np.ascontiguousarray(F, np.complex128)
    f = np.empty((nz, ny, nx))
    lib().naive_c2r_field(nx, ny, nz, _ptr(F.view(np.float64)), _ptr(f))
    return f


def r2c(f, nx, ny, nz):
    f = np.ascontiguousarray(f, np.float64)
    F = np.empty((nz, ny, nx // 2 + 1), np.complex128)
    lib().naive_r2c_field(nx, ny, nz, _ptr(f), _ptr(F.view(np.float64)))
    return F
