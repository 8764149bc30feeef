"""ctypes wrapper of tests/_probe.so (GPU probes that pin the oracle)."""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_probe.so")
_fp = C.POINTER(C.c_float)
_u64p = C.POINTER(C.c_ulonglong)
_lib = None


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(PATH)
        L.probe_curand.argtypes = [C.c_ulonglong, _u64p, _u64p, C.c_int, C.c_int,
                                   C.POINTER(C.c_uint), _fp, _fp]
        L.probe_dot.argtypes = [_fp, _fp, C.c_int, _fp]
        L.probe_fast.argtypes = [_fp, C.c_int, _fp, _fp]
        L.probe_tex3d.argtypes = [_fp, C.c_int, C.c_int, C.c_int, _fp, C.c_int, _fp]
        _lib = L
    return _lib


def _f(a):
    return a.ctypes.data_as(_fp)


def curand(seed, subseq, offs, ndraw):
    subseq = np.ascontiguousarray(subseq, dtype=np.uint64)
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    n = len(subseq)
    u = np.zeros((n, ndraw), dtype=np.uint32)
    f = np.zeros((n, ndraw), dtype=np.float32)
    g = np.zeros((n, ndraw), dtype=np.float32)
    rc = lib().probe_curand(seed, subseq.ctypes.data_as(_u64p), offs.ctypes.data_as(_u64p), n, ndraw,
                            u.ctypes.data_as(C.POINTER(C.c_uint)), _f(f), _f(g))
    assert rc == 0, rc
    return u, f, g


def dot(a, b):
    a = np.ascontiguousarray(a, dtype=np.float32)
    b = np.ascontiguousarray(b, dtype=np.float32)
    out = np.zeros(len(a), dtype=np.float32)
    assert lib().probe_dot(_f(a), _f(b), len(a), _f(out)) == 0
    return out


def fast(x):
    x = np.ascontiguousarray(x, dtype=np.float32)
    c = np.zeros_like(x)
    l = np.zeros_like(x)
    assert lib().probe_fast(_f(x), len(x), _f(c), _f(l)) == 0
    return c, l


def tex3d(vol, pts):
    vol = np.ascontiguousarray(vol, dtype=np.float32)
    pts = np.ascontiguousarray(pts, dtype=np.float32)
    out = np.zeros(len(pts), dtype=np.float32)
    X, Y, Z = vol.shape
    assert lib().probe_tex3d(_f(vol), X, Y, Z, _f(pts), len(pts), _f(out)) == 0
    return out
