"""ODF / PMF volumes from SH coefficients on the GPU (tensor cores).

The reference computes the ODF volume on the host before tracking
(``run_gpu_streamlines.py:357-380``: ``fit.odf(sphere)``, clipped to >= 0 for
the probabilistic getter).  ``odf_volume_gpu`` evaluates
``max(0, coef @ basis.T)`` with the library's BF16x3 tensor-core kernel
(``csl_odf_volume``) into library-owned device memory.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def device_input(x, device: int, dtype=np.float32):
    """(device pointer, keep-alive object, shape) of an array argument: a CUDA
    array that exposes ``data_ptr()`` and ``is_cuda`` (contiguous, of `dtype`)
    is used in place; anything else is copied to a new ``DeviceBuffer``."""
    if getattr(x, "is_cuda", False) and hasattr(x, "data_ptr"):
        if not x.is_contiguous() or np.dtype(str(x.dtype).replace("torch.", "")) != np.dtype(dtype):
            raise ValueError(f"device arrays must be contiguous {np.dtype(dtype).name}")
        return int(x.data_ptr()), x, tuple(int(d) for d in x.shape)
    a = np.ascontiguousarray(np.asarray(x), dtype=dtype)
    b = _lib.DeviceBuffer.from_array(a, device)
    return b.ptr, b, a.shape


def odf_volume_gpu(coef, basis, clip: bool = True, device: int = 0, return_ms: bool = False):
    """coef [..., C] and basis [V, C] -> DeviceBuffer float32 [..., V] on ``device``
    (``.numpy()`` copies it to the host, ``.ptr`` is the device address)."""
    cp, ckeep, cshape = device_input(coef, device)
    bp, bkeep, bshape = device_input(basis, device)
    ncoef = int(cshape[-1])
    nrows = int(np.prod(cshape[:-1], dtype=np.int64))
    if len(bshape) != 2 or bshape[1] != ncoef:
        raise ValueError("basis must be [n_vertices, n_coefficients]")
    nvert = int(bshape[0])
    out = _lib.DeviceBuffer(device, (nrows, nvert), np.float32)
    kp = (ncoef + 15) // 16 * 16
    ws_bytes = ((nvert + 255) // 256) * 256 * kp * 4 + 16
    ws = _lib.DeviceBuffer(device, (ws_bytes,), np.uint8)
    ms = np.zeros(1, dtype=np.float32)
    rc = _lib.load().csl_odf_volume(C.c_void_p(cp), nrows, ncoef, C.c_void_p(bp), nvert, 1 if clip else 0,
                                    C.c_void_p(out.ptr), C.c_void_p(ws.ptr), ws_bytes, _lib.fptr(ms), None)
    _lib.check(rc)
    _lib.device_sync(device)
    ws.close()
    out.reshape(*cshape[:-1], nvert)
    return (out, float(ms[0])) if return_ms else out
