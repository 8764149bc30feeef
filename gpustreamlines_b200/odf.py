"""ODF / PMF volumes from SH coefficients on the GPU (tensor cores).

The reference computes the ODF volume on the host before tracking
(``run_gpu_streamlines.py:357-380``: ``fit.odf(sphere)``, clipped to >= 0 for
the probabilistic getter).  ``odf_volume_gpu`` evaluates
``max(0, coef @ basis.T)`` with the library's BF16x3 tensor-core kernel
(``csl_odf_volume``); device memory comes from torch.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def odf_volume_gpu(coef, basis, clip: bool = True, device: int = 0, return_ms: bool = False):
    """coef [..., C] and basis [V, C] (numpy or torch) -> torch float32 [..., V] on ``device``."""
    import torch

    dev = torch.device("cuda", device)
    ct = torch.as_tensor(np.asarray(coef, dtype=np.float32) if not torch.is_tensor(coef) else coef)
    shape = ct.shape[:-1]
    ncoef = int(ct.shape[-1])
    ct = ct.to(dev, dtype=torch.float32).reshape(-1, ncoef).contiguous()
    bt = torch.as_tensor(np.asarray(basis, dtype=np.float32) if not torch.is_tensor(basis) else basis)
    bt = bt.to(dev, dtype=torch.float32).contiguous()
    nvert = int(bt.shape[0])
    if bt.shape[1] != ncoef:
        raise ValueError("basis must be [n_vertices, n_coefficients]")
    out = torch.empty((ct.shape[0], nvert), dtype=torch.float32, device=dev)
    kp = (ncoef + 15) // 16 * 16
    ws_bytes = ((nvert + 255) // 256) * 256 * kp * 4 + 16
    ws = torch.empty(ws_bytes, dtype=torch.uint8, device=dev)
    ms = np.zeros(1, dtype=np.float32)
    lib = _lib.load()
    with torch.cuda.device(dev):
        stream = torch.cuda.current_stream(dev).cuda_stream
        rc = lib.csl_odf_volume(C.c_void_p(ct.data_ptr()), int(ct.shape[0]), ncoef, C.c_void_p(bt.data_ptr()),
                                nvert, 1 if clip else 0, C.c_void_p(out.data_ptr()), C.c_void_p(ws.data_ptr()),
                                ws_bytes, _lib.fptr(ms), C.c_void_p(stream))
    _lib.check(rc)
    out = out.reshape(*shape, nvert)
    return (out, float(ms[0])) if return_ms else out
