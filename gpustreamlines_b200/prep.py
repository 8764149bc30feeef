"""FA map and seeds on the GPU: the steps before tracking that the reference
runs on the host through DIPY (``run_gpu_streamlines.py:289-314``:
``TensorModel(gtab, fit_method="WLS").fit(data, mask).fa`` and
``utils.random_seeds_from_mask``).  Device memory comes from torch.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def _stream(dev):
    import torch

    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def dti_fa_gpu(dwi, bvals, bvecs, mask=None, min_signal=1e-6, device: int = 0):
    """dwi [X, Y, Z, T] (numpy or torch) -> FA [X, Y, Z] float32 torch tensor on the GPU."""
    import torch

    dev = torch.device("cuda", device)
    d = torch.as_tensor(dwi if torch.is_tensor(dwi) else np.asarray(dwi, np.float32)).to(dev, torch.float32)
    shape, T = d.shape[:-1], int(d.shape[-1])
    d = d.reshape(-1, T).contiguous()
    b = np.ascontiguousarray(np.asarray(bvals, np.float64).reshape(T))
    g = np.ascontiguousarray(np.asarray(bvecs, np.float64).reshape(T, 3))
    m = None
    if mask is not None:
        m = torch.as_tensor(mask if torch.is_tensor(mask) else np.asarray(mask, np.float32))
        m = m.to(dev, torch.float32).reshape(-1).contiguous()
    fa = torch.empty(d.shape[0], dtype=torch.float32, device=dev)
    dp = C.POINTER(C.c_double)
    with torch.cuda.device(dev):
        rc = _lib.load().csl_dti_fa(C.c_void_p(d.data_ptr()), d.shape[0], T, b.ctypes.data_as(dp),
                                    g.ctypes.data_as(dp), C.c_void_p(m.data_ptr()) if m is not None else None,
                                    float(min_signal), C.c_void_p(fa.data_ptr()), _stream(dev))
    _lib.check(rc)
    return fa.reshape(shape)


def seeds_from_mask_gpu(mask, n, threshold=0.0, seed=0, device: int = 0):
    """n seeds [n, 3] float32 (voxel coordinates) uniform over voxels with mask > threshold."""
    import torch

    dev = torch.device("cuda", device)
    m = torch.as_tensor(mask if torch.is_tensor(mask) else np.asarray(mask, np.float32)).to(dev, torch.float32)
    X, Y, Z = (int(x) for x in m.shape)
    m = m.contiguous()
    out = torch.empty((int(n), 3), dtype=torch.float32, device=dev)
    nv = C.c_longlong()
    with torch.cuda.device(dev):
        rc = _lib.load().csl_seeds_from_mask(C.c_void_p(m.data_ptr()), X, Y, Z, float(threshold), int(n),
                                             int(seed), C.c_void_p(out.data_ptr()), C.byref(nv), _stream(dev))
    _lib.check(rc)
    return out
