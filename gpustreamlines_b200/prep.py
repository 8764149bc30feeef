"""FA map and seeds on the GPU: the steps before tracking that the reference
runs on the host through DIPY (``run_gpu_streamlines.py:289-314``:
``TensorModel(gtab, fit_method="WLS").fit(data, mask).fa`` and
``utils.random_seeds_from_mask``).  Results live in library-owned device
memory (``DeviceBuffer``: ``.numpy()`` copies to the host, ``.ptr`` is the
device address to pass on, e.g. as the seeds of ``csl_propagate_device``).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from .odf import device_input


def dti_fa_gpu(dwi, bvals, bvecs, mask=None, min_signal=1e-6, device: int = 0):
    """dwi [X, Y, Z, T] -> FA [X, Y, Z] float32 DeviceBuffer."""
    dp_, dkeep, dshape = device_input(dwi, device)
    shape, T = dshape[:-1], int(dshape[-1])
    nvox = int(np.prod(shape, dtype=np.int64))
    b = np.ascontiguousarray(np.asarray(bvals, np.float64).reshape(T))
    g = np.ascontiguousarray(np.asarray(bvecs, np.float64).reshape(T, 3))
    mp = None
    if mask is not None:
        mp, mkeep, _ = device_input(mask, device)
    fa = _lib.DeviceBuffer(device, (nvox,), np.float32)
    dp = C.POINTER(C.c_double)
    rc = _lib.load().csl_dti_fa(C.c_void_p(dp_), nvox, T, b.ctypes.data_as(dp), g.ctypes.data_as(dp),
                                C.c_void_p(mp) if mp is not None else None, float(min_signal),
                                C.c_void_p(fa.ptr), None)
    _lib.check(rc)
    _lib.device_sync(device)
    return fa.reshape(*shape)


def seeds_from_mask_gpu(mask, n, threshold=0.0, seed=0, device: int = 0):
    """n seeds [n, 3] float32 (voxel coordinates) uniform over voxels with
    mask > threshold, as a DeviceBuffer."""
    mp, mkeep, mshape = device_input(mask, device)
    X, Y, Z = (int(x) for x in mshape)
    out = _lib.DeviceBuffer(device, (int(n), 3), np.float32)
    nv = C.c_longlong()
    rc = _lib.load().csl_seeds_from_mask(C.c_void_p(mp), X, Y, Z, float(threshold), int(n), int(seed),
                                         C.c_void_p(out.ptr), C.byref(nv), None)
    _lib.check(rc)
    _lib.device_sync(device)
    return out
