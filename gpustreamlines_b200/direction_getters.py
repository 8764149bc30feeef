"""Direction getters: the host side of the bootstrap, probabilistic and PTT getters.

Mirrors ``cuslines/cuda_python/cu_direction_getters.py``: same class names,
constructor arguments, defaults and ``from_dipy_*`` factories.  The reference
compiles a CUDA program per tracker with NVRTC, baking volume sizes and
thresholds into macros (``compile_program``, ``cu_direction_getters.py:53-144``);
here one prebuilt sm_100a library serves every shape, so each getter only
contributes its fields of the C ABI's ``csl_params`` / ``csl_inputs``.
"""

from __future__ import annotations

import ctypes as C
import logging
import math
from abc import ABC

import numpy as np

from . import _lib
from . import shm as _shm

logger = logging.getLogger("GPUStreamlines")

REAL_DTYPE = np.float32
MAX_SLINE_LEN = 501        # points per tracking direction (reference _globals.py:3)
PMF_THRESHOLD_P = 0.05     # reference _globals.py:4
EXCESS_ALLOC_FACT = 2
MAX_SLINES_PER_SEED = 10


class GPUDirectionGetter(ABC):
    """Base class (``cu_direction_getters.py:35-144``)."""

    model = None

    def compile_program(self, gpu_tracker, debug: bool = False):
        """No JIT step: the kernels are prebuilt for sm_100a with runtime shapes."""
        self._compiled_for = (gpu_tracker.dimx, gpu_tracker.dimy, gpu_tracker.dimz,
                              gpu_tracker.dimt)

    def set_macros(self, gpu_tracker):
        pass

    def allocate_on_gpu(self, n):
        pass

    def deallocate_on_gpu(self, n):
        pass

    def fill(self, params: _lib.CslParams, inputs: _lib.CslInputs, tracker, keep: list):
        """Fill this getter's fields of the C ABI structures."""
        raise NotImplementedError


class BootDirectionGetter(GPUDirectionGetter):
    """Residual-bootstrap getter (``cu_direction_getters.py:147-364``)."""

    def __init__(self, model_type: str, min_signal: float, H: np.ndarray, R: np.ndarray,
                 delta_b: np.ndarray, delta_q: np.ndarray, sampling_matrix: np.ndarray,
                 b0s_mask: np.ndarray, *, fit: str = "fp32"):
        """``fit`` (keyword only, not in the reference): "fp32" runs the
        reference's per-warp FP32 fit with identical results; "bf16x3" runs the
        batched tensor-core fit (CSA or OPDT), 128 streamline halves per CTA with
        BF16x3 products and FP32 accumulation; "bf16x3_fp64" is the batched fit
        that also fits again in float64 any row whose peak decisions lie within
        the BF16x3 error of flipping."""
        if fit not in ("fp32", "bf16x3", "bf16x3_fp64"):
            raise ValueError(f"Invalid fit {fit!r}, must be one of 'fp32', 'bf16x3', 'bf16x3_fp64'")
        self.fit = fit
        if model_type.upper() == "OPDT":
            self.model_type = _lib.MODEL_OPDT
        elif model_type.upper() == "CSA":
            self.model_type = _lib.MODEL_CSA
        else:
            raise ValueError(f"Invalid model_type {model_type}, must be one of 'OPDT', 'CSA'")
        self.model = self.model_type
        self.H = np.ascontiguousarray(H, dtype=REAL_DTYPE)
        self.R = np.ascontiguousarray(R, dtype=REAL_DTYPE)
        self.delta_b = np.ascontiguousarray(delta_b, dtype=REAL_DTYPE)
        self.delta_q = np.ascontiguousarray(delta_q, dtype=REAL_DTYPE)
        self.delta_nr = int(delta_b.shape[0])
        self.min_signal = REAL_DTYPE(min_signal)
        self.sampling_matrix = np.ascontiguousarray(sampling_matrix, dtype=REAL_DTYPE)
        self.b0s_mask = np.ascontiguousarray(b0s_mask, dtype=np.int32)

    @classmethod
    def from_dipy_opdt(cls, gtab, sphere, sh_order_max=6, full_basis=False, sh_lambda=0.006,
                       min_signal=1, *, fit="fp32"):
        return cls(**_shm.prepare_opdt(gtab, sphere, sh_order_max, full_basis, sh_lambda, min_signal),
                   fit=fit)

    @classmethod
    def from_dipy_csa(cls, gtab, sphere, sh_order_max=6, full_basis=False, sh_lambda=0.006,
                      min_signal=1, *, fit="fp32"):
        return cls(**_shm.prepare_csa(gtab, sphere, sh_order_max, full_basis, sh_lambda, min_signal),
                   fit=fit)

    def fill(self, params, inputs, tracker, keep):
        hr = int((self.b0s_mask == 0).sum())
        if self.H.shape != (hr, hr) or self.R.shape != (hr, hr):
            raise ValueError(f"H and R must be {hr}x{hr} (non-b0 volumes)")
        if self.delta_b.shape[1] != hr or self.delta_q.shape != self.delta_b.shape:
            raise ValueError("delta_b/delta_q must be [n_coef, n_dwi]")
        if self.sampling_matrix.shape[1] != self.delta_nr:
            raise ValueError("sampling_matrix must be [n_vertices, n_coef]")
        if len(self.b0s_mask) != tracker.dimt:
            raise ValueError("b0s_mask length must match the last dimension of dataf")
        params.model = self.model_type
        params.boot_fit = {"fp32": 0, "bf16x3": 1, "bf16x3_fp64": 2}[self.fit]
        params.min_signal = float(self.min_signal)
        params.delta_nr = self.delta_nr
        params.samplm_nr = int(self.sampling_matrix.shape[0])
        for name in ("H", "R", "delta_b", "delta_q", "sampling_matrix"):
            a = getattr(self, name)
            keep.append(a)
            setattr(inputs, name, _lib.fptr(a))
        keep.append(self.b0s_mask)
        inputs.b0s_mask = _lib.iptr(self.b0s_mask)


class ProbDirectionGetter(GPUDirectionGetter):
    """Probabilistic getter (``cu_direction_getters.py:367-414``)."""

    model = _lib.MODEL_PROB

    def __init__(self, *, sampler: str = "inverse_cdf"):
        """``sampler`` (keyword only, not in the reference): "inverse_cdf" is
        the reference's sampler with identical results; "envelope" draws from
        the same distribution by exact rejection sampling, with proposals
        bounded by per-voxel vertex-cluster maxima (bfloat16, rounded up), and
        falls back to the inverse CDF after 16 rejected proposals."""
        if sampler not in ("inverse_cdf", "envelope"):
            raise ValueError(f"Invalid sampler {sampler!r}, must be one of 'inverse_cdf', 'envelope'")
        self.sampler = sampler

    def fill(self, params, inputs, tracker, keep):
        params.model = _lib.MODEL_PROB
        params.samplm_nr = tracker.dimt
        params.prob_sampler = 1 if self.sampler == "envelope" else 0


class PttDirectionGetter(ProbDirectionGetter):
    """Parallel transport tractography getter (``cu_direction_getters.py:417-648``)."""

    model = _lib.MODEL_PTT

    def __init__(self, odf_lut_res: int = 128, probe_length: float = 0.25,
                 target_short_step: float = 0.025, probe_quality: int = 8):
        self.odf_lut_res = odf_lut_res
        self.sphere_vertices_lut_h = None
        self.probe_length = probe_length
        self.probe_quality = probe_quality
        self.target_short_step = target_short_step

    def prepare_data(self, dataf, stop_map, stop_threshold, sphere_vertices, sphere_symm):
        """Normalise and tile the ODF for the texture, and build the vertex LUT,
        on the GPU (``csl_ptt_prepare``; device ``self.device``, default 0).

        Same transformation as ``cu_direction_getters.py:531-625``: clip at 0,
        zero outside the tracking mask, normalise each voxel to max 1, tile
        the vertex axis over (nx, ny, nz) power-of-two tiles, and map a
        ``res^3`` grid on [-1, 1]^3 to the nearest sphere vertex.  Returns the
        tiled data as a ``DeviceBuffer`` (``.numpy()`` copies it to the host);
        equal to ``prepare_data_host`` bit for bit except at exact vertex
        distance ties of the LUT.
        """
        dataf = np.ascontiguousarray(dataf, dtype=np.float32)
        X, Y, Z, T = dataf.shape
        lib = _lib.load()
        lay = [C.c_int() for _ in range(5)]
        _lib.check(lib.csl_ptt_layout(T, *[C.byref(x) for x in lay]))
        self.nx, self.ny, self.nz, self.log2_x, self.log2_y = (x.value for x in lay)
        dev = int(getattr(self, "device", 0))
        verts = np.ascontiguousarray(sphere_vertices, dtype=np.float32)
        # the host computation compares stop_map < stop_threshold with numpy's
        # promotion: in float32 for a Python or float32 threshold
        thr = np.asarray(stop_threshold)
        thr = float(np.float32(thr)) if np.result_type(np.float32, stop_threshold) == np.float32 else float(thr)
        odf = _lib.DeviceBuffer.from_array(dataf, dev)
        stop = _lib.DeviceBuffer.from_array(np.ascontiguousarray(stop_map, dtype=np.float32), dev)
        vd = _lib.DeviceBuffer.from_array(verts, dev)
        tiled = _lib.DeviceBuffer(dev, (self.nz * Z, self.ny * Y, self.nx * X), np.float32)
        res = int(self.odf_lut_res)
        lut = _lib.DeviceBuffer(dev, (res, res, res), np.float32)
        rc = lib.csl_ptt_prepare(C.c_void_p(odf.ptr), C.c_void_p(stop.ptr), X, Y, Z, T, thr, C.c_void_p(vd.ptr),
                                 len(verts), 1 if sphere_symm else 0, res, C.c_void_p(tiled.ptr),
                                 C.c_void_p(lut.ptr), None)
        _lib.check(rc)
        _lib.device_sync(dev)
        for b in (odf, stop, vd):
            b.close()
        logger.info("PTT ODF texture %dx%dx%d (%.2f GB), prepared on GPU %d", self.nx * X, self.ny * Y,
                    self.nz * Z, tiled.nbytes / 1e9, dev)
        self._lut_dev = lut
        self.sphere_vertices_lut_h = None
        return tiled

    def prepare_data_host(self, dataf, stop_map, stop_threshold, sphere_vertices, sphere_symm):
        """The host computation of ``prepare_data`` (numpy + a KD-tree), as the
        reference runs it (``cu_direction_getters.py:531-625``); returns the
        tiled array and sets ``sphere_vertices_lut_h``.  The library's own path
        is ``prepare_data`` (on the GPU); this one serves the CPU oracle."""
        from scipy.spatial import cKDTree

        dimx, dimy, dimz, dimt = dataf.shape
        dataf = np.asarray(dataf, dtype=np.float32).clip(min=0)
        dataf[np.asarray(stop_map) < stop_threshold, :] = 0
        odf_max = dataf.max(axis=3, keepdims=True)
        np.divide(dataf, odf_max, out=dataf, where=odf_max > 0)

        nx = ny = nz = 1
        while nx * ny * nz < dimt:
            if nx <= ny and nx <= nz:
                nx *= 2
            elif ny <= nx and ny <= nz:
                ny *= 2
            else:
                nz *= 2
        self.log2_x = int(math.log2(nx))
        self.log2_y = int(math.log2(ny))
        self.nx, self.ny, self.nz = nx, ny, nz
        slots = nx * ny * nz
        if dimt < slots:
            pad = np.zeros((dimx, dimy, dimz, slots - dimt), dtype=np.float32)
            dataf = np.concatenate([dataf, pad], axis=3)
        logger.info("PTT ODF texture %dx%dx%d (%.2f GB)", nx * dimx, ny * dimy, nz * dimz,
                    nx * dimx * ny * dimy * nz * dimz * 4 / 1e9)
        tiled = dataf.reshape(dimx, dimy, dimz, nz, ny, nx).transpose(3, 2, 4, 1, 5, 0)
        tiled = np.ascontiguousarray(tiled.reshape(nz * dimz, ny * dimy, nx * dimx), dtype=np.float32)

        coords = np.linspace(-1, 1, self.odf_lut_res)
        gx, gy, gz = np.meshgrid(coords, coords, coords, indexing="ij")
        grid = np.stack([gx.ravel(), gy.ravel(), gz.ravel()], axis=1)
        sv = np.asarray(sphere_vertices, dtype=np.float64)
        if sphere_symm:
            tree = cKDTree(np.concatenate([sv, -sv], axis=0))
            _, idx = tree.query(grid)
            idx = np.concatenate([np.arange(len(sv)), np.arange(len(sv))])[idx]
        else:
            _, idx = cKDTree(sv).query(grid)
        self.sphere_vertices_lut_h = np.ascontiguousarray(
            idx.reshape((self.odf_lut_res,) * 3), dtype=np.float32)
        return tiled

    def fill(self, params, inputs, tracker, keep):
        lut = getattr(self, "_lut_dev", None)
        if lut is None:
            lut = self.sphere_vertices_lut_h
        if lut is None:
            raise RuntimeError("PttDirectionGetter.prepare_data must run before allocation")
        params.model = _lib.MODEL_PTT
        params.samplm_nr = tracker.dimt
        params.odf_lut_res = int(self.odf_lut_res)
        params.step_frac = int(np.round(tracker.step_size / self.target_short_step))
        params.probe_step_size = float(self.probe_length)
        params.probe_quality = float(self.probe_quality)
        params.max_curvature = float(8.0 * np.sin(tracker.max_angle / 2.0))
        params.tile_log2_x, params.tile_log2_y = self.log2_x, self.log2_y
        params.tile_nx, params.tile_ny, params.tile_nz = self.nx, self.ny, self.nz
        keep.append(tracker.dataf)
        keep.append(lut)
        inputs.ptt_odf_tiled = _lib.any_fptr(tracker.dataf)
        inputs.ptt_lut = _lib.any_fptr(lut)
