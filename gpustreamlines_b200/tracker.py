"""``GPUTracker``: the reference's tracker API on the sm_100a library.

Same constructor, defaults and context-manager semantics as
``cuslines/cuda_python/cu_tractography.py:36-300``: ``__init__`` validates and
prepares host arrays, ``__enter__`` uploads everything to each GPU
(one ``csl_tracker`` handle per device), ``__exit__`` releases it.
"""

from __future__ import annotations

import logging
from math import radians

import numpy as np

from . import _lib
from .direction_getters import (MAX_SLINE_LEN, PMF_THRESHOLD_P, BootDirectionGetter,
                                GPUDirectionGetter, PttDirectionGetter)
from .generic_tracker import GenericTracker
from .propagate import SeedBatchPropagator

logger = logging.getLogger("GPUStreamlines")

REAL_DTYPE = np.float32


def device_count() -> int:
    """CUDA devices visible (through the library; 0 when none can be used)."""
    try:
        return _lib.device_count()
    except (RuntimeError, OSError):
        return 0


class GPUTracker(GenericTracker):
    def __init__(self, dg: GPUDirectionGetter, dataf: np.ndarray, stop_map: np.ndarray,
                 stop_threshold: float, sphere_vertices: np.ndarray, sphere_edges: np.ndarray,
                 sphere_symm: bool = False, max_angle: float = radians(60), step_size: float = 0.5,
                 min_pts=0, max_pts=np.inf, relative_peak_thresh: float = 0.25,
                 min_separation_angle: float = radians(45), ngpus: int = 1, rng_seed: int = 0,
                 rng_offset: int = 0, chunk_size: int = 25000, device_offset: int = 0):
        """Tracker over a 4D volume.

        dg: direction getter.  dataf: [X,Y,Z,T] ODF/PMF (prob, PTT) or DWI
        (bootstrap).  stop_map/stop_threshold: tracking continues while the
        (texture-filtered) stop map is above the threshold.  sphere_vertices /
        sphere_edges: the sampling sphere.  Angles are radians, step_size is in
        voxels, seeds are voxel coordinates.  ``device_offset`` selects the first
        CUDA device (one process per GPU).
        """
        self.dimx, self.dimy, self.dimz, self.dimt = (int(d) for d in np.shape(dataf))
        if hasattr(dg, "prepare_data"):
            dg.device = int(device_offset)  # the getter's data preparation runs on the first GPU
            self.dataf = dg.prepare_data(np.array(dataf, dtype=np.float32), stop_map, stop_threshold,
                                         sphere_vertices, sphere_symm)
        else:
            self.dataf = np.ascontiguousarray(dataf, dtype=REAL_DTYPE)
        self.metric_map = np.ascontiguousarray(stop_map, dtype=np.float32)
        if self.metric_map.shape != (self.dimx, self.dimy, self.dimz):
            raise ValueError("stop_map must have the spatial shape of dataf")
        self.sphere_vertices = np.ascontiguousarray(sphere_vertices, dtype=REAL_DTYPE)
        self.sphere_edges = np.ascontiguousarray(sphere_edges, dtype=np.int32)
        self.nedges = int(self.sphere_edges.shape[0])
        if isinstance(dg, BootDirectionGetter):
            self.samplm_nr = int(dg.sampling_matrix.shape[0])
        else:
            if len(self.sphere_vertices) != self.dimt:
                raise ValueError(
                    f"Number of sphere vertices ({len(self.sphere_vertices)}) must"
                    f" match last dimension of dataf ({self.dimt}), "
                    "because dataf should be an ODF when using prob or ptt tracking")
            self.samplm_nr = self.dimt
        self.n32dimt = ((self.dimt + 31) // 32) * 32
        self.dg = dg
        self.max_angle = REAL_DTYPE(max_angle)
        self.tc_threshold = REAL_DTYPE(stop_threshold)
        self.step_size = REAL_DTYPE(step_size)
        self.relative_peak_thresh = REAL_DTYPE(relative_peak_thresh)
        self.min_separation_angle = REAL_DTYPE(min_separation_angle)
        self.ngpus = int(ngpus)
        self.rng_seed = int(rng_seed)
        self.rng_offset = int(rng_offset)
        self.chunk_size = int(chunk_size)
        self.sphere_symm = bool(sphere_symm)
        self.device_offset = int(device_offset)
        avail = device_count()
        if self.device_offset + self.ngpus > avail:
            raise RuntimeError(f"Requested {self.ngpus} GPUs but only {avail} available")
        logger.info("Creating GPUTracker with %d GPUs...", self.ngpus)
        self.handles = []
        self.seed_propagator = SeedBatchPropagator(gpu_tracker=self, minlen=min_pts, maxlen=max_pts)
        self._allocated = False
        self.dg.compile_program(self)

    def c_params(self) -> _lib.CslParams:
        p = _lib.CslParams()
        p.dimx, p.dimy, p.dimz, p.dimt = self.dimx, self.dimy, self.dimz, self.dimt
        p.nvertices = len(self.sphere_vertices)
        p.nedges = self.nedges
        p.samplm_nr = self.samplm_nr
        p.sphere_symm = int(self.sphere_symm)
        p.max_sline_len = MAX_SLINE_LEN
        p.step_size = float(self.step_size)
        p.max_angle = float(self.max_angle)
        p.tc_threshold = float(self.tc_threshold)
        p.relative_peak_thresh = float(self.relative_peak_thresh)
        p.min_separation_angle = float(self.min_separation_angle)
        p.pmf_threshold = PMF_THRESHOLD_P
        p.rng_seed = self.rng_seed
        return p

    def _build(self):
        params = self.c_params()
        inputs = _lib.CslInputs()
        keep = [self.metric_map, self.sphere_vertices, self.sphere_edges]
        self.dg.fill(params, inputs, self, keep)
        if not isinstance(self.dg, PttDirectionGetter):
            keep.append(self.dataf)
            inputs.dataf = _lib.fptr(self.dataf)
        inputs.stop_map = _lib.fptr(self.metric_map)
        inputs.vertices = _lib.fptr(self.sphere_vertices)
        inputs.edges = _lib.iptr(self.sphere_edges)
        return params, inputs, keep

    def __enter__(self):
        self._allocate()
        return self

    def _allocate(self):
        if self._allocated:
            return
        params, inputs, keep = self._build()
        try:
            for ii in range(self.ngpus):
                self.handles.append(_lib.Handle(params, inputs, self.device_offset + ii, keep))
                self.dg.allocate_on_gpu(ii)
        except Exception:
            self._release()
            raise
        self._allocated = True

    def _release(self):
        for ii, h in enumerate(self.handles):
            try:
                h.close()
                self.dg.deallocate_on_gpu(ii)
            except Exception as e:  # soft errors on teardown, as the reference
                logger.warning("teardown: %s", e)
        self.handles = []
        self._allocated = False

    def __exit__(self, exc_type, exc, tb):
        logger.info("Destroying GPUTracker and freeing GPU memory...")
        self._release()
        return False

    def autotune(self, seeds: np.ndarray, sample: int = 20000, repeats: int = 2, seed: int = 0):
        """Choose the launch shape (threads per CTA, seed order) of every GPU's
        tracking path by timing the candidates on a random sample of ``seeds``
        (``csl_autotune``).  Streamlines do not depend on the shape.  Returns,
        per GPU, {(threads_per_block, seed_order): ms or None} and the chosen shape."""
        self._allocate()
        seeds = np.ascontiguousarray(np.asarray(seeds, dtype=np.float32).reshape(-1, 3))
        if len(seeds) == 0:
            raise ValueError("autotune needs at least one seed")
        rng = np.random.default_rng(seed)
        pick = seeds[rng.choice(len(seeds), size=min(sample, len(seeds)), replace=False)]
        out = []
        for h in self.handles:
            d = _lib.DeviceBuffer.from_array(pick, h.device, np.float32)
            ms = h.autotune(d.ptr, len(pick), 0, repeats)
            d.close()
            out.append((ms, h.get_launch()[:2]))
        return out
