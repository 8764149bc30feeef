"""Chunk propagator: the ``SeedBatchPropagator`` surface over the C ABI.

Mirrors ``cuslines/cuda_python/cu_propagate_seeds.py:26-262``.  Seeds of a
chunk are split into contiguous per-GPU blocks of ``ceil(n / ngpus)``
(``:45-54``); each GPU's tracker runs pass 1, the device scans, pass 2 and
the compaction in one ``csl_propagate`` call, and only the valid points are
copied back (the reference copies the padded nSlines x 1002 x float3 buffer,
``:171-204``).  Several GPUs run concurrently from one host thread each.
"""

from __future__ import annotations

import logging
import math
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from .io import MEGABYTE, ArraySequence

logger = logging.getLogger("GPUStreamlines")

REAL_SIZE = 4


class SeedBatchPropagator:
    def __init__(self, gpu_tracker, minlen=0, maxlen=np.inf):
        self.gpu_tracker = gpu_tracker
        self.ngpus = gpu_tracker.ngpus
        self.minlen = minlen
        self.maxlen = maxlen
        self.nSlines = np.zeros(self.ngpus, dtype=np.int64)
        self.nSlines_old = np.zeros(self.ngpus, dtype=np.int64)
        self.slines = [None] * self.ngpus       # [npts,3] float32 per GPU (compacted)
        self.sline_lens = [None] * self.ngpus   # [nSlines] int32 per GPU
        self.sline_seeds = [None] * self.ngpus  # [nSlines] int32 batch-local seed ids
        self.nseeds = 0
        self.nseeds_per_gpu = 0

    def _shard(self, n):
        nseeds_gpu = min(self.nseeds_per_gpu, max(0, self.nseeds - n * self.nseeds_per_gpu))
        return n * self.nseeds_per_gpu, nseeds_gpu

    def _run_gpu(self, ii, seeds):
        start, cnt = self._shard(ii)
        h = self.gpu_tracker.handles[ii]
        h.propagate(seeds[start:start + cnt], rng_index_base=0)
        L, S, P = h.fetch()
        return ii, L, S, P

    def propagate(self, seeds):
        seeds = np.ascontiguousarray(np.asarray(seeds), dtype=np.float32).reshape(-1, 3)
        self.nseeds = len(seeds)
        self.nseeds_per_gpu = (self.nseeds + self.ngpus - 1) // self.ngpus
        if not self.gpu_tracker._allocated:
            raise RuntimeError("GPUTracker must be entered (use `with`) before tracking")
        if self.ngpus == 1:
            results = [self._run_gpu(0, seeds)]
        else:
            with ThreadPoolExecutor(self.ngpus) as ex:
                results = list(ex.map(lambda i: self._run_gpu(i, seeds), range(self.ngpus)))
        self.nSlines_old = self.nSlines.copy()
        for ii, L, S, P in results:
            self.nSlines[ii] = len(L)
            self.sline_lens[ii] = L
            self.sline_seeds[ii] = S
            self.slines[ii] = P
        # the reference advances rng_offset per chunk (its kernels ignore it)
        self.gpu_tracker.rng_offset += self.nseeds

    def propagate_compressed(self, seeds, affine, tol_error, max_segment_length):
        """``propagate`` followed by the world transform and the linearisation
        on the device (``csl_compress``); only the compressed points are copied
        to the host.  Results: ``as_compressed_sequence()``."""
        seeds = np.ascontiguousarray(np.asarray(seeds), dtype=np.float32).reshape(-1, 3)
        self.nseeds = len(seeds)
        self.nseeds_per_gpu = (self.nseeds + self.ngpus - 1) // self.ngpus
        if not self.gpu_tracker._allocated:
            raise RuntimeError("GPUTracker must be entered (use `with`) before tracking")

        def run(ii):
            start, cnt = self._shard(ii)
            h = self.gpu_tracker.handles[ii]
            h.propagate(seeds[start:start + cnt], rng_index_base=0)
            counts, pts = h.compress(affine, tol_error, max_segment_length, int(max(0, self.minlen)),
                                     self.maxlen)
            return ii, counts[counts > 0], pts

        if self.ngpus == 1:
            results = [run(0)]
        else:
            with ThreadPoolExecutor(self.ngpus) as ex:
                results = list(ex.map(run, range(self.ngpus)))
        self.c_lens = [None] * self.ngpus
        self.c_pts = [None] * self.ngpus
        for ii, L, P in results:
            self.c_lens[ii] = L
            self.c_pts[ii] = P
        self.gpu_tracker.rng_offset += self.nseeds

    def as_compressed_sequence(self):
        """Compressed world-space streamlines of the last ``propagate_compressed``."""
        lens = [x for x in self.c_lens if x is not None and len(x)]
        pts = [p for x, p in zip(self.c_lens, self.c_pts) if x is not None and len(x)]
        if not lens:
            return ArraySequence()
        return ArraySequence.from_flat(np.concatenate(pts), np.concatenate(lens))

    def _keep(self, lens):
        return (lens >= self.minlen) & (lens <= self.maxlen)

    def get_buffer_size(self):
        total = 0
        for ii in range(self.ngpus):
            lens = self.sline_lens[ii]
            if lens is None:
                continue
            total += int(lens[self._keep(lens)].sum()) * 3 * REAL_SIZE
        return math.ceil(total / MEGABYTE)

    def as_generator(self):
        def _yield_slines():
            for ii in range(self.ngpus):
                lens = self.sline_lens[ii]
                if lens is None:
                    continue
                pts = self.slines[ii]
                off = 0
                for npts in lens:
                    if self.minlen <= npts <= self.maxlen:
                        yield pts[off:off + npts]
                    off += npts
        return _yield_slines()

    def as_array_sequence(self):
        """Kept streamlines of the last chunk as one flat ArraySequence (no copies per item)."""
        datas, lens_all = [], []
        for ii in range(self.ngpus):
            lens = self.sline_lens[ii]
            if lens is None or len(lens) == 0:
                continue
            keep = self._keep(lens)
            pts = self.slines[ii]
            if keep.all():
                datas.append(pts)
                lens_all.append(lens)
            else:
                starts = np.zeros(len(lens), dtype=np.int64)
                np.cumsum(lens[:-1], out=starts[1:])
                idx = np.concatenate([np.arange(s, s + l) for s, l, k in zip(starts, lens, keep) if k]) \
                    if keep.any() else np.zeros(0, dtype=np.int64)
                datas.append(pts[idx])
                lens_all.append(lens[keep])
        if not datas:
            return ArraySequence()
        return ArraySequence.from_flat(np.concatenate(datas), np.concatenate(lens_all))
