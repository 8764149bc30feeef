"""Multi-subject run: many trackers' seed batches in one CUDA-graph launch.

The reference tracks one subject per ``GPUTracker`` and per
``generate_streamlines`` call (cuslines/cuda_python/cu_tractography.py:264-300),
so a study of many subjects is a host loop of launches, each with its own
host round trips between pass 1, pass 2 and compaction.  ``MultiSubjectRun``
binds several trackers (any getter: probabilistic, bootstrap, PTT; one device)
to fixed-size seed batches and runs all of them as branches of ONE captured
CUDA graph (``csl_multi_*`` in the C library): the GPU interleaves the
subjects' CTAs, and the host waits once.  Each subject's streamlines are
identical to its tracker's own ``generate_streamlines`` on the same seeds
(bootstrap trackers with the batched tensor-core fit run it in the graph too).

    with GPUTracker(...) as a, GPUTracker(...) as b:
        run = MultiSubjectRun([a, b], [seeds_a, seeds_b])
        run.run()
        sl_a = run.streamlines(0)
"""

from __future__ import annotations

import numpy as np

from . import _lib


class MultiSubjectRun:
    """Seed batches of several trackers as one captured CUDA graph.

    trackers: allocated (entered) GPU trackers on one device; each takes part
    at most once.  seeds: one float array [n_i, 3] per tracker (voxel
    coordinates, n_i may be 0); copied to the device once.  ``update_seeds``
    rewrites a batch in place (same count) before the next launch.
    points_per_streamline: initial pool estimate (0: 128); a subject whose
    pool or streamline slots overflow is re-run on the plain path by
    ``wait`` and the next launch re-captures with grown capacities.
    """

    def __init__(self, trackers, seeds, points_per_streamline: int = 0, rng_index_base=None):
        if len(trackers) != len(seeds) or not trackers:
            raise ValueError("one seed array per tracker, at least one tracker")
        for tr in trackers:
            tr._allocate()
        self.trackers = list(trackers)
        handles = [tr.handles[0] for tr in trackers]
        device = handles[0].device
        self._seeds = []
        for s in seeds:
            a = np.ascontiguousarray(np.asarray(s, dtype=np.float32).reshape(-1, 3))
            t = _lib.DeviceBuffer(device, (max(len(a), 1), 3), np.float32)
            if len(a):
                t.upload(a)
            self._seeds.append((t, len(a)))
        self.plan = _lib.MultiPlan(handles, [t.ptr for t, _ in self._seeds], [n for _, n in self._seeds],
                                   rng_index_base, points_per_streamline)
        self.last = None

    def update_seeds(self, i: int, seeds):
        t, n = self._seeds[i]
        a = np.ascontiguousarray(np.asarray(seeds, dtype=np.float32).reshape(-1, 3))
        if len(a) != n:
            raise ValueError(f"subject {i}: the plan was built for {n} seeds, got {len(a)}")
        if n:
            t.upload(a)

    def launch(self, stream: int | None = None):
        """Launch the graph (asynchronous)."""
        self.plan.launch(stream)

    def wait(self):
        """Wait for the launch; returns per-subject streamline and point counts,
        the subjects re-run on the plain path, and the graph's device time (ms)."""
        self.last = self.plan.wait()
        return self.last

    def set_concurrency(self, max_concurrent: int):
        """At most this many subjects' tracking kernels in flight (0: no limit,
        default 2); takes effect at the next launch."""
        self.plan.set_concurrency(max_concurrent)

    def run(self):
        self.launch()
        return self.wait()

    def results(self, i: int):
        """(lengths int32 [nsl], seed_index int32 [nsl], points float32 [npts, 3]) of subject i."""
        return self.trackers[i].handles[0].fetch()

    def streamlines(self, i: int):
        """Subject i's streamlines as a list of [len, 3] float32 arrays (seed order)."""
        L, _, P = self.results(i)
        return np.split(P, np.cumsum(L)[:-1]) if len(L) else []

    def close(self):
        if getattr(self, "plan", None) is not None:
            self.plan.close()
            self.plan = None
        for t, _ in getattr(self, "_seeds", []):
            t.close()
        self._seeds = []

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False
