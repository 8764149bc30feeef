"""The allocation-free entry point (csl_track_noalloc) against csl_propagate.

For callers that cannot allocate device memory while tracking (a host
framework's pool owns it, or allocation after start-up is forbidden), the
library offers csl_track_noalloc: a tracking-kernel variant whose scratch is a
static device array.  This test calls it through the C ABI twice in a row on
the same buffers and checks both calls against the compacted output of the
regular entry point, bit for bit (the bar of the probabilistic parity tests).
The file is named to be collected last.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_noalloc_matches_propagate_on_two_calls():
    import torch

    from oracle import cases
    from test_gpu_parity import _handle

    h = _handle("prob_s")
    seeds = cases.seeds("prob_s", 400, seed=13)
    h.propagate(seeds)
    L, S, P = h.fetch()
    counts_ref, _, _ = h.seed_peaks(seeds, 64)
    n, maxp = len(seeds), 8
    dev = torch.device("cuda:0")
    sd = torch.from_numpy(seeds).to(dev)
    counts = torch.empty(n, dtype=torch.int32, device=dev)
    lens = torch.empty(n * maxp, dtype=torch.int32, device=dev)
    pts = torch.empty((n * maxp, 2 * 501, 3), dtype=torch.float32, device=dev)
    off = np.concatenate([[0], np.cumsum(L)])
    sl_off = np.concatenate([[0], np.cumsum(counts_ref)])
    stream = torch.cuda.current_stream(dev)
    for _ in range(2):
        counts.fill_(-1)
        lens.fill_(-1)
        pts.fill_(np.nan)
        h.track_noalloc(sd.data_ptr(), n, 0, maxp, counts.data_ptr(), lens.data_ptr(),
                        pts.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        c = counts.cpu().numpy()
        l = lens.cpu().numpy().reshape(n, maxp)
        p = pts.cpu().numpy()
        assert np.array_equal(c, counts_ref)
        assert (c <= maxp).all()
        for s in range(n):
            for k in range(c[s]):
                j = sl_off[s] + k
                assert l[s, k] == L[j]
                assert np.array_equal(p[s * maxp + k, :L[j]], P[off[j]:off[j + 1]])
    h.close()


def test_noalloc_rejects_sizes_beyond_its_limits():
    from test_gpu_parity import _handle

    h = _handle("prob_s")
    with pytest.raises(ValueError, match="max_peaks"):
        h.track_noalloc(0, 10, 0, 0, 0, 0, 0)
    with pytest.raises(ValueError, match="max_peaks"):
        h.track_noalloc(0, 10, 0, 33, 0, 0, 0)
    h.close()
