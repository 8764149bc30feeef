"""The allocation-free entry point (csl_track_noalloc) against csl_propagate.

For callers that cannot allocate device memory while tracking (a host
framework's pool owns it, or allocation after start-up is forbidden), the
library offers csl_track_noalloc: a tracking-kernel variant whose scratch is a
static device array.  This test calls it through the C ABI twice in a row on
the same buffers and checks both calls against the compacted output of the
regular entry point, bit for bit, for the probabilistic, bootstrap (CSA,
per-warp fit, truncated peak lists, non-zero Philox index base) and PTT getters.
The file is named to be collected last.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name,nseeds,maxp,base", [
    ("prob_s", 400, 8, 0),
    # bootstrap: the peak list copied from shared memory, max_peaks below some
    # seeds' peak counts, and a non-zero Philox index base
    ("csa_s", 120, 1, 7),
    # PTT: the initial-frame search and its frames in the static scratch's warp buffers
    ("ptt_s", 150, 8, 0),
])
def test_noalloc_matches_propagate_on_two_calls(name, nseeds, maxp, base):
    import torch

    from oracle import cases
    from test_gpu_parity import _handle

    h = _handle(name)
    seeds = cases.seeds(name, nseeds, seed=13)
    h.propagate(seeds, rng_index_base=base)
    L, S, P = h.fetch()
    # peaks per seed of that batch (bootstrap pass 1 depends on the Philox base)
    counts_ref = np.bincount(S, minlength=len(seeds)).astype(np.int32)
    if maxp == 1:
        assert (counts_ref > maxp).any(), "the case should truncate some seeds' peak lists"
    n = len(seeds)
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
        h.track_noalloc(sd.data_ptr(), n, base, maxp, counts.data_ptr(), lens.data_ptr(),
                        pts.data_ptr(), stream.cuda_stream)
        torch.cuda.synchronize()
        c = counts.cpu().numpy()
        l = lens.cpu().numpy().reshape(n, maxp)
        p = pts.cpu().numpy()
        assert np.array_equal(c, counts_ref)
        for s in range(n):
            for k in range(min(c[s], maxp)):
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
