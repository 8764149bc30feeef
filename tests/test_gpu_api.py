"""The drop-in API end to end on the GPU: ``Tracker(...).generate_sft`` /
``generate_trx`` (``cuslines/generic_tracker.py:79-172``) on real tracking,
checked against the C ABI's own results for the same chunks.

  * generate_sft with a chunk size smaller than the seed count equals the
    chunk-by-chunk C-ABI results (each chunk restarts its Philox indices at 0,
    as the reference's chunk loop does), in voxel space;
  * generate_trx holds the same streamlines in RAS mm (the reference image's
    affine applied), survives a TRX save / load round trip, and grows its
    memory map past the reference's size guesses;
  * the envelope sampler through the same API returns the same streamline
    count and seed order as the inverse-CDF sampler.
"""

from __future__ import annotations

import math
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _tracker(inp, c, **kw):
    from gpustreamlines_b200 import ProbDirectionGetter, Tracker

    return Tracker(ProbDirectionGetter(**kw), inp["dataf"], inp["stop_map"], float(np.float32(c["fa_thr"])),
                   inp["vertices"], inp["edges"], max_angle=float(np.float32(math.radians(c["max_angle"]))),
                   step_size=float(np.float32(c["step"])), chunk_size=500)


def _chunks_by_abi(inp, c, seeds, chunk):
    from test_gpu_parity import _handle

    h = _handle("prob_s", inp=inp)
    Ls, Ps = [], []
    for i in range(0, len(seeds), chunk):
        h.propagate(seeds[i:i + chunk], 0)
        L, S, P = h.fetch()
        Ls.append(L)
        Ps.append(P)
    h.close()
    return np.concatenate(Ls), np.concatenate(Ps)


def test_generate_sft_and_trx(tmp_path):
    from gpustreamlines_b200 import io
    from oracle import cases

    inp = cases.inputs("prob_s")
    c = inp["case"]
    seeds = cases.seeds("prob_s", 1300, seed=51)
    L0, P0 = _chunks_by_abi(inp, c, seeds, 500)
    aff = np.array([[2.0, 0, 0, -80.0], [0, 2.0, 0, -110.0], [0, 0, 2.0, -70.0], [0, 0, 0, 1]])
    ref = io.RefImage(aff, inp["stop_map"].shape)
    with _tracker(inp, c) as tr:
        sft = tr.generate_sft(seeds, ref)
        assert np.array_equal(np.asarray(sft.streamlines._lengths), L0)
        assert np.array_equal(np.asarray(sft.streamlines._data), P0)
        trx = tr.generate_trx(seeds, ref)
    n = len(trx)
    assert n == len(L0)
    s = trx.streamlines
    assert np.array_equal(np.asarray(s._lengths[:n]), L0)
    world = io.apply_affine(aff, P0.astype(np.float64)).astype(np.float32)
    assert np.allclose(np.asarray(s._data[:len(P0)]), world, atol=1e-4)
    path = os.path.join(tmp_path, "t.trx")
    io.save_trx(trx, path)
    hdr, seq = io.load_trx(path)
    assert hdr["NB_STREAMLINES"] == n and hdr["NB_VERTICES"] == len(P0)
    assert np.array_equal(np.asarray(seq._lengths), L0)
    assert np.allclose(np.asarray(seq._data), world, atol=1e-4)
    trx.close()


def test_envelope_sampler_through_api():
    from gpustreamlines_b200 import io
    from oracle import cases

    inp = cases.inputs("prob_s")
    c = inp["case"]
    seeds = cases.seeds("prob_s", 800, seed=52)
    ref = io.RefImage(np.eye(4), inp["stop_map"].shape)
    out = []
    for sampler in ("inverse_cdf", "envelope"):
        with _tracker(inp, c, sampler=sampler) as tr:
            sft = tr.generate_sft(seeds, ref)
            out.append((np.asarray(sft.streamlines._lengths), tr.seed_propagator.sline_seeds[0]))
    assert len(out[0][0]) == len(out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
