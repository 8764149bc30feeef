"""PTT data preparation on the GPU (csl_ptt_prepare, PttDirectionGetter.prepare_data)
against the host computation the reference runs (cu_direction_getters.py:531-625,
restated in PttDirectionGetter.prepare_data_host with numpy and a KD-tree):

  * the tiled, clipped, masked, normalised texture data identical, bit for bit;
  * the 128^3 nearest-vertex LUT identical except at exact distance ties
    (|d1 - d2| <= 1e-12 between the two candidates), which must be fewer than
    1 in 10,000 grid points -- apart from antipodal pairs when the sphere is
    symmetric: there a vertex and its antipode are always at the same
    distance (+-v), the KD-tree over [v; -v] picks either copy and the GPU
    the lower index, and both address the same direction;
  * with the sphere symmetric and with a float64 threshold as well;
  * tracking through the Tracker API on the GPU-prepared data equals tracking
    on the host-prepared data when the LUTs agree everywhere.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _lut_ties_ok(lut_gpu, lut_host, verts, res, symm):
    bad = np.nonzero(lut_gpu.ravel() != lut_host.ravel())[0]
    if len(bad) == 0:
        return 0
    c = np.linspace(-1, 1, res)
    i, j, k = np.unravel_index(bad, (res, res, res))
    g = np.stack([c[i], c[j], c[k]], axis=1)
    v = verts.astype(np.float64)
    a = v[lut_gpu.ravel()[bad].astype(int)]
    b = v[lut_host.ravel()[bad].astype(int)]
    da = ((g - a) ** 2).sum(1)
    db = ((g - b) ** 2).sum(1)
    if symm:
        da = np.minimum(da, ((g + a) ** 2).sum(1))
        db = np.minimum(db, ((g + b) ** 2).sum(1))
    assert np.all(np.abs(da - db) <= 1e-12), np.abs(da - db).max()
    if symm:  # antipodal pairs are the same direction
        return int((np.abs(a + b).max(axis=1) > 1e-6).sum())
    return len(bad)


@pytest.mark.parametrize("symm,thr", [(False, 0.1), (True, np.float64(0.2))])
def test_ptt_prepare_matches_host(symm, thr):
    from gpustreamlines_b200 import PttDirectionGetter
    from oracle import cases

    inp = cases.inputs("ptt_s")
    g = PttDirectionGetter()
    tiled = g.prepare_data(inp["dataf"], inp["stop_map"], thr, inp["vertices"], symm).numpy()
    lut = g._lut_dev.numpy()
    h = PttDirectionGetter()
    tiled_h = h.prepare_data_host(inp["dataf"].copy(), inp["stop_map"], thr, inp["vertices"], symm)
    assert (g.nx, g.ny, g.nz, g.log2_x, g.log2_y) == (h.nx, h.ny, h.nz, h.log2_x, h.log2_y)
    assert tiled.shape == tiled_h.shape
    assert np.array_equal(tiled, tiled_h)
    nbad = _lut_ties_ok(lut, h.sphere_vertices_lut_h, inp["vertices"], g.odf_lut_res, symm)
    assert nbad <= 1e-4 * lut.size, nbad


def test_tracking_on_gpu_prepared_data():
    from gpustreamlines_b200 import PttDirectionGetter, Tracker, io
    from oracle import cases
    from test_gpu_parity import _handle

    name = "ptt_s"
    inp = cases.inputs(name)
    c = inp["case"]
    seeds = cases.seeds(name, 300, seed=71)
    h = _handle(name, inp=inp)
    h.propagate(seeds)
    L0, S0, P0 = h.fetch()
    h.close()
    lay = cases.ptt_layout(name)
    with Tracker(PttDirectionGetter(), inp["dataf"], inp["stop_map"], float(np.float32(c["fa_thr"])),
                 inp["vertices"], inp["edges"], max_angle=float(np.float32(math.radians(c["max_angle"]))),
                 step_size=float(np.float32(c["step"])), chunk_size=1000) as tr:
        same_lut = np.array_equal(tr.dg._lut_dev.numpy(), lay["lut"])
        sft = tr.generate_sft(seeds, io.RefImage(np.eye(4), inp["stop_map"].shape))
    L1 = np.asarray(sft.streamlines._lengths)
    P1 = np.asarray(sft.streamlines._data)
    assert len(L1) == len(L0)
    if same_lut:
        assert np.array_equal(L1, L0) and np.array_equal(P1, P0)
