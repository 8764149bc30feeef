"""The reference's command-line script (run_gpu_streamlines.py) runs unchanged
on this package: `cuslines` resolves to gpustreamlines_b200, and its DIPY,
nibabel and trx-python imports (absent here) resolve to small stand-ins that
serve the synthetic phantom.  The script's own --cache-dir option supplies
the FA map and the ODF, so its DIPY model fits are not needed.

The device is replaced by a recording handle that returns deterministic
streamlines (this suite has no GPU); the test checks what crosses the
boundary -- the tracker parameters the script sets (angles converted to
radians, step, thresholds, chunking, sphere) and the seeds of every chunk --
and that the script's TRX and TRK outputs hold exactly the handle's
streamlines.  Real tracking through the same calls is covered on the GPU by
tests/test_gpu_api.py.  Skipped when the reference checkout is not present
($CSL_REFERENCE_ROOT, else the checkout's usual place).
"""

from __future__ import annotations

import math
import os
import runpy
import sys
import types

import numpy as np
import pytest

REF = os.environ.get("CSL_REFERENCE_ROOT", "/root/reference")
SCRIPT = os.path.join(REF, "run_gpu_streamlines.py")


class _Img:
    def __init__(self, data, affine):
        self._d = data
        self.affine = affine
        self.shape = data.shape

    def get_fdata(self):
        return self._d.astype(np.float64)


class _RecordingHandle:
    """Stand-in for gpustreamlines_b200._lib.Handle: records, returns fixed streamlines."""

    calls = []

    def __init__(self, params, inputs, device, keepalive=()):
        self.params = params
        self.device = device
        _RecordingHandle.calls.append(("create", {f: getattr(params, f) for f, _ in params._fields_}))

    def propagate(self, seeds, rng_index_base=0, stream=None):
        seeds = np.asarray(seeds, np.float32)
        _RecordingHandle.calls.append(("propagate", seeds.copy(), rng_index_base))
        # two streamlines per seed: the seed and one step along +-x
        n = len(seeds)
        self.L = np.full(2 * n, 2, np.int32)
        self.S = np.repeat(np.arange(n, dtype=np.int32), 2)
        pts = []
        for s in seeds:
            pts += [s, s + [0.5, 0, 0], s, s - [0.5, 0, 0]]
        self.P = np.asarray(pts, np.float32).reshape(-1, 3)

    def fetch(self):
        return self.L, self.S, self.P

    def close(self):
        pass


def _stubs(ph, sph, dwi_img, wm_img):
    from gpustreamlines_b200 import io

    mods = {}

    def mod(name, **attrs):
        m = types.ModuleType(name)
        m.__dict__.update(attrs)
        mods[name] = m
        return m

    class _Gtab:
        def __init__(self, bvals=None, bvecs=None):
            self.bvals = np.asarray(bvals)
            self.bvecs = np.asarray(bvecs)
            self.b0s_mask = self.bvals <= 50

    class _Any:
        def __init__(self, *a, **k):
            raise AssertionError("the GPU path must not construct DIPY models")

    def random_seeds_from_mask(mask, seeds_count=1, seed_count_per_voxel=True, random_seed=None, affine=None):
        from gpustreamlines_b200.phantom import seeds_from_mask

        return seeds_from_mask(np.asarray(mask, np.float32), seeds_count, threshold=0.5,
                               seed=0 if random_seed is None else random_seed)

    class HemiSphere:
        pass

    mod("dipy")
    mod("dipy.reconst")
    mod("dipy.reconst.dti", TensorModel=_Any)
    mod("dipy.core")
    mod("dipy.core.gradients", gradient_table=lambda bvals=None, bvecs=None: _Gtab(bvals, bvecs),
        unique_bvals_magnitude=lambda b: np.unique(np.asarray(b)))
    mod("dipy.data", get_sphere=lambda name="repulsion724": sph, small_sphere=sph, HemiSphere=HemiSphere,
        get_fnames=lambda name=None: ("dwi.nii", "dwi.bval", "dwi.bvec"),
        read_stanford_pve_maps=lambda: (wm_img, wm_img, wm_img))
    mod("dipy.direction", BootDirectionGetter=_Any, ProbabilisticDirectionGetter=_Any, PTTDirectionGetter=_Any)
    mod("dipy.io", read_bvals_bvecs=lambda a, b: (ph.bvals, ph.bvecs))
    mod("dipy.io.stateful_tractogram", Space=io.Space, StatefulTractogram=io.StatefulTractogram)
    mod("dipy.io.streamline", save_tractogram=io.save_tractogram)
    mod("dipy.reconst.csdeconv", ConstrainedSphericalDeconvModel=_Any, auto_response_ssst=_Any)
    mod("dipy.reconst.shm", CsaOdfModel=_Any, OpdtModel=_Any)
    mod("dipy.tracking")
    mod("dipy.tracking.utils", random_seeds_from_mask=random_seeds_from_mask)
    mod("dipy.tracking.local_tracking", LocalTracking=_Any)
    mod("dipy.tracking.stopping_criterion", ThresholdStoppingCriterion=lambda fa, thr: None)
    mod("nibabel", load=lambda path: dwi_img)
    mod("nibabel.orientations", aff2axcodes=lambda aff: ("R", "A", "S"))
    mod("trx")
    mod("trx.io", save=io.save_trx)
    import gpustreamlines_b200

    mods["cuslines"] = gpustreamlines_b200
    return mods


@pytest.mark.skipif(not os.path.isfile(SCRIPT), reason="reference checkout not present")
@pytest.mark.parametrize("dg,write", [("prob", "trx"), ("ptt", "trk")])
def test_reference_cli_runs_unchanged(tmp_path, monkeypatch, dg, write):
    from gpustreamlines_b200 import _lib, direction_getters, io, tracker
    from gpustreamlines_b200.phantom import make_phantom, odf_volume
    from gpustreamlines_b200.sphere import get_sphere

    ph = make_phantom((12, 14, 10), seed=3)
    sph = get_sphere("repulsion724")
    aff = np.diag([2.0, 2.0, 2.0, 1.0])
    dwi_img = _Img(ph.dwi, aff)
    wm_img = _Img((ph.fa > 0.3).astype(np.float32), aff)
    cache = tmp_path / "cache"
    cache.mkdir()
    np.save(cache / "fa.npy", ph.fa.astype(np.float64))
    np.save(cache / "csd_odf.npy", odf_volume(ph, sph).astype(np.float64))

    for name, m in _stubs(ph, sph, dwi_img, wm_img).items():
        monkeypatch.setitem(sys.modules, name, m)
    _RecordingHandle.calls = []
    monkeypatch.setattr(_lib, "Handle", _RecordingHandle)
    monkeypatch.setattr(tracker, "device_count", lambda: 1)
    if dg == "ptt":
        # the GPU data preparation runs on the host restatement (no device here)
        monkeypatch.setattr(direction_getters.PttDirectionGetter, "prepare_data",
                            direction_getters.PttDirectionGetter.prepare_data_host)
    out = tmp_path / "out"
    argv = ["run_gpu_streamlines.py", "hardi", "hardi", "hardi", "hardi", "hardi", "--dg", dg, "--nseeds", "150",
            "--chunk-size", "64", "--max-angle", "40", "--step-size", "0.25", "--fa-threshold", "0.15",
            "--cache-dir", str(cache), "--output-prefix", str(out), "--write-method", write, "--seed-seed", "5"]
    monkeypatch.setattr(sys, "argv", argv)
    runpy.run_path(SCRIPT, run_name="__main__")

    creates = [c for c in _RecordingHandle.calls if c[0] == "create"]
    props = [c for c in _RecordingHandle.calls if c[0] == "propagate"]
    assert len(creates) == 1
    p = creates[0][1]
    assert p["model"] == (_lib.MODEL_PROB if dg == "prob" else _lib.MODEL_PTT)
    assert abs(p["max_angle"] - float(np.float32(math.radians(40)))) < 1e-7
    assert abs(p["step_size"] - 0.25) < 1e-7
    assert abs(p["tc_threshold"] - float(np.float32(0.15))) < 1e-7
    assert abs(p["min_separation_angle"] - float(np.float32(math.radians(45)))) < 1e-7
    assert p["nvertices"] == len(sph.vertices)
    # chunks of 64 seeds, Philox indices restarting per chunk as in the reference
    assert [len(c[1]) for c in props] == [64, 64, 22]
    assert all(c[2] == 0 for c in props)
    seeds = np.concatenate([c[1] for c in props])
    if write == "trx":
        hdr, seq = io.load_trx(str(out) + ".trx")
        assert hdr["NB_STREAMLINES"] == 2 * len(seeds)
        want = np.concatenate([np.stack([s, s + [0.5, 0, 0], s, s - [0.5, 0, 0]]) for s in seeds]).astype(np.float64)
        assert np.allclose(np.asarray(seq._data), io.apply_affine(aff, want), atol=1e-4)
    else:
        hdr, seq = io.load_trk(str(out) + ".trk")
        assert len(seq) == 2 * len(seeds)
