"""The reference's cross-backend benchmark script (webgpu/benchmark.py) runs
unchanged on this package as its "cuda" backend: `cuslines.cuda_python`
resolves to gpustreamlines_b200, and the script's DIPY, nibabel and
cuda-python imports resolve to small stand-ins that serve the synthetic
phantom (its tensor fit is DIPY preprocessing, outside the package).

As in test_cpu_cli, the device is replaced by a recording handle (no GPU in
this suite).  Checked: the tracker parameters the script sets (OPDT getter at
sh_order 4 with its sh_lambda and min_signal, 60 degree angle in radians, step,
thresholds, rng_seed 0, one chunk of 100,000), the seeds reaching the device,
and the script's own statistics (compute_metrics: streamline count, lengths,
commissural count) over the StatefulTractogram our generate_sft returns.
Skipped when the reference checkout is not present ($CSL_REFERENCE_ROOT, else
the checkout's usual place).
"""

from __future__ import annotations

import math
import os
import runpy
import sys
import types

import numpy as np
import pytest

from test_cpu_cli import REF, _Img, _RecordingHandle, _stubs

SCRIPT = os.path.join(REF, "cuslines", "webgpu", "benchmark.py")


@pytest.mark.skipif(not os.path.isfile(SCRIPT), reason="reference checkout not present")
def test_reference_benchmark_runs_unchanged(monkeypatch, capsys):
    import gpustreamlines_b200
    from gpustreamlines_b200 import _lib, tracker
    from gpustreamlines_b200.phantom import make_phantom
    from gpustreamlines_b200.sphere import get_sphere

    ph = make_phantom((12, 14, 10), seed=4)
    sph = get_sphere("repulsion724")
    aff = np.diag([2.0, 2.0, 2.0, 1.0])
    dwi_img = _Img(ph.dwi, aff)
    wm_img = _Img((ph.fa > 0.3).astype(np.float32), aff)
    mods = _stubs(ph, sph, dwi_img, wm_img)

    class _TensorFit:
        fa = ph.fa.astype(np.float64)

    class _TensorModel:
        def __init__(self, gtab, fit_method="WLS"):
            assert fit_method == "WLS"

        def fit(self, data, mask=None):
            return _TensorFit()

    mods["dipy.reconst.dti"].TensorModel = _TensorModel
    mods["dipy.data"].default_sphere = sph
    mods["cuslines.cuda_python"] = gpustreamlines_b200
    props = types.SimpleNamespace(name=b"B200 (recording stand-in)\x00")
    mods["cuda"] = types.ModuleType("cuda")
    mods["cuda.bindings"] = types.ModuleType("cuda.bindings")
    mods["cuda.bindings.runtime"] = types.ModuleType("cuda.bindings.runtime")
    mods["cuda.bindings.runtime"].cudaGetDeviceCount = lambda: (0, 1)
    mods["cuda.bindings.runtime"].cudaGetDeviceProperties = lambda dev: (0, props)
    mods["cuda.bindings"].runtime = mods["cuda.bindings.runtime"]
    mods["cuda"].bindings = mods["cuda.bindings"]
    for name, m in mods.items():
        monkeypatch.setitem(sys.modules, name, m)
    _RecordingHandle.calls = []
    monkeypatch.setattr(_lib, "Handle", _RecordingHandle)
    monkeypatch.setattr(tracker, "device_count", lambda: 1)
    monkeypatch.setattr(sys, "argv", ["benchmark.py", "--nseeds", "120", "--skip-cpu", "--backends", "cuda"])
    runpy.run_path(SCRIPT, run_name="__main__")

    creates = [c for c in _RecordingHandle.calls if c[0] == "create"]
    prop = [c for c in _RecordingHandle.calls if c[0] == "propagate"]
    assert len(creates) == 1 and len(prop) == 1  # chunk_size 100,000: one chunk
    p = creates[0][1]
    assert p["model"] == _lib.MODEL_OPDT
    assert p["delta_nr"] == 15  # sh_order 4
    assert abs(p["min_signal"] - 1.0) < 1e-12
    assert abs(p["max_angle"] - float(np.float32(math.radians(60)))) < 1e-7
    assert abs(p["step_size"] - 0.5) < 1e-7
    assert abs(p["tc_threshold"] - float(np.float32(0.1))) < 1e-7
    assert abs(p["relative_peak_thresh"] - 0.25) < 1e-7
    assert abs(p["min_separation_angle"] - float(np.float32(math.radians(45)))) < 1e-7
    assert p["rng_seed"] == 0
    seeds = prop[0][1]
    assert len(seeds) == 120 and prop[0][2] == 0
    # the script's own statistics over our StatefulTractogram
    out = capsys.readouterr().out
    assert f"-> {2 * len(seeds):,} streamlines" in out
    assert "CUDA" in out
