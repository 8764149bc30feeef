"""Parity cases shared by the oracle builds and the tests -- TEST INFRASTRUCTURE ONLY.

Each case fixes a phantom, a sphere and the tracker parameters.  The
reference takes volume shapes and thresholds as compile-time macros
(``cuslines/cuda_python/cu_direction_getters.py:70-107``), so
``oracle/build_ref.py`` compiles one reference library per case with the
macro strings formatted exactly as the reference formats them
(``str(float(np.float32(x)))``).
"""

from __future__ import annotations

import functools
import math

import numpy as np

from gpustreamlines_b200 import shm
from gpustreamlines_b200.phantom import make_phantom, odf_volume, seeds_from_mask
from gpustreamlines_b200.sphere import get_sphere

CASES = {
    # probabilistic getter on a small phantom (step 0.5, 45 deg cone: the 1M-seed benchmark's parameters)
    "prob_s": dict(model="PROB", shape=(24, 28, 20), phantom_seed=7, max_angle=45.0,
                   step=0.5, fa_thr=0.1, rel=0.25, min_sep=45.0, rng_seed=0),
    # bootstrap CSA, sh_order 6 (the 1000-seed bootstrap benchmark's parameters)
    "csa_s": dict(model="CSA", shape=(24, 28, 20), phantom_seed=7, max_angle=60.0, step=0.5,
                  fa_thr=0.1, rel=0.25, min_sep=45.0, rng_seed=0, sh_order=6),
    # bootstrap OPDT, sh_order 4 (the reference CLI's default model)
    "opdt_s": dict(model="OPDT", shape=(24, 28, 20), phantom_seed=7, max_angle=60.0, step=0.5,
                   fa_thr=0.1, rel=0.25, min_sep=45.0, rng_seed=0, sh_order=4),
    # parallel transport tractography on the small phantom's ODF
    "ptt_s": dict(model="PTT", shape=(24, 28, 20), phantom_seed=7, max_angle=60.0, step=0.5,
                  fa_thr=0.1, rel=0.25, min_sep=45.0, rng_seed=0),
    # probabilistic getter with other tracker parameters: finer step, narrower
    # cone, lower relative peak threshold, symmetric-sphere peak separation,
    # higher stop threshold and a non-zero generator seed
    "prob_v": dict(model="PROB", shape=(24, 28, 20), phantom_seed=7, max_angle=30.0,
                   step=0.25, fa_thr=0.2, rel=0.1, min_sep=30.0, rng_seed=77, sphere_symm=1),
    # probabilistic getter at the full 81x106x76x724 size
    "prob_full": dict(model="PROB", shape=(81, 106, 76), phantom_seed=1234, max_angle=45.0,
                      step=0.5, fa_thr=0.1, rel=0.25, min_sep=45.0, rng_seed=0),
    # PTT at the full 81x106x76 size (timing of the reference's PTT kernels)
    "ptt_full": dict(model="PTT", shape=(81, 106, 76), phantom_seed=1234, max_angle=60.0, step=0.5,
                     fa_thr=0.1, rel=0.25, min_sep=45.0, rng_seed=0),
    # bootstrap CSA at the full 81x106x76x160 size, sh_order 8 (the batched-fit
    # benchmark's parameters); statistics only, so no reference library is built for it
    "csa_full": dict(model="CSA", shape=(81, 106, 76), phantom_seed=1234, max_angle=60.0, step=0.5,
                     fa_thr=0.1, rel=0.25, min_sep=45.0, rng_seed=0, sh_order=8, ref=False),
}

MODEL_ID = {"OPDT": 0, "CSA": 1, "PROB": 2, "PTT": 3}
MAX_SLINE_LEN = 501


def f32s(x):
    """The reference's macro formatting of a float parameter."""
    return str(float(np.float32(x)))


@functools.lru_cache(maxsize=4)
def phantom(name):
    c = CASES[name]
    with_dwi = c["model"] in ("CSA", "OPDT") or c["shape"] != (81, 106, 76)
    return make_phantom(c["shape"], seed=c["phantom_seed"], with_dwi=with_dwi)


@functools.lru_cache(maxsize=4)
def inputs(name):
    """Host arrays of a case: dataf, stop map, sphere, getter matrices."""
    c = CASES[name]
    ph = phantom(name)
    sph = get_sphere("repulsion724")
    out = dict(case=c, phantom=ph, vertices=np.ascontiguousarray(sph.vertices, dtype=np.float32),
               edges=np.ascontiguousarray(sph.edges, dtype=np.int32),
               stop_map=np.ascontiguousarray(ph.fa, dtype=np.float32), sphere=sph)
    if c["model"] in ("CSA", "OPDT"):
        prep = (shm.prepare_csa if c["model"] == "CSA" else shm.prepare_opdt)(
            ph.gtab, sph, sh_order_max=c["sh_order"], sh_lambda=0.006, min_signal=1)
        out["dataf"] = np.ascontiguousarray(ph.dwi, dtype=np.float32)
        for k in ("H", "R", "delta_b", "delta_q", "sampling_matrix"):
            out[k] = np.ascontiguousarray(prep[k], dtype=np.float32)
        out["b0s_mask"] = np.ascontiguousarray(prep["b0s_mask"], dtype=np.int32)
        out["min_signal"] = np.float32(1.0)
    else:
        out["dataf"] = np.ascontiguousarray(odf_volume(ph, sph), dtype=np.float32)
    return out


def seeds(name, n, seed=0):
    return seeds_from_mask(phantom(name).fa, n, threshold=0.3, seed=seed).astype(np.float32)


def macros(name):
    """Macro set of the reference build for this case (cu_direction_getters.py:70-107)."""
    c = CASES[name]
    inp = inputs(name)
    X, Y, Z = c["shape"]
    T = inp["dataf"].shape[3]
    boot = c["model"] in ("CSA", "OPDT")
    samplm = inp["sampling_matrix"].shape[0] if boot else T
    m = {
        "DIMX": str(X), "DIMY": str(Y), "DIMZ": str(Z), "DIMT": str(T),
        "N32DIMT": str(((T + 31) // 32) * 32),
        "STEP_SIZE": f32s(c["step"]),
        "MAX_ANGLE": f32s(math.radians(c["max_angle"])),
        "TC_THRESHOLD": f32s(c["fa_thr"]),
        "RELATIVE_PEAK_THRESH": f32s(c["rel"]),
        "MIN_SEPARATION_ANGLE": f32s(math.radians(c["min_sep"])),
        "RNG_SEED": str(int(c["rng_seed"])),
        "SAMPLM_NR": str(int(samplm)),
        "NUM_EDGES": str(int(len(inp["edges"]))),
        "SPHERE_SYMM": str(int(c.get("sphere_symm", 0))),
        "EXCESS_ALLOC_FACT": "2", "MAX_SLINES_PER_SEED": "10",
        "MAX_SLINE_LEN": str(MAX_SLINE_LEN), "PMF_THRESHOLD_P": str(float(0.05)),
        "REAL_SIZE": "4", "THR_X_BL": "64", "THR_X_SL": "32",
        "REF_MODEL": str(MODEL_ID[c["model"]]),
    }
    if c["model"] == "PTT":
        p = ptt_tiles(T)
        max_angle32 = np.float32(math.radians(c["max_angle"]))
        step32 = np.float32(c["step"])
        m.update({
            "LOG2_X": str(p["log2_x"]), "LOG2_Y": str(p["log2_y"]),
            "WIDTH_MASK": str(p["nx"] - 1), "HEIGHT_MASK": str(p["ny"] - 1),
            "PROBE_QUALITY": str(float(8)), "PROBE_STEP_SIZE": str(float(0.25)),
            "STEP_FRAC": str(int(np.round(step32 / 0.025))),
            "MAX_CURVATURE": str(float(8.0 * np.sin(max_angle32 / 2.0))),
        })
    else:
        for k in ("LOG2_X", "LOG2_Y", "WIDTH_MASK", "HEIGHT_MASK", "PROBE_STEP_SIZE",
                  "MAX_CURVATURE", "PROBE_QUALITY", "STEP_FRAC"):
            m[k] = "0"
    return m


def ptt_tiles(T):
    """Power-of-two tile counts of the PTT texture's vertex axis (the getter's
    prepare_data rule), without building the texture."""
    nx = ny = nz = 1
    while nx * ny * nz < T:
        if nx <= ny and nx <= nz:
            nx *= 2
        elif ny <= nx and ny <= nz:
            ny *= 2
        else:
            nz *= 2
    return dict(nx=nx, ny=ny, nz=nz, log2_x=int(math.log2(nx)), log2_y=int(math.log2(ny)))


@functools.lru_cache(maxsize=2)
def ptt_layout(name):
    """Tiled texture + LUT exactly as the PTT getter prepares them."""
    from gpustreamlines_b200.direction_getters import PttDirectionGetter

    c = CASES[name]
    inp = inputs(name)
    dg = PttDirectionGetter()
    tiled = dg.prepare_data_host(inp["dataf"].copy(), inp["stop_map"], np.float32(c["fa_thr"]),
                            inp["vertices"], False)
    return dict(tiled=tiled, lut=dg.sphere_vertices_lut_h, log2_x=dg.log2_x, log2_y=dg.log2_y,
                nx=dg.nx, ny=dg.ny, nz=dg.nz, res=dg.odf_lut_res)
