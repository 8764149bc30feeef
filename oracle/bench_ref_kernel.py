"""Time the REFERENCE's own kernels on the benchmark workloads.

TEST/MEASUREMENT INFRASTRUCTURE ONLY (GPU).  Runs oracle/_ref/ref_prob_full.so
or ref_ptt_full.so (the reference's getNumStreamlines*_k +
genStreamlinesMerge*_k compiled from its sources for sm_100a, launched with its
own block shape (32, 2)) on the same phantom, PMF / ODF and seeds as
``bench.py --getter prob`` / ``--getter ptt``, and prints one JSON line with
CUDA-event kernel times and tracking steps/s (PTT: also sub-steps/s).  The
reference processes the seeds in chunks (its default 25,000 per GPU,
cu_tractography.py:55) because its padded output needs nSlines x 1002 x 12 B;
pass --chunk to change.

Usage: python -m oracle.bench_ref_kernel [--getter prob|ptt] [--seeds N] [--chunk M]
"""

from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seeds", type=int, default=1_000_000)
    ap.add_argument("--chunk", type=int, default=100_000)
    ap.add_argument("--getter", default="prob", choices=["prob", "ptt"])
    a = ap.parse_args()
    from bench import build_workload
    from oracle import api, cases

    ph, sph, pmf, seeds = build_workload(0, a.seeds, a.getter)
    name = f"{a.getter}_full"
    ptt = None
    if a.getter == "ptt":
        from gpustreamlines_b200.direction_getters import PttDirectionGetter

        inp = dict(stop_map=np.ascontiguousarray(ph.fa, dtype=np.float32),
                   vertices=np.ascontiguousarray(sph.vertices, dtype=np.float32),
                   edges=np.ascontiguousarray(sph.edges, dtype=np.int32))
        dg = PttDirectionGetter()
        tiled = dg.prepare_data_host(pmf, inp["stop_map"], np.float32(0.1), inp["vertices"], False)
        ptt = dict(tiled=tiled, lut=dg.sphere_vertices_lut_h, res=dg.odf_lut_res)
    else:
        inp = cases.inputs(name)
        assert inp["dataf"].shape == pmf.shape
    ref = api.Reference(name)
    p1 = p2 = 0.0
    steps = nsl = 0
    for s in range(0, len(seeds), a.chunk):
        chunk = seeds[s:s + a.chunk]
        counts, lens, _, _ = ref.track(inp, chunk, ptt=ptt, points=False)
        p1 += ref.last_ms[0]
        p2 += ref.last_ms[1]
        steps += int((lens - 1).sum())
        nsl += len(lens)
    extra = {}
    if a.getter == "ptt":
        frac = int(np.round(np.float32(0.5) / 0.025))
        extra = {"step_frac": frac, "sub_steps_per_s_pass2": steps * frac / (p2 / 1e3)}
    print(json.dumps({"impl": "reference CUDA kernels (sm_100a build)", "getter": a.getter, "seeds": a.seeds,
                      "chunk": a.chunk, "streamlines": nsl, "steps": steps,
                      "pass1_ms": p1, "pass2_ms": p2,
                      "steps_per_s_pass2": steps / (p2 / 1e3),
                      "steps_per_s_both": steps / ((p1 + p2) / 1e3), **extra}))


if __name__ == "__main__":
    main()
