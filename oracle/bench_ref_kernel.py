"""Time the REFERENCE's own probabilistic kernels on the benchmark workload.

TEST/MEASUREMENT INFRASTRUCTURE ONLY (GPU).  Runs oracle/_ref/ref_prob_full.so
(the reference's getNumStreamlinesProb_k + genStreamlinesMergeProb_k compiled
from its sources for sm_100a, launched with its own block shape (32, 2)) on
the same phantom, PMF and seeds as bench.py, and prints one JSON line with
CUDA-event kernel times and tracking steps/s.  The reference processes the
seeds in chunks (its default 25,000 per GPU, cu_tractography.py:55) because
its padded output needs nSlines x 1002 x 12 B; pass --chunk to change.

Usage: python -m oracle.bench_ref_kernel [--seeds 1000000] [--chunk 100000]
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
    a = ap.parse_args()
    from bench import build_workload
    from oracle import api, cases

    ph, sph, pmf, seeds = build_workload(0, a.seeds)
    inp = cases.inputs("prob_full")
    assert inp["dataf"].shape == pmf.shape
    ref = api.Reference("prob_full")
    p1 = p2 = 0.0
    steps = nsl = 0
    for s in range(0, len(seeds), a.chunk):
        chunk = seeds[s:s + a.chunk]
        counts, lens, _, _ = ref.track(inp, chunk, points=False)
        p1 += ref.last_ms[0]
        p2 += ref.last_ms[1]
        steps += int((lens - 1).sum())
        nsl += len(lens)
    print(json.dumps({"impl": "reference CUDA kernels (sm_100a build)", "seeds": a.seeds,
                      "chunk": a.chunk, "streamlines": nsl, "steps": steps,
                      "pass1_ms": p1, "pass2_ms": p2,
                      "steps_per_s_pass2": steps / (p2 / 1e3),
                      "steps_per_s_both": steps / ((p1 + p2) / 1e3)}))


if __name__ == "__main__":
    main()
