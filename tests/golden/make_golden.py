"""Generate the golden fixtures of tests/golden/ on a B200 (GPU required).

The fixtures pin the CPU oracle to the reference and to the CUDA toolkit:
  curand.npz      curand() / curand_uniform() / curand_normal() streams for
                  curand_init(seed, subsequence, offset) as the reference calls it
  fastmath.npz    __cosf of the angle thresholds the parity cases use
  dot.npz         the reference's 3-term dot expression compiled with --use_fast_math
  tex.npz         hardware-filtered stop-map samples (border -1) at random points
  ref_<case>.npz  the reference's own kernels (oracle/_ref) on a few hundred seeds:
                  pass-1 counts, streamline seeds, lengths and points (bootstrap:
                  pass-1 counts only)

Usage: python tests/golden/make_golden.py OUTDIR
"""

from __future__ import annotations

import math
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import probe  # noqa: E402
from oracle import api, cases  # noqa: E402

CURAND_SUBSEQ = np.array([0, 1, 2, 31, 32, 33, 1000, 65537, (1 << 32) + 5, 123456789], dtype=np.uint64)
CURAND_OFFS = np.array([0, 1, 3, 4, 5, 17, 0, 2, 0, 9], dtype=np.uint64)
SEEDS_PER_CASE = {"prob_s": 300, "csa_s": 60, "opdt_s": 60, "ptt_s": 60}


def main(out):
    os.makedirs(out, exist_ok=True)
    for seed in (0, 1234):
        u, f, g = probe.curand(seed, CURAND_SUBSEQ, CURAND_OFFS, 24)
        np.savez_compressed(os.path.join(out, f"curand_{seed}.npz"), subseq=CURAND_SUBSEQ,
                            offs=CURAND_OFFS, u32=u, uniform=f, normal=g)
    angles = np.float32([math.radians(a) for a in (30.0, 45.0, 60.0, 90.0)])
    c, l = probe.fast(angles)
    np.savez_compressed(os.path.join(out, "fastmath.npz"), angle=angles, cos=c)
    rng = np.random.default_rng(5)
    a = rng.normal(size=(4000, 3)).astype(np.float32)
    b = rng.normal(size=(4000, 3)).astype(np.float32)
    np.savez_compressed(os.path.join(out, "dot.npz"), a=a, b=b, dot=probe.dot(a, b))
    inp = cases.inputs("prob_s")
    X, Y, Z = inp["stop_map"].shape
    pts = np.concatenate([
        rng.uniform([-1, -1, -1], [X + 1, Y + 1, Z + 1], (3000, 3)),
        cases.seeds("prob_s", 3000, seed=11)]).astype(np.float32)
    np.savez_compressed(os.path.join(out, "tex.npz"), pts=pts, val=probe.tex3d(inp["stop_map"], pts))
    for name, n in SEEDS_PER_CASE.items():
        ref = api.Reference(name)
        s = cases.seeds(name, n, seed=21)
        inp = cases.inputs(name)
        ptt = cases.ptt_layout(name) if inp["case"]["model"] == "PTT" else None
        counts, lens, sidx, pts = ref.track(inp, s, ptt=ptt)
        if lens is None:  # bootstrap: pass 1 only
            np.savez_compressed(os.path.join(out, f"ref_{name}.npz"), seeds=s, counts=counts)
            print(name, "pass-1 streamlines", int(counts.sum()))
            continue
        np.savez_compressed(os.path.join(out, f"ref_{name}.npz"), seeds=s, counts=counts, lens=lens,
                            sidx=sidx, pts=pts)
        print(name, "streamlines", len(lens), "points", len(pts))


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(ROOT, "tests", "golden"))
