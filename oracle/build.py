"""Recipe: build the C oracle (``oracle/liboracle.so``) and the test probes.

TEST INFRASTRUCTURE ONLY.  The oracle is plain C compiled with gcc (OpenMP
over seeds, no floating-point contraction: fused multiply-adds appear only as
explicit ``fmaf`` calls, where the reference's CUDA compiler contracts).
``tests/_probe.so`` holds GPU probes the tests use to pin the oracle.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "liboracle.so")
PROBE_SRC = os.path.join(ROOT, "tests", "csrc", "probe.cu")
PROBE = os.path.join(ROOT, "tests", "_probe.so")


def _newer(a, b):
    return not os.path.exists(b) or os.path.getmtime(a) > os.path.getmtime(b)


def build(force=False):
    src = os.path.join(HERE, "oracle.c")
    if force or _newer(src, LIB):
        subprocess.run(["gcc", "-O2", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared", src,
                        "-o", LIB, "-lm"], check=True)
    if force or _newer(PROBE_SRC, PROBE):
        subprocess.run(["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3",
                        "--use_fast_math", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                        PROBE_SRC, "-o", PROBE], check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
