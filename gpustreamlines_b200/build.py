"""Build the sm_100a tracking library in-tree: ``gpustreamlines_b200/_csl.so``.

Usage: python -m gpustreamlines_b200.build
Flags mirror the reference's NVRTC options (``use_fast_math``, C++17, -O3;
``cuslines/cuda_python/cu_direction_getters.py:111-125``) so that the same
source-level float expressions compile to the same arithmetic.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_csl.so")
SOURCES = ["kernels.cu", "boot_batch.cu", "odf_gemm.cu", "compress.cu", "mlp.cu", "dti.cu", "multi.cu", "capi.cu", "noalloc.cu"]
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--use_fast_math", "-lineinfo",
              "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-diag-suppress", "20281"]


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "gpustreamlines_b200.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return OUT
    cmd = ["nvcc", *NVCC_FLAGS, *(os.path.join(CSRC, s) for s in SOURCES), "-o", OUT]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stderr[-6000:])
    if verbose:
        print(r.stderr)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
