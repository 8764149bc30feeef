"""Build the sm_100a tracking library in-tree: ``gpustreamlines_b200/_csl.so``.

Usage: python -m gpustreamlines_b200.build [--force] [-v]
Flags mirror the reference's NVRTC options (``use_fast_math``, C++17, -O3;
``cuslines/cuda_python/cu_direction_getters.py:111-125``) so that the same
source-level float expressions compile to the same arithmetic.  Each source
is compiled to its own object (in parallel, under ``_build/``) and the
objects are linked into one shared library.
"""

from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_csl.so")
OBJ = os.path.join(HERE, "_build")
SOURCES = ["kernels.cu", "boot_batch.cu", "odf_gemm.cu", "compress.cu", "mlp.cu", "dti.cu", "multi.cu",
           "capi.cu", "noalloc.cu", "envelope.cu", "ptt_prep.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [*ARCH, "-O3", "--use_fast_math", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-diag-suppress", "20281"]


def _deps(path: str, seen=None) -> set:
    """The file and the local headers it includes, transitively."""
    seen = set() if seen is None else seen
    path = os.path.normpath(path)
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path) as f:
        for line in f:
            line = line.strip()
            if line.startswith("#include \""):
                _deps(os.path.join(os.path.dirname(path), line.split('"')[1]), seen)
    return seen


def _obj(src: str) -> str:
    return os.path.join(OBJ, src.replace(".cu", ".o"))


def _stale_obj(src: str) -> bool:
    o = _obj(src)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    return any(os.path.getmtime(d) > t for d in _deps(os.path.join(CSRC, src)))


def _compile(src: str, verbose: bool) -> str:
    cmd = ["nvcc", *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", _obj(src)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n" + r.stderr[-6000:])
    return r.stderr if verbose else ""


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(OBJ, exist_ok=True)
    todo = [s for s in SOURCES if force or verbose or _stale_obj(s)]
    if todo:
        with ThreadPoolExecutor(len(todo)) as ex:
            for log in ex.map(lambda s: _compile(s, verbose), todo):
                if log:
                    print(log)
    objs = [_obj(s) for s in SOURCES]
    if todo or not os.path.exists(OUT) or any(os.path.getmtime(o) > os.path.getmtime(OUT) for o in objs):
        r = subprocess.run(["nvcc", *ARCH, "-shared", *objs, "-o", OUT], capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stderr[-6000:])
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
