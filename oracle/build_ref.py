"""Recipe: compile the REFERENCE's CUDA kernels from their own sources.

TEST INFRASTRUCTURE ONLY.  Compiles ``cuslines/cuda_c/generate_streamlines_cuda.cu``
(and the files it includes) where they lie under the read-only reference
checkout, wrapped by ``oracle/ref_launcher.cu``, once per parity case of
``oracle/cases.py`` (the reference takes shapes and thresholds as macros).
Outputs go to ``oracle/_ref/ref_<case>.so`` only; the sources are never
copied.  nvcc flags mirror the reference's NVRTC options
(``cu_direction_getters.py:111-125``: ``use_fast_math``, c++17, ``-O3``).

Usage: python -m oracle.build_ref [case ...]
"""

from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference's CUDA sources: $CSL_REFERENCE_SRC, else the checkout's usual place.
REF_SRC = os.environ.get("CSL_REFERENCE_SRC", "/root/reference/cuslines/cuda_c")
OUT = os.path.join(HERE, "_ref")


def available() -> bool:
    return os.path.isfile(os.path.join(REF_SRC, "generate_streamlines_cuda.cu"))


def require_sources():
    if not available():
        raise FileNotFoundError(
            f"reference CUDA sources not found in {REF_SRC!r}: set CSL_REFERENCE_SRC to the directory that "
            "holds cuslines/cuda_c/generate_streamlines_cuda.cu")


def build_case(name: str, force: bool = False) -> str:
    from oracle.cases import macros

    out = os.path.join(OUT, f"ref_{name}.so")
    src = os.path.join(HERE, "ref_launcher.cu")
    require_sources()
    if os.path.exists(out) and not force and os.path.getmtime(out) > os.path.getmtime(src):
        return out
    os.makedirs(OUT, exist_ok=True)
    defs = [f"-D{k}={v}" for k, v in macros(name).items()]
    cmd = ["nvcc", "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "--use_fast_math",
           "-std=c++17", "-Xcompiler", "-fPIC", "-shared", "-include", "cstdio",
           "-diag-suppress", "177,550,20281", "-I", REF_SRC, *defs, src, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference build for {name} failed:\n{r.stderr[-4000:]}")
    return out


def main(argv=None):
    from oracle.cases import CASES

    if not available():
        print("reference sources not present; keeping prebuilt oracle/_ref")
        return 0
    names = (argv or sys.argv[1:]) or [k for k, c in CASES.items() if c.get("ref", True)]
    with ThreadPoolExecutor(min(4, len(names))) as ex:
        for path in ex.map(build_case, names):
            print("built", path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
