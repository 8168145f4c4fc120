"""Build the native engine ``libgpusw_sm100.so`` in-tree with nvcc (sm_100a only).

    python -m gpusw_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "engine.cu")
DEPS = [os.path.join(HERE, "csrc", f) for f in ("engine.cu", "dp_core.cuh", "kernels.cuh", "server.cuh", "fasta.cuh")]
HEADER = os.path.join(os.path.dirname(HERE), "include", "gpusw_b200.h")
OUT = os.path.join(HERE, "libgpusw_sm100.so")
# No -split-compile: it parallelises the build but changes code generation, and the
# streaming kernel measured 7 % slower (6,061 vs 6,532 GCUPS on the 16S step) built with it.
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
              "-Xcompiler", "-fPIC", "-shared", "-Xptxas", "-v"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if cand and (os.path.isabs(cand) and os.path.exists(cand) or not os.path.isabs(cand)):
            return cand
    return "nvcc"


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile the engine if any source is newer than the library; return its path."""
    newest = max(os.path.getmtime(p) for p in DEPS + [HEADER])
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= newest:
        return OUT
    tmp = OUT + ".tmp"
    cmd = [nvcc(), *NVCC_FLAGS, "-o", tmp, SRC]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("nvcc failed building the engine")
    if verbose:
        sys.stderr.write(res.stderr)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
