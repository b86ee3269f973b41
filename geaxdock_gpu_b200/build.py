"""Builds the CUDA library libgeauxdock_b200.so in-tree for sm_100a.

    python -m geaxdock_gpu_b200.build [--verbose]

nvcc cross-compiles without a GPU; the .so sits next to this file so that it travels with
the source tree.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgeauxdock_b200.so")
SOURCES = ["gd_kernels.cu", "gd_capi.cu", "gd_capi_layout.cu", "gd_capi_stream.cu",
           "gd_capi_noalloc.cu", "gd_capi_da.cu", "gd_capi_eval.cu", "gd_capi_tile.cu",
           "gd_peak.cu", "gd_mlp.cu", "gd_da.cu", "gd_umma.cu", "gd_kmeans.cu"]
HEADERS = ["gd_capi_internal.cuh", "gd_device.cuh", "gd_numerics.h", "gd_mlp.cuh", "gd_mlp_fwd.cuh", "gd_umma.cuh", "gd_kmeans.cuh", os.path.join("..", "..", "include", "geauxdock_b200.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-shared",
    "-Xcompiler", "-fPIC,-ffp-contract=off",
    "--expt-relaxed-constexpr",
]


def _nvcc():
    for cand in ("nvcc", "/usr/local/cuda/bin/nvcc"):
        try:
            subprocess.run([cand, "--version"], check=True, capture_output=True)
            return cand
        except (OSError, subprocess.CalledProcessError):
            continue
    raise RuntimeError("nvcc not found")


def stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose: bool = False, ptxas_info: bool = False) -> str:
    cmd = [_nvcc()] + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_info else []) + \
        ["-o", LIB] + [os.path.join(CSRC, s) for s in SOURCES]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
    if verbose or ptxas_info:
        sys.stderr.write(r.stdout + r.stderr)
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, ptxas_info="--ptxas" in sys.argv)
