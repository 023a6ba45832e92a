"""Build libedlut_b200.so in-tree with nvcc for sm_100a.

    python -m edlut_b200.build

The whole library is compiled with ``--fmad=false`` so no multiply-add is
contracted: the neuron updates must round exactly like the reference CPU code.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OUT = os.path.join(OUT_DIR, "libedlut_b200.so")
SOURCES = ["eb_kernels.cu", "eb_runtime.cu", "eb_fold.cu", "eb_sweep.cu", "eb_adjoint.cu", "eb_tables.cpp", "eb_cfg.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "edlut_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return OUT
    os.makedirs(OUT_DIR, exist_ok=True)
    tmp = OUT + ".tmp"
    cmd = [nvcc(), *ARCH, "-std=c++17", "-O3", "--fmad=false", "-lineinfo",
           "-Xcompiler", "-fPIC,-ffp-contract=off", "-diag-suppress", "128",
           "-shared", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC,
           *[os.path.join(CSRC, s) for s in SOURCES], "-o", tmp]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stdout[-4000:] + r.stderr[-4000:])
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
