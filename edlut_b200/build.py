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
SOURCES = ["eb_kernels.cu", "eb_runtime.cu", "eb_record.cu", "eb_fold.cu", "eb_sweep.cu", "eb_adjoint.cu", "eb_tables.cpp", "eb_cfg.cpp"]
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


def _compile_flags():
    return [*ARCH, "-std=c++17", "-O3", "--fmad=false", "-lineinfo", "-Xcompiler", "-fPIC,-ffp-contract=off",
            "-diag-suppress", "128", "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile every source to an object (in parallel, one nvcc per file) and link
    the shared library.  Objects newer than every source and header are reused
    unless ``force``."""
    if not force and not _stale():
        return OUT
    from concurrent.futures import ThreadPoolExecutor
    obj_dir = os.path.join(OUT_DIR, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(ROOT, "include", "edlut_b200.h"))
    newest_header = max(os.path.getmtime(h) for h in headers)

    def compile_one(src):
        path = os.path.join(CSRC, src)
        obj = os.path.join(obj_dir, src + ".o")
        if (not force and os.path.exists(obj)
                and os.path.getmtime(obj) > max(os.path.getmtime(path), newest_header)):
            return obj, None
        cmd = [nvcc(), *_compile_flags(), "-c", path, "-o", obj + ".tmp"]
        if verbose:
            print(" ".join(cmd))
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            return obj, "nvcc failed on %s:\n%s%s" % (src, r.stdout[-4000:], r.stderr[-4000:])
        os.replace(obj + ".tmp", obj)
        return obj, None

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 4)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    errors = [e for _, e in results if e]
    if errors:
        raise RuntimeError("\n".join(errors))
    tmp = OUT + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", *[o for o, _ in results], "-o", tmp]
    if verbose:
        print(" ".join(cmd))
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("link failed:\n" + r.stdout[-4000:] + r.stderr[-4000:])
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
