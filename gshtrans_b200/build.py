"""Builds libgsht_cuda.so in-tree from gshtrans_b200/csrc/*.cu for sm_100a.

    python gshtrans_b200/build.py

(run as a script: importing the package loads the library it builds)

The library is built next to this file so that it travels with the source
tree; it has no dependency on PyTorch.
"""

from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, "libgsht_cuda.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cuh"))) + [
        os.path.join(ROOT, "include", "gsht.h")
    ]


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in sources() + headers())


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every translation unit to an object in parallel (they share
    no device symbols), then links the shared library."""
    if not force and not needs_build():
        return LIB
    from concurrent.futures import ThreadPoolExecutor

    nvcc = os.environ.get("NVCC", "nvcc")
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
             "-I", os.path.join(ROOT, "include")]

    def compile_one(src):
        obj = os.path.join(objdir, os.path.basename(src) + ".o")
        cmd = [nvcc, *flags, "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        r = subprocess.run(cmd, capture_output=True, text=True)
        return src, obj, r

    jobs = max(1, min(len(sources()), os.cpu_count() or 1))
    with ThreadPoolExecutor(jobs) as ex:
        results = list(ex.map(compile_one, sources()))
    failed = [(src, r) for src, _, r in results if r.returncode != 0]
    for src, r in failed:
        sys.stderr.write(r.stdout + r.stderr)
    if failed:
        raise subprocess.CalledProcessError(failed[0][1].returncode, f"nvcc {failed[0][0]}")
    cmd = [nvcc, *ARCH, "-shared", *[o for _, o, _ in results], "-o", LIB + ".tmp"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
