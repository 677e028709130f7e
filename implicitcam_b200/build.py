"""Builds the CUDA library libicam_cuda.so in this directory (sm_100a only).

    python -m implicitcam_b200.build
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libicam_cuda.so")
SOURCES = ["api.cu", "kernels.cu", "bricks.cu", "bricks_mixed.cu", "decide.cu", "seednet.cu", "batch.cu", "pack_build.cpp", "host_geom.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def sources_newer() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(HERE, "..", "include", "icam_cuda.h"))
    deps.append(os.path.join(HERE, "..", "include", "icam_solid.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    """Compiles every source to an object in parallel (one nvcc a file, the kernels
    launched across files need no relocatable device code), then links the library."""
    if not force and not sources_newer():
        return OUT
    from concurrent.futures import ThreadPoolExecutor

    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    flags = ["-Xcompiler", "-fPIC", "-std=c++17", "-O3", "-lineinfo", *ARCH]
    if verbose:
        flags.insert(0, "-Xptxas=-v")

    def compile_one(src):
        obj = os.path.join(objdir, src + ".o")
        r = subprocess.run([nvcc(), "-c", *flags, "-o", obj, os.path.join(CSRC, src)], capture_output=True, text=True)
        return src, obj, r

    with ThreadPoolExecutor(max_workers=min(len(SOURCES), os.cpu_count() or 1)) as ex:
        results = list(ex.map(compile_one, SOURCES))
    for src, _, r in results:
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src}:\n" + r.stdout + r.stderr)
        if verbose:
            sys.stderr.write(r.stderr)
    r = subprocess.run([nvcc(), "-shared", *ARCH, "-o", OUT + ".tmp", *[o for _, o, _ in results]],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + r.stdout + r.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
