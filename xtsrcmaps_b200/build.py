"""Build libxts_cuda.so in-tree for sm_100a.

    python -m xtsrcmaps_b200.build [--verbose-ptxas]

Compiles every .cu file of xtsrcmaps_b200/csrc with nvcc into
xtsrcmaps_b200/libxts_cuda.so (the file travels with the source tree; nothing
is installed into site-packages).
"""
from __future__ import annotations

import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libxts_cuda.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = sources() + glob.glob(os.path.join(CSRC, "*.cuh")) + [
        os.path.join(HERE, "..", "include", "xtsrcmaps_b200.h")]
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose_ptxas: bool = False) -> str:
    if not force and not needs_build():
        return OUT
    # cuFFT (the diffuse-map convolution) from the toolkit next to nvcc, found at run time by rpath
    lib64 = os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(nvcc()))), "lib64")
    cmd = [nvcc(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-o", OUT + ".tmp", *sources(), "-L" + lib64, "-lcufft", "-Xlinker", "-rpath=" + lib64]
    if verbose_ptxas:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("nvcc failed building libxts_cuda.so")
    if verbose_ptxas:
        sys.stderr.write(r.stderr)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force=True, verbose_ptxas="--verbose-ptxas" in sys.argv))
