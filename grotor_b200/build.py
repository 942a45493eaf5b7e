"""Build recipe for the native library (nvcc, sm_100a, in-tree output)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libgrb.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
SOURCES = [os.path.join(CSRC, "grb_api.cu"), os.path.join(CSRC, "synth.cpp"), os.path.join(CSRC, "traffic.cpp")]


def _deps():
    files = list(SOURCES)
    for base in (os.path.join(CSRC, "device"), os.path.join(ROOT, "include")):
        files += [os.path.join(base, f) for f in os.listdir(base)]
    return files


def needs_build() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(f) > t for f in _deps())


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not needs_build():
        return OUT
    cmd = ["nvcc", *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           *SOURCES, "-o", OUT + ".tmp", "-lpthread"]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    subprocess.run(cmd, check=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
