"""Build recipe for the native library (nvcc, sm_100a, in-tree output)."""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libgrb.so")
SYNTH_OUT = os.path.join(HERE, "libgrb_synth.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# The routing path (CUDA) and its byte model.
SOURCES = [os.path.join(CSRC, "grb_api.cu"), os.path.join(CSRC, "traffic.cpp")]
# The seeded workload generator: host code only, a library of its own.
SYNTH_SOURCES = [os.path.join(CSRC, "synth.cpp")]


def _deps(sources, dirs):
    files = list(sources)
    for base in dirs:
        files += [os.path.join(base, f) for f in os.listdir(base)]
    return files


def _stale(out, deps) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(f) > t for f in deps)


def needs_build() -> bool:
    inc = os.path.join(ROOT, "include")
    return (_stale(OUT, _deps(SOURCES, (os.path.join(CSRC, "device"), inc)))
            or _stale(SYNTH_OUT, _deps(SYNTH_SOURCES, (inc,))))


def build(force: bool = False, verbose: bool = False) -> str:
    inc = os.path.join(ROOT, "include")
    if force or _stale(OUT, _deps(SOURCES, (os.path.join(CSRC, "device"), inc))):
        cmd = ["nvcc", *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
               *SOURCES, "-o", OUT + ".tmp", "-lpthread"]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
        os.replace(OUT + ".tmp", OUT)
    if force or _stale(SYNTH_OUT, _deps(SYNTH_SOURCES, (inc,))):
        subprocess.run(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", *SYNTH_SOURCES, "-o", SYNTH_OUT + ".tmp",
                        "-lpthread"], check=True)
        os.replace(SYNTH_OUT + ".tmp", SYNTH_OUT)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
