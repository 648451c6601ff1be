"""Build liblbdem.so (sm_100a) in-tree with nvcc.

    python -m lbdem_taichi_b200.build [--force]

Each translation unit is compiled separately:
  lbm.cu      fused PSC collide-stream and lattice helpers (FMA contraction on)
  psc_map.cu  particle -> lattice mapping, FP64, -fmad=false (bit-exact counts)
  dem.cu      DEM sub-step, FP64, -fmad=false (reference operation order)
  adjoint.cu  reverse mode of the step on a frozen bed (drag gradients)
and linked into one shared library with a static CUDA runtime.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_build")
LIB = os.path.join(OUT, "liblbdem.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xptxas", "-v", "-I", INCLUDE]
UNITS = {
    "lbm.cu": [],
    "psc_map.cu": ["-fmad=false"],
    "dem.cu": ["-fmad=false"],
    "adjoint.cu": [],
}


def nvcc():
    cand = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    return cand if os.path.exists(cand) else "nvcc"


def _deps():
    files = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, "lbdem.h"), __file__]
    return max(os.path.getmtime(f) for f in files)


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= _deps():
        return LIB
    os.makedirs(OUT, exist_ok=True)
    objs = []
    for unit, extra in UNITS.items():
        obj = os.path.join(OUT, unit.replace(".cu", ".o"))
        cmd = [nvcc(), *ARCH, *COMMON, *extra, "-c", os.path.join(CSRC, unit), "-o", obj]
        res = subprocess.run(cmd, capture_output=True, text=True)
        log = os.path.join(OUT, unit + ".ptxas.txt")
        with open(log, "w") as fh:
            fh.write(res.stdout + res.stderr)
        if res.returncode != 0:
            sys.stderr.write(res.stdout + res.stderr)
            raise RuntimeError(f"nvcc failed on {unit}")
        if verbose:
            sys.stdout.write(res.stderr)
        objs.append(obj)
    tmp = LIB + ".tmp"
    subprocess.check_call([nvcc(), *ARCH, "-shared", "-o", tmp, *objs])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
