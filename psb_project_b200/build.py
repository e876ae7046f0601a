"""Builds libpsb.so in-tree (psb_project_b200/lib/) for sm_100a.

    python -m psb_project_b200.build

CUDA sources go through nvcc with -gencode arch=compute_100a,code=sm_100a;
the host-only scene generator through g++ with FMA contraction off (its
output must match the test-suite's generator bit for bit). The CUDA runtime
is linked statically, so the library needs only the driver at run time.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(OUT_DIR, "libpsb.so")
OBJ_DIR = os.path.join(ROOT, "_build")

CU_SOURCES = ["grid.cu", "sph.cu", "api.cu", "noalloc.cu", "mlp.cu", "dem.cu", "mc.cu", "compat.cu", "compat_sph.cu",
              "batch.cu", "diag.cu", "boundary.cu", "colliders.cu", "emit.cu"]
# Per-file additions: the reference-signature FP64 kernels keep separate
# multiplies and adds, as the reference's own kernels compiled for the host do.
CU_EXTRA_FLAGS = {"compat_sph.cu": ["-fmad=false"]}
CPP_SOURCES = ["scene.cpp", "io.cpp", "emitters.cpp"]
NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {' '.join(cmd)}")
    return r


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    inc = ["-I", os.path.join(ROOT, "include"), "-I", CSRC]
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers += [os.path.join(ROOT, "include", "psb.h"), os.path.join(ROOT, "include", "psb_compat.h")]
    objs = []
    nvcc = _nvcc()
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ_DIR, src + ".o")
        if force or _stale(o, [s] + headers):
            cmd = [nvcc] + NVCC_FLAGS + CU_EXTRA_FLAGS.get(src, []) + inc + ["-Xptxas", "-v", "-c", s, "-o", o]
            r = _run(cmd)
            if verbose:
                sys.stderr.write(r.stderr)
        objs.append(o)
    for src in CPP_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ_DIR, src + ".o")
        if force or _stale(o, [s] + headers):
            _run(["g++", "-O2", "-fPIC", "-ffp-contract=off", "-fopenmp", "-std=c++17"] + inc + ["-c", s, "-o", o])
        objs.append(o)
    if force or _stale(LIB, objs):
        # linked beside the library and renamed over it: a process that has
        # the old file mapped keeps its pages instead of seeing them rewritten
        tmp = LIB + f".{os.getpid()}.tmp"
        _run([nvcc, "-shared", "-o", tmp] + objs + ["-Xcompiler", "-fopenmp"])
        os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
