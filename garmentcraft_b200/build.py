"""Builds the device library libklon3d_b200.so in-tree with nvcc for sm_100a.

Usage: python -m garmentcraft_b200.build
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_native")
LIB = os.path.join(OUT_DIR, "libklon3d_b200.so")
SOURCES = ["k3d_step.cu", "k3d_step_f32.cu", "k3d_build.cu", "k3d_host.cpp", "scene_build.cpp", "k3d_noalloc.cu", "k3d_selbst.cu",
           "k3d_selbst_host.cpp", "k3d_adjoint.cu", "k3d_netz.cu"]
HEADERS = ["k3d_step.h", "k3d_device.cuh", "k3d_step_common.cuh", "k3d_solve.cuh", "scene_build.h", "k3d_selbst.h",
           "k3d_selbst_host.h", "k3d_adjoint.h", "k3d_vec.cuh", "k3d_netz.cuh", "k3d_netz.h"]
# Per-file flags. The build of the system and the self-collision stage round
# every product and sum on their own (no fused multiply-add), as the
# reference's arithmetic does: the element term of k3d_build.cu needs it, and
# the self-collision cell indices, buckets and pairs come out bit-exact. So
# does the PCG with FP64 vectors (k3d_step.cu): its bits then do not depend on
# the compiler's choice of which products to fuse, and the mesh-body parity
# tests hold; the FP32-vector PCG (k3d_step_f32.cu) keeps fused products. The
# adjoint replays the forward's contact queries and rounds the same way; the
# body mesh's nearest-point regions and distances round as the reference's;
# the allocation-free operator evaluates the same element products as the build.
EXTRA = {"k3d_step.cu": ["-fmad=false"], "k3d_build.cu": ["-fmad=false"], "k3d_selbst.cu": ["-fmad=false"], "k3d_adjoint.cu": ["-fmad=false"],
         "k3d_netz.cu": ["-fmad=false"], "k3d_noalloc.cu": ["-fmad=false"]}

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
    "-Xcompiler", "-O3", "-Xcompiler", "-ffp-contract=off",
]


def _stale() -> bool:
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    deps.append(os.path.join(HERE, "..", "include", "klon3d_step.h"))
    deps.append(os.path.join(HERE, "..", "include", "klon3d_mesh.h"))
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    if not force and not _stale():
        return LIB
    obj_dir = os.path.join(OUT_DIR, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    objs = []
    for f in SOURCES:
        p = os.path.join(CSRC, f)
        o = os.path.join(obj_dir, f + ".o")
        lang = ["-x", "cu"] if f.endswith(".cpp") else []
        cmd = [NVCC, *FLAGS, *EXTRA.get(f, []), "-c", *lang, p, "-o", o]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd))
        subprocess.run(cmd, check=True, cwd=CSRC)
        objs.append(o)
    link = [NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "--shared", "-cudart", "shared",
            "-o", LIB + ".tmp", *objs]
    subprocess.run(link, check=True, cwd=CSRC)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
