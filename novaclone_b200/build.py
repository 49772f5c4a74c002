"""Build libnova_b200.so in-tree with nvcc for sm_100a.

    python -m novaclone_b200.build          # incremental
    python -m novaclone_b200.build --force  # rebuild everything

Objects go to novaclone_b200/_build/, the shared library to
novaclone_b200/libnova_b200.so (found by novaclone_b200.nova at import).
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "libnova_b200.so")
INCLUDE = os.path.join(ROOT, "include")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
NVCC = os.path.join(CUDA_HOME, "bin", "nvcc")

SOURCES = ["nova_stage.cu", "nova_stage_tma.cu", "nova_stage_mhd_tma.cu", "nova_proj_tma.cu", "nova_ops.cu", "nova_pois_i.cu",
    "nova_pois_dct.cu", "nova_fft2d.cu", "nova_adjoint.cu", "nova_adj_tma.cu", "nova_wc.cu", "nova_io.cu", "nova_im.cu", "nova_capi.cu"]
HEADERS = ["nova_internal.cuh", "nova_ops.cuh", "nova_tile.cuh", "nova_stage_math.cuh", "nova_tma.cuh", "nova_adj_math.cuh", "nova_wc.cuh", "nova_mesh.cuh", "nova_diag.cuh", "nova_fft.cuh"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-diag-suppress", "177", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC]


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    hdrs = [os.path.join(CSRC, h) for h in HEADERS] + [os.path.join(INCLUDE, "nova_gpu.h")]
    objs = []
    procs = []
    for src in SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src.replace(".cu", ".o"))
        objs.append(o)
        if force or _newer(o, [s] + hdrs):
            cmd = [NVCC] + ARCH + FLAGS + ["-c", s, "-o", o]
            if verbose:
                print(" ".join(cmd))
            procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            sys.stderr.write(out.decode())
            raise RuntimeError("nvcc failed: " + " ".join(cmd))
    if force or _newer(LIB, objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + [
            "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcufft",
            "-Xlinker", "-rpath," + os.path.join(CUDA_HOME, "lib64")]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(force=a.force, verbose=True))
