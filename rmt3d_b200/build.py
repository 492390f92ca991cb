"""Build the in-tree CUDA library (sm_100a) of the FSI step.

Produces ``rmt3d_b200/librmt3d_gpu.so`` next to this file.  Device code is
compiled for sm_100a only; both device and host code are built without
floating-point contraction (``--fmad=false``, ``-ffp-contract=off``) so the
FP64 plain form follows the reference's operation order, which is compiled
with ``-std=c++11`` (ISO mode, no contraction).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "librmt3d_gpu.so")
BUILD = os.path.join(ROOT, "_build")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_FLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "--fmad=false",
                   "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
                   "-I" + INCLUDE, "-I" + CSRC]
CU_SOURCES = ["k_fluid.cu", "k_mg.cu", "k_mgb.cu", "k_mgc.cu", "k_solid.cu", "k_chk.cu", "k_diag.cu", "k_tracer.cu", "scene.cu", "batch.cu"]
PER_FILE = {}
CC_SOURCES = ["cfg.cc", "files.cc"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    return r


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(INCLUDE, "rmt3d_gpu.h"))
    objs = []
    for src in CU_SOURCES:
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        obj = os.path.join(BUILD, src + ".o")
        if _stale(obj, [path] + headers):
            _run([NVCC] + CU_FLAGS + PER_FILE.get(src, []) + ["-c", path, "-o", obj])
            if verbose:
                print("built", obj)
        objs.append(obj)
    for src in CC_SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(BUILD, src + ".o")
        if _stale(obj, [path] + headers):
            _run([NVCC, "-std=c++17", "-O2", "-Xcompiler", "-fPIC,-ffp-contract=off",
                  "-I" + INCLUDE, "-I" + CSRC, "-c", path, "-o", obj])
        objs.append(obj)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs)
        if verbose:
            print("linked", LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose=True))
