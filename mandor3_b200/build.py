"""Builds the B200 PIC core in-tree: ``mandor3_b200/libmandor_b200.so`` (the
C ABI of include/mandor_b200.h, all kernels compiled for sm_100a) and the
host driver ``mandor3_b200/core_b200.out`` (a drop-in for the reference
``core.out``).

    python -m mandor3_b200.build          # incremental
    python -m mandor3_b200.build --force  # rebuild everything
"""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
OBJ = os.path.join(PKG, "_build")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(PKG, "libmandor_b200.so")
DRIVER = os.path.join(PKG, "core_b200.out")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE]

# Translation units and their extra flags.  The FP64 form is compiled
# without FMA contraction so that its arithmetic rounds exactly as the
# reference's C does (bit-identical cell indices and marker updates).
CUDA_UNITS = {
    "api.cu": ["-fmad=false"],
    "fields64.cu": ["-fmad=false"],
    "push64.cu": ["-fmad=false"],
    "placer.cu": ["-fmad=false"],
    "gauss.cu": ["-fmad=false"],
    "tags.cu": ["-fmad=false"],
    "tecplot.cu": ["-fmad=false"],
    "tfsf.cu": ["-fmad=false"],
    "api32.cu": [],
    "fields32.cu": [],
    "push32.cu": [],
}
HOST_UNITS = []


def _newer(src, dst, extra=()):
    if not os.path.exists(dst):
        return True
    t = os.path.getmtime(dst)
    return any(os.path.getmtime(p) > t for p in (src,) + tuple(extra))


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build(force=False, verbose=False):
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(INCLUDE, "mandor_b200.h"))
    objs = []
    for unit, flags in CUDA_UNITS.items():
        src = os.path.join(CSRC, unit)
        obj = os.path.join(OBJ, unit + ".o")
        if force or _newer(src, obj, headers):
            _run([NVCC] + ARCH + COMMON + flags + ["-c", src, "-o", obj], verbose)
        objs.append(obj)
    for unit in HOST_UNITS:
        src = os.path.join(HOST, unit)
        if not os.path.exists(src):
            continue
        obj = os.path.join(OBJ, unit + ".o")
        if force or _newer(src, obj, headers):
            _run(["gcc", "-O2", "-std=gnu99", "-fPIC", "-Wall", "-I" + INCLUDE, "-I" + HOST,
                  "-c", src, "-o", obj], verbose)
        objs.append(obj)
    if force or any(_newer(o, LIB) for o in objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static"], verbose)
    main_src = os.path.join(HOST, "core_main.c")
    if os.path.exists(main_src) and (force or _newer(main_src, DRIVER, [LIB])):
        _run(["gcc", "-O2", "-std=gnu99", "-Wall", "-I" + INCLUDE, "-I" + HOST, main_src,
              "-o", DRIVER, "-L" + PKG, "-lmandor_b200", "-Wl,-rpath,$ORIGIN", "-lm", "-lpthread"], verbose)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
