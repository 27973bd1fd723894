"""Builds libakmc_b200.so in-tree for sm_100a.

    python misa-akmc-gpu_b200/build.py [--force]

The kernels are compiled with -fmad=false (and the host sources with
-ffp-contract=off) so that multiplies and adds round separately everywhere; the
fused multiply-adds the arithmetic relies on are explicit fma() calls.  This is
what makes the GPU results bit-identical to the CPU semantics.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libakmc_b200.so")
SOURCES = ["akmc_kernels.cu", "akmc_cluster.cu", "akmc_api.cu", "akmc_model.cpp", "akmc_host.cpp", "akmc_server.cpp"]
HEADERS = ["akmc_common.cuh", "akmc_device.h", "akmc_model.h"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _inputs():
    files = [os.path.join(CSRC, s) for s in SOURCES + HEADERS]
    files.append(os.path.join(ROOT, "include", "akmc.h"))
    files.append(os.path.abspath(__file__))
    missing = [f for f in files if not os.path.exists(f)]
    if missing:
        raise FileNotFoundError("build inputs missing: %s" % ", ".join(missing))
    return files


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _inputs())


def build(force=False, verbose=False, extra_flags=(), lib_path=None):
    lib = lib_path or LIB
    if not force and not extra_flags and up_to_date():
        return LIB
    os.makedirs(LIBDIR, exist_ok=True)
    objdir = os.path.join(HERE, "_build")
    os.makedirs(objdir, exist_ok=True)
    objs = []
    common = [
        "-std=c++17",
        "-O3",
        "-lineinfo",
        "-fmad=false",
        "-Xcompiler",
        "-fPIC,-fvisibility=hidden,-ffp-contract=off",
        "-I" + os.path.join(ROOT, "include"),
        "-I" + CSRC,
    ] + ARCH + list(extra_flags)
    for s in SOURCES:
        src = os.path.join(CSRC, s)
        obj = os.path.join(objdir, s + (".prof" if extra_flags else "") + ".o")
        cmd = [nvcc()] + common + ["-x", "cu" if s.endswith(".cu") else "c++", "-c", src, "-o", obj]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", lib] + objs + ["-lpthread"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
