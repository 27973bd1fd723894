"""Builds the reference-side binding of the B200 engine for its tests.

    python tests/shim/build_shim.py

Compiles misa-akmc-gpu_b200/integration/gpu_simulate_b200.cpp against the reference's own
gpu/gpu_simulate.h (and the lattice, model and lattice-store headers it includes), with the
stand-in headers of tests/shim/stubs for the packages the reference does not vendor (HIP,
libcomm, kiwi) and for its CMake-generated building_config.h.  The reference's lattice-store
sources (src/lattice/*.cpp, models/abvi/defect/vac_hash.cpp) are compiled from where they lie,
together with tests/shim/shim_driver.cpp, into tests/shim/_build/libgpu_simulate_b200_shim.so,
linked to misa-akmc-gpu_b200/lib/libakmc_b200.so.  The reference must be present (it is read
only at build time); the built library is self-contained apart from libakmc_b200.so.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REFERENCE = os.environ.get("AKMC_REFERENCE", "/root/reference")
OUT_DIR = os.path.join(HERE, "_build")
OUT = os.path.join(OUT_DIR, "libgpu_simulate_b200_shim.so")
SHIM = os.path.join(ROOT, "misa-akmc-gpu_b200", "integration", "gpu_simulate_b200.cpp")
LIBDIR = os.path.join(ROOT, "misa-akmc-gpu_b200", "lib")
REF_SOURCES = ["src/lattice/lattices_list.cpp", "src/lattice/period_lattice_list.cpp",
               "src/lattice/lattice_list_meta.cpp", "src/lattice/lattice.cpp", "src/lattice/lattice_types.cpp",
               "models/abvi/defect/vac_hash.cpp"]


def available():
    return os.path.exists(os.path.join(REFERENCE, "gpu", "gpu_simulate.h"))


def includes():
    return ["-I" + os.path.join(HERE, "stubs"), "-I" + REFERENCE, "-I" + os.path.join(REFERENCE, "src"),
            "-I" + os.path.join(REFERENCE, "models"), "-I" + os.path.join(REFERENCE, "gpu"),
            "-I" + os.path.join(ROOT, "include")]


def build(verbose=False):
    if not available():
        raise FileNotFoundError("the reference sources are needed to build the shim (%s)" % REFERENCE)
    os.makedirs(OUT_DIR, exist_ok=True)
    srcs = [SHIM, os.path.join(HERE, "shim_driver.cpp")] + [os.path.join(REFERENCE, s) for s in REF_SOURCES]
    cmd = (["g++", "-std=c++17", "-O2", "-fPIC", "-shared", "-o", OUT] + includes() + srcs +
           ["-L" + LIBDIR, "-lakmc_b200", "-Wl,-rpath,$ORIGIN/../../../misa-akmc-gpu_b200/lib"])
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
