"""Build recipe for libcatn_b200.so (sm_100a) -- compiled in-tree so that the
shared library travels with the source tree.

    python catn.jl_b200/build.py          # build the library
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcatn_b200.so")
NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
              "-Xcompiler", "-fPIC"]
# Each unit compiles the device engine on its own (no device linking), so one
# kernel's register allocation never depends on another unit's kernels.
UNITS = ["capi.cu", "capi_static.cu", "capi_grad.cu", "capi_braket.cu", "capi_tc.cu", "capi_lean.cu", "pool.cu"]
OBJ = os.path.join(HERE, "_build")


def _sources():
    return [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC))] + [os.path.join(ROOT, "include", "catn_b200.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build_library(force=False, verbose=False):
    """Compile the translation units in UNITS with nvcc (in parallel) and link
    them into libcatn_b200.so."""
    if not force and not _stale(LIB, _sources() + [__file__]):
        return LIB
    nvcc = os.environ.get("NVCC", "nvcc")
    os.makedirs(OBJ, exist_ok=True)
    objs, procs = [], []
    for u in UNITS:
        obj = os.path.join(OBJ, u.replace(".cu", ".o"))
        cmd = [nvcc, *NVCC_FLAGS, "-I", os.path.join(ROOT, "include"), "-c", "-o", obj, os.path.join(CSRC, u)]
        if verbose:
            print(" ".join(cmd))
        objs.append(obj)
        procs.append(subprocess.Popen(cmd))
    if any(p.wait() != 0 for p in procs):
        raise RuntimeError("nvcc failed on one of " + ", ".join(UNITS))
    link = [nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB + ".tmp", *objs]
    if verbose:
        print(" ".join(link))
    subprocess.run(link, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose=True)
    print(LIB)
