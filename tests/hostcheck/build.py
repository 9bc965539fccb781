"""Build the test-only host harness (tests/hostcheck/hostcheck.cpp): the
device engine compiled as plain C++ with a team of one thread, optionally
under AddressSanitizer/UBSan.  Used by the CPU test-suite only."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
OUT = os.path.join(HERE, "_build")


def _deps():
    csrc = os.path.join(ROOT, "catn.jl_b200", "csrc")
    return [os.path.join(HERE, "hostcheck.cpp"), os.path.join(ROOT, "include", "catn_b200.h")] + \
        [os.path.join(csrc, f) for f in os.listdir(csrc)]


def build(asan=False):
    os.makedirs(OUT, exist_ok=True)
    target = os.path.join(OUT, "hostcheck_asan.so" if asan else "hostcheck.so")
    if os.path.exists(target) and all(os.path.getmtime(d) <= os.path.getmtime(target) for d in _deps()):
        return target
    flags = ["-O1", "-g", "-fsanitize=address,undefined", "-fno-omit-frame-pointer"] if asan else ["-O2"]
    cmd = ["g++", "-std=c++17", *flags, "-shared", "-fPIC", "-I", os.path.join(ROOT, "include"),
           "-o", target + ".tmp", os.path.join(HERE, "hostcheck.cpp")]
    subprocess.run(cmd, check=True)
    os.replace(target + ".tmp", target)
    return target


if __name__ == "__main__":
    print(build(), build(asan=True))
