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


def build(asan=False, stall=False):
    """``stall=True`` builds the timeout-test variant: the shared-job poll
    limit is 2000 and every published round starts with one claim that no
    warp ever reports done (a helper that stopped)."""
    os.makedirs(OUT, exist_ok=True)
    name = "hostcheck_asan.so" if asan else ("hostcheck_stall.so" if stall else "hostcheck.so")
    target = os.path.join(OUT, name)
    if os.path.exists(target) and all(os.path.getmtime(d) <= os.path.getmtime(target) for d in _deps()):
        return target
    flags = ["-O1", "-g", "-fsanitize=address,undefined", "-fno-omit-frame-pointer"] if asan else ["-O2"]
    if stall:
        flags += ["-DCATN_JOB_SPIN_CAP=2000", "-DCATN_JOB_PHANTOM_CLAIMS=1"]
    cmd = ["g++", "-std=c++17", *flags, "-shared", "-fPIC", "-I", os.path.join(ROOT, "include"),
           "-o", target + ".tmp", os.path.join(HERE, "hostcheck.cpp")]
    subprocess.run(cmd, check=True)
    os.replace(target + ".tmp", target)
    return target


if __name__ == "__main__":
    print(build(), build(asan=True))
