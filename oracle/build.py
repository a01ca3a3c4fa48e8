"""Build the FP64 host oracle (TEST INFRASTRUCTURE ONLY) into oracle/liboracle.so.

The oracle is compiled with -ffp-contract=off so that its arithmetic follows the source
order of the reference exactly, and with OpenMP so that the CPU baseline can use every
host core.  Usage: python oracle/build.py [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
LIB = os.path.join(HERE, "liboracle.so")
SRCS = [os.path.join(HERE, f) for f in ("oracle.cpp", "reactor.cpp", "two_temp.cpp", "oracle_capi.cpp")]
HDRS = [os.path.join(HERE, "oracle.hpp"), os.path.join(REPO, "include", "cb200.h"),
        os.path.join(REPO, "include", "cb200_serve.h")]


def build(force=False):
    newest = max(os.path.getmtime(f) for f in SRCS + HDRS)
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= newest:
        return LIB
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-fopenmp", "-ffp-contract=off",
           "-fno-fast-math", "-I", os.path.join(REPO, "include"), *SRCS, "-o", LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
