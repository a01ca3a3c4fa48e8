"""Build libcb200.so (the sm_100a kernels + C ABI) in-tree with nvcc.

Usage: python corefl-cpc_b200/build.py [--force]

Each .cu file under csrc/ is compiled to an object in _build/ (in parallel) and linked
into corefl-cpc_b200/libcb200.so.  Objects are rebuilt when their source or any header
under csrc/ or include/ is newer.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcb200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
         "--expt-relaxed-constexpr", "-I", os.path.join(REPO, "include"), "-I", CSRC]


# The mixed form's FP32 reconstruction, fluxes and viscous stencils: FP32 division and square
# root use the hardware approximations (about 2 ulp) instead of the IEEE-rounded instruction
# sequences.  These flags change single-precision arithmetic only; every FP64 operation in these
# files (the plain form, the mixture thermodynamics, the state) is compiled as before.
FAST_F32_FILES = {"inviscid_pv_f32.cu": ["-prec-div=false", "-prec-sqrt=false"],
                  "viscous.cu": ["-prec-div=false", "-prec-sqrt=false"]}


def _newest_header():
    t = 0.0
    for d in (CSRC, os.path.join(REPO, "include")):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh", ".hpp")):
                t = max(t, os.path.getmtime(os.path.join(d, f)))
    return t


def _compile(src, force, verbose):
    obj = os.path.join(BUILD, os.path.basename(src).replace(".cu", ".o"))
    if (not force and os.path.exists(obj)
            and os.path.getmtime(obj) >= max(os.path.getmtime(src), _newest_header())):
        return obj, None
    cmd = [NVCC, *ARCH, *FLAGS, *FAST_F32_FILES.get(os.path.basename(src), []), "-c", src, "-o", obj]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, r.stderr + r.stdout
    if verbose:
        sys.stderr.write(r.stderr)
    return obj, None


def build(force=False, verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        results = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    errs = [e for _, e in results if e]
    if errs:
        raise RuntimeError("nvcc failed:\n" + "\n".join(errs))
    objs = [o for o, _ in results]
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stderr + r.stdout)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
