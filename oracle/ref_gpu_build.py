"""Build the reference-kernel runner into oracle/_ref/ (TEST INFRASTRUCTURE ONLY).

Compiles the reference's own hot-path CUDA and host sources, straight from the reference source
tree (never copied into this repository), for sm_100a with nvcc / g++, against the single-process
oracle/ref/mpi.h, and links them with oracle/ref/ref_stage_runner.cu into two executables:

  oracle/_ref/ref_stage_runner     the default build (Combustion2Part, one temperature)
  oracle/_ref/ref_stage_runner_2t  the same sources with COREFL_ENABLE_TWO_TEMPERATURE=1

The defines are the reference's own (CMakeLists.txt: MAX_SPEC_NUMBER=9, MAX_REAC_NUMBER=19,
MAX_PASSIVE_SCALAR_NUMBER=1, Combustion2Part) and its separable compilation
(CUDA_SEPARABLE_COMPILATION ON, src/CMakeLists.txt).  The reference's CMake build itself is not
used: it requires an MPI installation.  The runner is executed on a GPU by
tests/golden/make_ref_kernels.py; nothing else runs it.

Usage: python oracle/ref_gpu_build.py [--ref DIR] [--jobs N] [--only 1t|2t]
The reference directory comes from --ref, else oracle/ref_build.py's reference_dir().
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")

# Reference sources linked into the runner: the hot path, the field/boundary/communication code it
# calls, and the host code those pull in.  main.cu, Driver.cu, Simulate and the integrators are
# left out; the runner has its own main.
SOURCES = [
    "WENO.cu", "InviscidScheme.cu", "Reconstruction.cu", "ViscousScheme.cu", "FieldOperation.cu", "Thermo.cu",
    "Transport.cu", "FiniteRateChem.cu", "DParameter.cu", "DataCommunication.cu", "TimeAdvanceFunc.cu",
    "BoundCond.cu", "BoundCond.cpp", "Field.cu", "DigitalFilter.cu", "Initialize.cu", "Mesh.cpp", "Mesh.cu",
    "MixingLayer.cu", "MixtureFraction.cpp", "Parameter.cpp", "ChemData.cpp", "Element.cpp", "kernels.cu",
    "UDIO.cu", "Parallel.cpp", "SinglePointStat.cu", "stat_lib/TkeBudget.cu", "stat_lib/SpeciesStat.cu", "gxl_lib/MyString.cpp",
    "gxl_lib/MyAlgorithm.cpp", "gxl_lib/Time.cpp",
]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
DEFS = ["-DMAX_SPEC_NUMBER=9", "-DMAX_REAC_NUMBER=19", "-DMAX_PASSIVE_SCALAR_NUMBER=1", "-DCombustion2Part"]


def reference_dir(ref=None):
    import importlib.util
    spec = importlib.util.spec_from_file_location("ref_build", os.path.join(HERE, "ref_build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.reference_dir(ref)


def _compile(src_dir, rel, obj_dir, two_t):
    src = os.path.join(src_dir, rel)
    obj = os.path.join(obj_dir, rel.replace("/", "_") + ".o")
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src),
                                                              os.path.getmtime(os.path.join(HERE, "ref", "mpi.h"))):
        return obj
    defs = DEFS + ["-DCOREFL_ENABLE_TWO_TEMPERATURE=%d" % (1 if two_t else 0)]
    inc = ["-I", os.path.join(HERE, "ref"), "-I", src_dir]
    if rel.endswith(".cu"):
        cmd = ["nvcc", "-std=c++17", "-O3", "-rdc=true", *ARCH, *defs, *inc, "-c", src, "-o", obj]
    else:
        cmd = ["g++", "-std=c++20", "-O2", *defs, *inc, "-I", "/usr/local/cuda/include", "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compiling %s failed:\n%s" % (rel, r.stderr[-3000:]))
    return obj


def build_one(ref, two_t, jobs=8):
    src_dir = os.path.join(ref, "src")
    tag = "2t" if two_t else "1t"
    obj_dir = os.path.join(OUT, "obj_" + tag)
    os.makedirs(obj_dir, exist_ok=True)
    rels = list(SOURCES)
    with cf.ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(lambda r: _compile(src_dir, r, obj_dir, two_t), rels))
    runner_src = os.path.join(HERE, "ref", "ref_stage_runner.cu")
    runner_obj = os.path.join(obj_dir, "ref_stage_runner.o")
    exe = os.path.join(OUT, "ref_stage_runner" + ("_2t" if two_t else ""))
    if os.path.exists(exe) and os.path.getmtime(exe) >= max(os.path.getmtime(f) for f in objs + [runner_src]):
        return exe
    defs = DEFS + ["-DCOREFL_ENABLE_TWO_TEMPERATURE=%d" % (1 if two_t else 0)]
    r = subprocess.run(["nvcc", "-std=c++17", "-O2", "-rdc=true", *ARCH, *defs, "-I", os.path.join(HERE, "ref"),
                        "-I", src_dir, "-c", runner_src, "-o", runner_obj], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compiling the runner failed:\n" + r.stderr[-3000:])
    r = subprocess.run(["nvcc", *ARCH, "-rdc=true", runner_obj, *objs, "-o", exe, "-lcurand"],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("linking the runner failed:\n" + r.stderr[-4000:])
    return exe


def build(ref=None, jobs=8, only=None):
    ref = reference_dir(ref)
    if ref is None:
        return None
    out = []
    for two_t in (False, True):
        if only and only != ("2t" if two_t else "1t"):
            continue
        out.append(build_one(ref, two_t, jobs))
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    ap.add_argument("--jobs", type=int, default=8)
    ap.add_argument("--only", default=None)
    a = ap.parse_args()
    res = build(a.ref, a.jobs, a.only)
    if res is None:
        sys.exit("reference sources not found: pass --ref or set COREFL_REFERENCE")
    print("\n".join(res))
