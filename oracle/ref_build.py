"""Build the reference's own host code into oracle/_ref/ (TEST INFRASTRUCTURE ONLY).

Compiles, straight from the reference source tree (never copied into this repository):
  dump_mech : cfd::Species / cfd::Reaction (src/ChemData.cpp) + cfd::Parameter
              (src/Parameter.cpp) + src/Element.cpp + src/gxl_lib/MyString.cpp, with the
              single-process oracle/ref/mpi.h, oracle/ref/stubs.cpp and
              oracle/ref/dump_mech.cpp; it writes the mechanism tables as JSON.
The reference's CMake build needs MPI and is not used.
Usage: python oracle/ref_build.py [/path/to/reference]   (default: $COREFL_REFERENCE, else
DEFAULT_REFERENCE below)
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
# where the reference checkout lives in the build container; $COREFL_REFERENCE overrides it
DEFAULT_REFERENCE = "/root/reference"


def reference_dir(ref=None):
    """The reference source tree: `ref`, else $COREFL_REFERENCE, else DEFAULT_REFERENCE; None if
    it holds no src/ directory (as on a machine without the reference)."""
    ref = ref or os.environ.get("COREFL_REFERENCE") or DEFAULT_REFERENCE
    return ref if os.path.isdir(os.path.join(ref, "src")) else None


def build(ref=None, force=False):
    ref = reference_dir(ref)
    if ref is None:
        return None
    src = os.path.join(ref, "src")
    os.makedirs(OUT, exist_ok=True)
    exe = os.path.join(OUT, "dump_mech")
    mine = [os.path.join(HERE, "ref", f) for f in ("stubs.cpp", "dump_mech.cpp", "mpi.h")]
    drivers = [os.path.join(HERE, "ref", f) for f in ("dump_chem.cpp", "dump_reactor.cpp", "chem_stubs.cpp",
                                                       "dump_2t.cpp", "dump_air5.cpp")]
    theirs = [os.path.join(src, f) for f in ("ChemData.cpp", "Parameter.cpp", "Element.cpp",
                                             os.path.join("gxl_lib", "MyString.cpp"))]
    if not force and os.path.exists(exe) and os.path.getmtime(exe) >= max(os.path.getmtime(f) for f in mine + drivers):
        return exe
    cmd = ["g++", "-std=c++20", "-O1", "-DMAX_SPEC_NUMBER=9", "-DMAX_REAC_NUMBER=20", "-DCombustion2Part",
           "-I", os.path.join(HERE, "ref"), "-I", src,
           *[f for f in theirs], *[f for f in mine if f.endswith(".cpp")], "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference host build failed:\n" + r.stderr[-4000:])
    # dump_chem: the same parser plus the host chemistry of src/ConstVolumeReactor.cpp
    exe2 = os.path.join(OUT, "dump_chem")
    cmd2 = [c for c in cmd if not c.endswith("dump_mech.cpp")]
    cmd2[-1] = exe2
    cmd2[-2:-2] = [os.path.join(src, "ConstVolumeReactor.cpp"), os.path.join(HERE, "ref", "dump_chem.cpp"),
                   os.path.join(HERE, "ref", "chem_stubs.cpp")]
    r = subprocess.run(cmd2, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference host chemistry build failed:\n" + r.stderr[-4000:])
    # dump_reactor: the same host chemistry driven through the ROK4E reactor sequence
    exe3 = os.path.join(OUT, "dump_reactor")
    cmd3 = [c if not c.endswith("dump_chem.cpp") else os.path.join(HERE, "ref", "dump_reactor.cpp") for c in cmd2]
    cmd3[-1] = exe3
    r = subprocess.run(cmd3, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference reactor driver build failed:\n" + r.stderr[-4000:])
    # dump_2t: the parser and host chemistry rebuilt with the reference's two-temperature switch on
    # (COREFL_ENABLE_TWO_TEMPERATURE, src/Define.h:10-12), so Species reads two_temperature.dat
    exe4 = os.path.join(OUT, "dump_2t")
    cmd4 = [c if not c.endswith("dump_chem.cpp") else os.path.join(HERE, "ref", "dump_2t.cpp") for c in cmd2]
    cmd4.insert(1, "-DCOREFL_ENABLE_TWO_TEMPERATURE=1")
    cmd4[-1] = exe4
    r = subprocess.run(cmd4, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference two-temperature driver build failed:\n" + r.stderr[-4000:])
    # dump_air5: the same two-temperature build driven on the AIR5 data; the host Species thermo
    # and compute_gibbs_div_rt evaluate NASA9 multi-range polynomials whenever therm_nasa_7_9 = 9
    # (src/ChemData.cpp:326-520, src/ConstVolumeReactor.cpp:1401-1454)
    exe5 = os.path.join(OUT, "dump_air5")
    cmd5 = [c if not c.endswith("dump_2t.cpp") else os.path.join(HERE, "ref", "dump_air5.cpp") for c in cmd4]
    cmd5[-1] = exe5
    r = subprocess.run(cmd5, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("reference AIR5 driver build failed:\n" + r.stderr[-4000:])
    return exe


if __name__ == "__main__":
    print(build(sys.argv[1] if len(sys.argv) > 1 else None, force=True))
