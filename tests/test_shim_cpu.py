"""The reference-side shim (corefl-cpc_b200/shim/cb200_shim.cu) compiles against the reference's
own headers, in its one- and two-temperature builds, with the reference's defines
(CMakeLists.txt) and the single-process MPI stand-in the reference-kernel runner uses.  It checks
that every reference name the shim reads (Parameter keys aside, which are runtime strings) exists
with the type the shim expects.  Needs the reference sources (COREFL_REFERENCE or the default
location); skipped where they are absent."""
import importlib.util
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SHIM = os.path.join(REPO, "corefl-cpc_b200", "shim", "cb200_shim.cu")


def _reference_dir():
    spec = importlib.util.spec_from_file_location("ref_build", os.path.join(REPO, "oracle", "ref_build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.reference_dir()


@pytest.mark.parametrize("two_t", [0, 1])
def test_shim_compiles_against_reference_headers(tmp_path, two_t):
    ref = _reference_dir()
    if ref is None:
        pytest.skip("reference sources not present")
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-std=c++17", "-rdc=true", "-gencode", "arch=compute_100a,code=sm_100a",
           "-DMAX_SPEC_NUMBER=9", "-DMAX_REAC_NUMBER=19", "-DMAX_PASSIVE_SCALAR_NUMBER=1", "-DCombustion2Part",
           "-DCOREFL_ENABLE_TWO_TEMPERATURE=%d" % two_t,
           "-I", os.path.join(REPO, "oracle", "ref"), "-I", os.path.join(ref, "src"),
           "-I", os.path.join(REPO, "include"), "-c", SHIM, "-o", str(tmp_path / "shim.o")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
