"""Write the mechanism fixtures of tests/golden/ with the reference's own parser.

Runs oracle/_ref/dump_mech (cfd::Species + cfd::Reaction of the reference, built by
oracle/ref_build.py) on the reference's example data files and keeps its JSON output:
  h2_li2004.json : 9 species / 19 reactions, Li et al. 2004 H2/O2 mechanism
                   (example/constantVolumeReactor/input/chemistry/2004-Li-IntJ.Chem.Kinet.inp)
                   with NASA7 thermo and transport from example/reactiveShockTube/input/chemistry/
                   (therm_nasa_7_9 = 7)
  h2_chem_states.json : 48 seeded (rho, T, Y) states with the reference's host chemistry
                   source cfd::compute_src, h_k/cp_k from Species::compute_enthalpy_and_cp and
                   the Newton temperature of cfd::update_t (src/ConstVolumeReactor.cpp)
  h2_two_temperature.json : the vibrational-electronic data of two_temperature.dat
                   (example/squareCylinder2D_M10_air5_dns/input/chemistry/) as
                   Species::read_two_temperature parses it for the 9 H2/air species, the
                   species e_ve / cv_ve of Species::compute_ve_energy / compute_ve_cv on a
                   temperature ladder, and on 40 seeded (rho, T, Tve, Y) states the mixture
                   e_ve, Species::invert_tve_from_eve and cfd::compute_vt_relaxation_source
  air5_park.json : the AIR5 two-temperature case (5 species, Park's 17 dissociation and exchange
                   reactions of example/squareCylinder2D_M10_air5_dns/input/chemistry/) with NASA9
                   multi-range thermo and the AIR5 control-temperature model: the tables, species
                   h / cp / g/RT / e_ve / cv_ve on a temperature ladder, and on 32 seeded
                   (rho, T, Tve, Y) states the source of compute_src(T, Tve), the e_ve chemical
                   source and update_t_two_temperature
  h2_reactor_runs.json : 0-D reactors run with the reference's host chemistry, Jacobian, LU
                   and Newton through the adaptive ROK4E sequence (RTol 1e-6, ATol 1e-12,
                   first step 1e-8): the reference's example case to 1.2 ms and 8 seeded
                   (T0, p0, phi) requests to 1 ms, each after 8 step attempts and at the end
  h2_reactor_fixed_runs.json : the same reactors (the example case and 2 seeded requests) with
                   the fixed-step forms of const_volume_reactor, the reference's own EPI and DA:
                   explicit and EPI (each also with conserve_mass_corefl), DA and the explicit
                   three-stage Runge-Kutta (dt 1e-9 to 20 us, DA to 50 us, EPI dt 1e-7 to 0.4 ms), after 100
                   steps and at the end
  h2_reactor_krylov_runs.json : the example case and 2 seeded requests through the ROK4E sequence
                   with build_arnoldi = 1 (cfd::buildArnoldi, Krylov limit MAX_SPEC_NUMBER = 9),
                   after 8 and after 2000 attempts (its steps shrink until they stall short of
                   t_end: 1e6 attempts end at 0.82 ms, 0.30 ms and 19 us of 1.2, 1 and 1 ms)
Usage: python tests/golden/make_mech.py [/path/to/reference]  (default: oracle/ref_build.py's
reference_dir())
"""
import os
import shutil
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def run(ref, name, files, nasa, prog="dump_mech", extra=()):
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import importlib.util
    spec = importlib.util.spec_from_file_location("ref_build", os.path.join(REPO, "oracle", "ref_build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    exe = mod.build(ref)
    with tempfile.TemporaryDirectory() as d:
        os.makedirs(os.path.join(d, "input", "chemistry"))
        for key, rel in files.items():
            shutil.copy(os.path.join(ref, rel), os.path.join(d, "input", "chemistry", os.path.basename(rel)))
        setup = os.path.join(d, "setup.txt")
        with open(setup, "w") as f:
            f.write("int species = 1\nint reaction = 1\nint myid = 0\nint chemSrcMethod = 0\n"
                    "int n_var = 5\nint n_scalar = 0\n")
            f.write(f"int therm_nasa_7_9 = {nasa}\n")
            for key, rel in files.items():
                f.write(f"string {key} = chemistry/{os.path.basename(rel)}\n")
        out = os.path.join(HERE, name)
        exe_p = os.path.join(os.path.dirname(exe), prog)
        r = subprocess.run([exe_p, setup, out, *extra], cwd=d, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(r.stdout + r.stderr)
    return out


def main(ref):
    chem = "example/reactiveShockTube/input/chemistry/"
    files = {"mechanism_file": "example/constantVolumeReactor/input/chemistry/2004-Li-IntJ.Chem.Kinet.inp",
             "therm_file": chem + "therm.dat", "transport_file": chem + "tran.dat"}
    print(run(ref, "h2_li2004.json", files, 7))
    print(run(ref, "h2_chem_states.json", files, 7, prog="dump_chem", extra=("48",)))
    print(run(ref, "h2_reactor_runs.json", files, 7, prog="dump_reactor", extra=("9",)))
    print(run(ref, "h2_reactor_fixed_runs.json", files, 7, prog="dump_reactor", extra=("3", "fixed")))
    print(run(ref, "h2_reactor_krylov_runs.json", files, 7, prog="dump_reactor", extra=("3", "krylov")))
    files_2t = dict(files, two_temperature_file="example/squareCylinder2D_M10_air5_dns/input/chemistry/"
                                                "two_temperature.dat")
    print(run(ref, "h2_two_temperature.json", files_2t, 7, prog="dump_2t", extra=("40",)))
    air = "example/squareCylinder2D_M10_air5_dns/input/chemistry/"
    files_air5 = {"mechanism_file": air + "air5_park.inp", "therm_file": air + "therm.dat",
                  "transport_file": air + "tran.dat", "two_temperature_file": air + "two_temperature.dat"}
    print(run(ref, "air5_park.json", files_air5, 9, prog="dump_air5", extra=("32",)))


if __name__ == "__main__":
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))
    import ref_build
    ref = ref_build.reference_dir(sys.argv[1] if len(sys.argv) > 1 else None)
    if ref is None:
        sys.exit("reference sources not found: pass the path or set COREFL_REFERENCE")
    main(ref)
