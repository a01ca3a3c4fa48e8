"""Reference GPU baseline: the reference's own CUDA kernels (oracle/_ref/ref_stage_runner, built by
oracle/ref_gpu_build.py) timed on the benchmark configurations beside this library on the same
GPU.  TEST INFRASTRUCTURE ONLY (a measurement of the reference, not of the library's product path).

Each configuration runs the same scheme combination on the same grid in both: the reference runs
its RK3 stage sequence (src/RK.cuh:107-237) through its own setup, mesh, field and boundary code;
the library runs cb2_rk3_step (and cb2_rk3_run where the step is device-driven).  Both are timed
with CUDA events over the same number of steps after warm-up steps.
  c2   sine wave, 257^3 nodes curvilinear periodic, WENO7 characteristic + 8th-order viscous,
       fixed dt (the reference has no WENO7 + AUSM+ kernel, so its closest scheme is timed)
  c3   H2/air box, 192^3 nodes periodic, 9 species / 19 reactions, HLLC + MUSCL, 2nd-order
       viscous, chemistry, dt 2e-9 s (the reference's closest scheme to WENO5 + HLLC)
  c1   Sod tube, 1000 x 7 nodes, WENO5 characteristic, CFL 0.5, the reference's CFL step
  c5   two-temperature AIR5 square cylinder, four blocks of 256 x 512 nodes, WENO5
       characteristic, positivity limiter, 2nd-order viscous, Park chemistry, limit_flow, CFL 0.3
The reference's state starts from its own uniform initial condition (c2, c3) or from the same
state file as the library (c1, c5); timing does not depend on the values.

  python oracle/ref_gpu_time.py write --work DIR [--ref REFDIR]   (build container: setup files)
  python oracle/ref_gpu_time.py run --work DIR [--only c2,c3]     (GPU: grids, states, both timings)
"""
import argparse
import json
import math
import os
import shutil
import subprocess
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path[:0] = [os.path.join(REPO, "corefl-cpc_b200"), os.path.join(REPO, "tests")]

import numpy as np  # noqa: E402

GOLD = os.path.join(REPO, "tests", "golden")
CONFIGS = ("c2", "c3", "c1", "c5")


def _setup_lines(scheme, rec, visc, fixed_dt, dt, cfl, species, extra):
    s = ["bool parallel = 0", "int gridIsBinary = 1", "int mesh_file_type = 0", "bool steady = 0", "int initial = 0",
         "int temporal_scheme = 3", "int total_step = 100000000", "int output_screen = 100000000",
         "int inviscid_scheme = %d" % scheme, "int reconstruction = %d" % rec, "int limiter = 0",
         "int viscous_order = %d" % visc, "real prandtl_number = 0.72", "real entropy_fix_factor = 0.125",
         "int shock_sensor = 0", "real shockSensor_threshold = 0", "real shockSensor_epsilon = -1",
         "bool fixed_time_step = %d" % (1 if fixed_dt else 0), "real dt = %r" % dt, "real cfl = %r" % cfl,
         "array int viscous_flux_tpb_3d {", " 16 8 2", "}", "array int viscous_derivative_tpb_3d {", " 16 8 2", "}"]
    s += species
    s += extra
    return s


def _copy_chem(ref, case_dir, files):
    os.makedirs(os.path.join(case_dir, "input", "chemistry"), exist_ok=True)
    out = []
    for key, rel in files.items():
        shutil.copy(os.path.join(ref, rel), os.path.join(case_dir, "input", "chemistry", os.path.basename(rel)))
        out.append("string %s = chemistry/%s" % (key, os.path.basename(rel)))
    return out


def write(args):
    import refcases
    sys.path.insert(0, HERE)
    import ref_build
    ref = ref_build.reference_dir(args.ref)
    if ref is None:
        sys.exit("reference sources not found: pass --ref or set COREFL_REFERENCE")
    for name in CONFIGS:
        d = os.path.join(args.work, name)
        for sub in ("grid", "boundary_condition"):
            os.makedirs(os.path.join(d, "input", sub), exist_ok=True)
        os.makedirs(os.path.join(d, "output", "message"), exist_ok=True)
        if name == "c2":
            s = _setup_lines(72, 2, 8, True, 6.517965367111679e-4, 0.5, ["int species = 0", "int reaction = 0"],
                             ["array string boundary_conditions {", "    periodic", "}",
                              "struct periodic {", "    string type = periodic", "    int label = 8", "}",
                              "string reference_state = freestream", "string default_init = freestream",
                              "struct freestream {", "    string type = inflow", "    int label = 5",
                              "    real density = 1.0", "    real velocity = 1.7320508075688772",
                              "    real u = 0.5773502691896258", "    real v = 0.5773502691896258",
                              "    real w = 0.5773502691896258", "    real pressure = 1.0", "}"])
        elif name == "c3":
            chem = _copy_chem(ref, d, refcases.H2_FILES)
            m = refcases._mech("mix")[0]
            from cb200 import mech as mechmod
            y = mechmod.stoich_h2_air(m)
            s = _setup_lines(4, 2, 2, True, 2e-9, 0.5, ["int species = 1", "int reaction = 1", "int chemSrcMethod = 0",
                                                         "int therm_nasa_7_9 = 7"] + chem,
                             ["array string boundary_conditions {", "    periodic", "}",
                              "struct periodic {", "    string type = periodic", "    int label = 8", "}",
                              "string reference_state = freestream", "string default_init = freestream",
                              "struct freestream {", "    string type = inflow", "    int label = 5",
                              "    real temperature = 1200.0", "    real pressure = 101325.0", "    real velocity = 10.0",
                              "    real u = 1.0", "    real v = 0.0", "    real w = 0.0"] +
                             ["    real %s = %r" % (n, float(v)) for n, v in zip(m.species, y)] + ["}"])
        elif name == "c1":
            s = _setup_lines(52, 2, 0, False, 1e-8, 0.5, ["int species = 0", "int reaction = 0"],
                             ["real total_simulation_time = 0.2", "array string boundary_conditions {", "    outflow",
                              "}", "struct outflow {", "    string type = outflow", "    int label = 6", "}",
                              "string reference_state = refstate", "string default_init = refstate",
                              "struct refstate {", "    string type = inflow", "    int label = 5",
                              "    real density = 1.0", "    real velocity = 0.0", "    real pressure = 1.0", "}"])
        else:  # c5
            chem = _copy_chem(ref, d, refcases.AIR5_FILES)
            m = refcases._mech("air5")[0]
            from cb200 import cases
            tt = refcases._mech("air5")[1]
            fs = cases.air5_freestream(m, tt)
            s = _setup_lines(52, 2, 2, False, 1e-10, 0.3, ["int species = 1", "int reaction = 1", "int chemSrcMethod = 0",
                                                           "int therm_nasa_7_9 = 9", "bool enable_vt_relaxation = 1",
                                                           "bool positive_preserving = 1", "bool limit_flow = 1"] + chem,
                             ["array string boundary_conditions {", "    freestream outflow wall", "}",
                              "struct freestream {", "    string type = inflow", "    int label = 5",
                              "    int inflow_type = 0", "    real velocity = %r" % fs["u"],
                              "    real temperature = %r" % fs["T"], "    real Tve = %r" % fs["Tve"],
                              "    real pressure = %r" % fs["p"], "    real u = 1.0", "    real v = 0.0",
                              "    real w = 0.0"] +
                             ["    real %s = %r" % (n, float(v)) for n, v in zip(m.species, fs["y"])] +
                             ["}", "struct outflow {", "    string type = outflow", "    int label = 6", "}",
                              "struct wall {", "    string type = wall", "    int label = 2",
                              "    string thermal_type = isothermal", "    real temperature = 300.0",
                              "    real Tve = 300.0", "}", "string reference_state = freestream",
                              "string default_init = freestream"])
        with open(os.path.join(d, "input", "setup.txt"), "w") as f:
            f.write("\n".join(s) + "\n")
        print("wrote", d)


def _write_grid_binary(case_dir, xyz):
    """The binary grid the reference's Mesh reads (gridIsBinary = 1, src/Mesh.cpp:702-738)."""
    with open(os.path.join(case_dir, "input", "grid", "grid%4d.dat" % 0), "wb") as f:
        np.array([len(xyz)], dtype=np.int32).tofile(f)
        for x, _, _ in xyz:
            np.array([x.shape[2], x.shape[1], x.shape[0]], dtype=np.int32).tofile(f)
        for x, y, z in xyz:
            for a in (x, y, z):
                np.ascontiguousarray(a, dtype=np.float64).tofile(f)


def _write_faces(case_dir, faces_raw, inner_raw):
    with open(os.path.join(case_dir, "input", "boundary_condition", "boundary%4d.txt" % 0), "w") as f:
        for fl in faces_raw:
            f.write("%d\n" % len(fl))
            for line in fl:
                f.write("%d %d %d %d %d %d %d\n" % tuple(line))
    with open(os.path.join(case_dir, "input", "boundary_condition", "inner%4d.txt" % 0), "w") as f:
        f.write("%d\n" % sum(len(x) for x in inner_raw))
        f.write(" ".join("%d" % len(x) for x in inner_raw) + "\n")
        f.write("iMin iMax jMin jMax kMin kMax id\n")
        for pairs in inner_raw:
            for a, b in pairs:
                f.write("%d %d %d %d %d %d %d\n" % a)
                f.write("%d %d %d %d %d %d %d\n" % b)


def _box_faces_raw(m, periodic_or_outflow, dim=3, my=None):
    lab = periodic_or_outflow
    mx, myy, mz = m
    out = [(0, 0, 0, myy - 1, 0, mz - 1, lab), (mx - 1, mx - 1, 0, myy - 1, 0, mz - 1, lab),
           (0, mx - 1, 0, 0, 0, mz - 1, lab), (0, mx - 1, myy - 1, myy - 1, 0, mz - 1, lab)]
    if dim == 3:
        out += [(0, mx - 1, 0, myy - 1, 0, 0, lab), (0, mx - 1, 0, myy - 1, mz - 1, mz - 1, lab)]
    return out


def _run_reference(case_dir, family, task, timeout):
    with open(os.path.join(case_dir, "task.txt"), "w") as f:
        for k, v in task.items():
            f.write("%s %s\n" % (k, v))
    exe = os.path.join(HERE, "_ref", "ref_stage_runner" + ("_2t" if family == "c5" else ""))
    t0 = time.perf_counter()
    r = subprocess.run([exe, os.path.abspath(case_dir)], capture_output=True, text=True, timeout=timeout)
    wall = time.perf_counter() - t0
    if r.returncode != 0:
        return {"error": (r.stdout[-800:] + r.stderr[-800:])}
    with open(os.path.join(case_dir, "time.txt")) as f:
        n, ms, dt = f.read().split()
    return {"steps": int(n), "ms_per_step": float(ms), "dt_last": float(dt), "process_wall_s": wall}


def _time_lib(ctx, nb, steps, warm, dt, fixed, sh, graph=False):
    import torch
    for _ in range(warm):
        ctx.rk3_step(dt, fixed, sh)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s = torch.cuda.current_stream()
    e0.record(s)
    if graph:
        _, n, _ = ctx.rk3_run(steps, fixed_dt=fixed, dt=dt, stream=sh)
    else:
        n = steps
        for _ in range(steps):
            ctx.rk3_step(dt, fixed, sh)
    e1.record(s)
    torch.cuda.synchronize()
    return {"steps": n, "ms_per_step": e0.elapsed_time(e1) / max(n, 1), "status": ctx.read_status(sh)}


def run(args):
    import torch
    import cb200
    from cb200 import abi, cases, mech as mechmod
    from cb200.field import DeviceBlock
    import refcases
    torch.cuda.set_device(0)
    sh = torch.cuda.current_stream().cuda_stream
    only = args.only.split(",") if args.only else CONFIGS
    results = {}
    for name in only:
        d = os.path.join(args.work, name)
        res = {}
        if name == "c2":
            n = args.c2_n
            c = cases.sine_wave(n=n, scheme=abi.INV_WENO7_CH, reconstruction=abi.REC_MUSCL, viscous_order=8)
            (X, Y, Z), _, _ = cases.sine_wave_metrics(n, 4, 0.05)
            g = 4
            sl = (slice(g, g + n + 1),) * 3
            _write_grid_binary(d, [(X[sl], Y[sl], Z[sl])])
            _write_faces(d, [_box_faces_raw((n + 1, n + 1, n + 1), 8)], [[]])
            nodes = (n + 1) ** 3
            res["reference"] = _run_reference(d, "c2", {"mode": "time", "init": "reference", "fixed_dt": 1,
                                                        "dt": c.meta.get("dt", 6.517965367111679e-4), "warmup": 2,
                                                        "n_steps": args.steps}, args.timeout)
            p, hb, faces = c.param, c.blocks[0], c.faces[0]
            dev = DeviceBlock(hb)
            del c, hb
            ctx = cb200.Context(p)
            ctx.bind(0, dev.view(), faces)
            ctx.properties(0, sh)
            res["library"] = _time_lib(ctx, 1, args.steps, 2, 6.517965367111679e-4, True, sh)
            ctx.close()
            del dev
        elif name == "c3":
            n = args.c3_n
            m = mechmod.load_json(os.path.join(GOLD, "h2_li2004.json"))
            c = cases.h2_air_box(m, n_nodes=n, scheme=abi.INV_HLLC, reconstruction=abi.REC_MUSCL, viscous_order=2)
            q = np.arange(n) * c.meta["dx"]
            Z3, Y3, X3 = np.meshgrid(q, q, q, indexing="ij")
            _write_grid_binary(d, [(X3, Y3, Z3)])
            _write_faces(d, [_box_faces_raw((n, n, n), 8)], [[]])
            nodes = n ** 3
            res["reference"] = _run_reference(d, "c3", {"mode": "time", "init": "reference", "fixed_dt": 1,
                                                        "dt": 2e-9, "warmup": 2, "n_steps": args.steps},
                                              args.timeout)
            p, hb, faces = c.param, c.blocks[0], c.faces[0]
            dev = DeviceBlock(hb)
            del c, hb
            ctx = cb200.Context(p)
            ctx.bind(0, dev.view(), faces)
            ctx.properties(0, sh)
            res["library"] = _time_lib(ctx, 1, args.steps, 2, 2e-9, True, sh)
            ctx.close()
            del dev
        elif name == "c1":
            case = refcases.case_by_name("sod_1000x7")
            p, hb, faces, _ = refcases.build(case)
            dx = 1.0 / 999
            Z1, Y1, X1 = np.meshgrid([0.0], np.arange(7) * 1.0, np.arange(1000) * dx, indexing="ij")
            _write_grid_binary(d, [(X1, Y1, Z1)])
            _write_faces(d, [_box_faces_raw((1000, 7, 1), 6, dim=2)], [[]])
            with open(os.path.join(d, "state.bin"), "wb") as f:
                for a in refcases.state_arrays(case, hb)[:-2]:
                    f.write(np.ascontiguousarray(a).tobytes())
            nodes = 7000
            res["reference"] = _run_reference(d, "c1", {"mode": "time", "init": "file", "fixed_dt": 0, "warmup": 0,
                                                        "n_steps": 874, "load_metric": 0}, args.timeout)
            dev = DeviceBlock(hb)
            ctx = cb200.Context(p)
            ctx.bind(0, dev.view(), faces)
            ctx.properties(0, sh)
            ctx.boundary(0, sh)
            ctx.properties(0, sh)
            ctx.cv_from_bv(0, sh)
            res["library"] = _time_lib(ctx, 1, 874, 0, 0.0, False, sh)
            dev.load(hb)
            ctx.properties(0, sh)
            res["library_graph"] = _time_lib(ctx, 1, 874, 0, 0.0, False, sh, graph=True)
            ctx.close()
        else:  # c5
            m, tt = refcases._mech("air5")
            c = cases.square_cylinder_air5(m, tt, n_side=args.c5_side, n_normal=args.c5_normal)
            g = c.meta["grid"]
            _write_grid_binary(d, g["xyz"])
            _write_faces(d, g["faces"], g["inner"])
            with open(os.path.join(d, "state.bin"), "wb") as f:
                for hb in c.blocks:
                    for a in refcases.state_arrays({"family": "air5"}, hb)[:-2]:
                        f.write(np.ascontiguousarray(a).tobytes())
            nodes = sum(hb.mx * hb.my for hb in c.blocks)
            res["reference"] = _run_reference(d, "c5", {"mode": "time", "init": "file", "fixed_dt": 0,
                                                        "warmup": args.c5_warmup, "n_steps": args.c5_steps,
                                                        "load_metric": 0}, args.timeout)
            p = c.param
            p.positive_preserving, p.limit_flow = 1, 1
            devs = [DeviceBlock(hb) for hb in c.blocks]
            ctx = cb200.Context(p)
            for b in range(4):
                ctx.bind(b, devs[b].view(), c.faces[b])
                ctx.bind_inner_faces(b, c.meta["inner"][b])
            for fn in (ctx.properties, ctx.boundary):
                for b in range(4):
                    fn(b, sh)
            ctx.halo(sh)
            for fn in (ctx.properties, ctx.cv_from_bv):
                for b in range(4):
                    fn(b, sh)
            for _ in range(args.c5_warmup):
                ctx.rk3_step(0.0, False, sh)
            res["library"] = _time_lib(ctx, 4, args.c5_steps, 0, 0.0, False, sh)
            res["library_graph"] = _time_lib(ctx, 4, args.c5_steps, 0, 0.0, False, sh, graph=True)
            ctx.close()
            del devs
        res["nodes"] = nodes
        for k in ("reference", "library", "library_graph"):
            if k in res and "ms_per_step" in res[k]:
                res[k]["cell_updates_per_s"] = nodes / (res[k]["ms_per_step"] * 1e-3)
        if "ms_per_step" in res.get("reference", {}) and "ms_per_step" in res.get("library", {}):
            res["speedup_library_vs_reference"] = res["reference"]["ms_per_step"] / res["library"]["ms_per_step"]
        results[name] = res
        print(name, json.dumps(res), flush=True)
        torch.cuda.empty_cache()
    with open(args.out, "w") as f:
        json.dump(results, f, indent=1)


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    w = sub.add_parser("write")
    w.add_argument("--work", required=True)
    w.add_argument("--ref", default=None)
    r = sub.add_parser("run")
    r.add_argument("--work", required=True)
    r.add_argument("--out", default="ref_gpu_time.json")
    r.add_argument("--only", default=None)
    r.add_argument("--steps", type=int, default=5)
    r.add_argument("--c2-n", type=int, default=256)
    r.add_argument("--c3-n", type=int, default=192)
    r.add_argument("--c5-side", type=int, default=256)
    r.add_argument("--c5-normal", type=int, default=512)
    r.add_argument("--c5-steps", type=int, default=50)
    r.add_argument("--c5-warmup", type=int, default=20)
    r.add_argument("--timeout", type=float, default=900)
    a = ap.parse_args()
    {"write": write, "run": run}[a.cmd](a)


if __name__ == "__main__":
    main()
