"""Cases run by the reference's own CUDA kernels (oracle/_ref/ref_stage_runner) and, with the same
inputs, by this library: the definitions, the writer of the reference's input files and the reader
of the runner's dumps.

A case is a dict (kept in the fixture, so a test rebuilds exactly the inputs the reference saw):
  family   "air" (calorically perfect air, curvilinear 3-D block), "mix" (9-species H2/air box),
           "air5" (two-temperature AIR5 box, the runner's two-temperature build) or "sod"
  name     unique key;  scheme / rec / visc: the reference's inviscid_scheme, reconstruction,
           viscous_order;  bc: "periodic" | "outflow";  stages: RK3 stages run from the initial
           state (1..3) or, for "sod", the run to t_end at CFL;  dt: the fixed step.
The reference sees the case through its own input files: input/setup.txt (the keys of
src/Parameter.cpp), the ASCII grid and boundary files that cfd::Mesh reads (src/Mesh.cpp:739-962),
state.bin (the initial bv / sv / T_ve and the metric / Jacobian of every padded node, which the
runner loads over the reference's own, so both sides use the same geometry) and task.txt.
"""
import hashlib
import math
import os
import shutil
import struct

import numpy as np

from cb200 import abi, cases, mech as mechmod
from cb200.field import box_faces

import helpers

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")

# reference data files each family reads (paths inside the reference tree)
H2_FILES = {"mechanism_file": "example/constantVolumeReactor/input/chemistry/2004-Li-IntJ.Chem.Kinet.inp",
            "therm_file": "example/reactiveShockTube/input/chemistry/therm.dat",
            "transport_file": "example/reactiveShockTube/input/chemistry/tran.dat"}
AIR5_DIR = "example/squareCylinder2D_M10_air5_dns/input/chemistry/"
AIR5_FILES = {"mechanism_file": AIR5_DIR + "air5_park.inp", "therm_file": AIR5_DIR + "therm.dat",
              "transport_file": AIR5_DIR + "tran.dat", "two_temperature_file": AIR5_DIR + "two_temperature.dat"}

AIR_DIMS = (10, 9, 8)
MIX_NODES = 8
CHAN_DIMS = (24, 16, 1)
# the channel's faces: supersonic inflow (i-), outflow (i+), isothermal wall (j-), symmetry (j+)
CHAN_INFLOW = dict(rho=1.1, u=2.5, p=1.0)
CHAN_WALL_T = 0.004
# the farfield channel: farfield (i- and j+), back-pressure outflow (i+), isothermal wall (j-)
CHAN_FARFIELD = dict(rho=1.1, u=0.6, p=1.0)
CHAN_BACK_PRESSURE = 1.05
# the blowing wall of the channel (Wall::if_blow_shock_wave): coefficient and step window
CHAN_BLOW = {"coefficient": 0.5, "start": 0, "end": 10}
# fully catalytic isothermal walls of the mixture boxes (low x face): wall temperature and the
# wall's mass fractions (Wall::yk), by species name
CAT_WALL = {"mix": (1000.0, {"H2O": 0.25, "N2": 0.75}), "air5": (2000.0, {"N2": 0.767, "O2": 0.233})}
# a non-reflecting outflow face: its type (and the label of its struct in the reference's setup)
BC_OUTFLOW_NR = abi.BC_OUTFLOW | abi.BC_NONREFLECTING


def ref_ngg(scheme, visc):
    """Ghost layers the reference allocates for a scheme (Parameter::deduce_known_info,
    src/Parameter.cpp:213-316)."""
    g = 2
    if scheme in (51, 52):
        g = 3
    if scheme in (71, 72):
        g = 4
    if visc == 8:
        g = max(g, 4)
    return g


def _air(name, scheme, rec, visc, bc, stages=3, dt=2e-3, seed=11):
    return dict(family="air", name=name, scheme=scheme, rec=rec, visc=visc, bc=bc, stages=stages, dt=dt,
                seed=seed, pp=0, limit_flow=0, reaction=0)


def _mix(name, scheme, rec, visc, reaction, pp=0, stages=3, dt=2e-9, bc="periodic", plt=0):
    return dict(family="mix", name=name, scheme=scheme, rec=rec, visc=visc, bc=bc, stages=stages, dt=dt,
                seed=2024, pp=pp, limit_flow=0, reaction=reaction, plt=plt)


def _air5(name, visc, reaction, pp=0, limit_flow=0, stages=3, dt=2e-9, bc="periodic", plt=0, scheme=52, rec=2):
    return dict(family="air5", name=name, scheme=scheme, rec=rec, visc=visc, bc=bc, stages=stages, dt=dt,
                seed=91, pp=pp, limit_flow=limit_flow, reaction=reaction, plt=plt)


def _chan(name, scheme, rec, visc, stages=3, dt=2e-3, bc="channel", plt=0):
    return dict(family="chan", name=name, scheme=scheme, rec=rec, visc=visc, bc=bc, stages=stages, dt=dt,
                seed=9, pp=0, limit_flow=0, reaction=0, plt=plt)


AIR_SCHEMES = [("weno5ch", 52, 2, 0), ("weno7ch", 72, 2, 0), ("weno5cp", 51, 2, 0), ("weno7cp", 71, 2, 0),
               ("ausm_muscl", 3, 2, 0), ("ausm_first", 3, 1, 0), ("hllc_nnd2", 4, 3, 0), ("hllc_muscl", 4, 2, 0),
               ("roe_muscl", 2, 2, 0), ("roe_first", 2, 1, 0), ("weno5ch_visc2", 52, 2, 2),
               ("weno7ch_visc8", 72, 2, 8), ("ausm_muscl_visc2", 3, 2, 2)]

CASES = ([_air(n + "_" + bc, s, r, v, bc) for n, s, r, v in AIR_SCHEMES for bc in ("periodic", "outflow")] +
         [_mix("mix_weno5ch_visc2_chem", 52, 2, 2, 1), _mix("mix_weno7ch", 72, 2, 0, 0),
          _mix("mix_weno5ch_pp", 52, 2, 0, 1, pp=1), _mix("mix_hllc_muscl_visc2", 4, 2, 2, 1),
          _mix("mix_ausm_muscl", 3, 2, 0, 0), _mix("mix_roe_muscl", 2, 2, 0, 0),
          _mix("mix_weno7ch_visc8", 72, 2, 8, 0)] +
         [_air5("air5_weno5ch_visc2_chem", 2, 1), _air5("air5_weno5ch_chem_pp_limit", 0, 1, pp=1, limit_flow=1),
          _air5("air5_weno5ch_visc2_outflow", 2, 1, bc="outflow"), _air5("air5_weno5ch_visc8_chem", 8, 1)] +
         [_chan("chan_hllc_muscl_visc2", 4, 2, 2), _chan("chan_weno5ch_visc2", 52, 2, 2),
          _chan("chan_roe_muscl", 2, 2, 0), _chan("chan_farfield_weno5ch", 52, 2, 0, bc="farfield"),
          _chan("chan_farfield_hllc_visc2", 4, 2, 2, bc="farfield"), _chan("chan_nr_weno5ch", 52, 2, 0, bc="nr", plt=1),
          _chan("chan_nr_ausm_muscl", 3, 2, 0, bc="nr"), _chan("chan_blow_weno5ch", 52, 2, 0, bc="blow"), _mix("mix_nr_weno5ch", 52, 2, 0, 0, bc="nr"),
          _mix("mix_catwall_weno5ch", 52, 2, 0, 0, bc="catwall", plt=1),
          _air5("air5_catwall_weno5ch", 0, 1, bc="catwall", plt=1),
          _air5("air5_hllc_muscl_visc2_chem", 2, 1, scheme=4), _air5("air5_ausm_muscl_chem", 0, 1, scheme=3)] +
         [dict(family="sod", name="sod_1000x7", scheme=52, rec=2, visc=0, bc="outflow", stages=0, dt=0.0, seed=0,
               pp=0, limit_flow=0, reaction=0, mx=1000, my=7, cfl=0.5, t_end=0.2)])


def case_by_name(name):
    for c in CASES:
        if c["name"] == name:
            return c
    raise KeyError(name)


# ---- inputs ---------------------------------------------------------------------------------
def _mech(family):
    if family == "mix":
        return mechmod.load_json(os.path.join(GOLDEN, "h2_li2004.json")), None
    if family == "air5":
        m = mechmod.load_json(os.path.join(GOLDEN, "air5_park.json"))
        tt = mechmod.load_two_temperature_json(os.path.join(GOLDEN, "air5_park.json"))
        return m, tt
    return None, None


def build(case):
    """(param, host_block, faces, extra) for a case; extra holds the mechanism objects, which must
    outlive the param's pointers into them."""
    fam = case["family"]
    g = ref_ngg(case["scheme"], case["visc"])
    if fam == "air":
        p, hb, faces = helpers.curvilinear_air_case(*AIR_DIMS, ngg=g, scheme=case["scheme"],
                                                    reconstruction=case["rec"], viscous_order=case["visc"],
                                                    bc=case["bc"], seed=case["seed"], mu=1e-3)
        extra = {}
    elif fam == "chan":
        from cb200.field import face
        mx, my, mz = CHAN_DIMS
        p, hb, _ = helpers.curvilinear_air_case(mx, my, mz, ngg=g, scheme=case["scheme"], reconstruction=case["rec"],
                                                viscous_order=case["visc"], bc="outflow", seed=case["seed"],
                                                jump=False, mu=1e-3)
        p.dim = 2
        # a planar 2-D grid: metrics and Jacobian the same on every k plane, no z components, w = 0
        # (the reference fills the wall/symmetry ghosts of the k-ghost planes once before its
        # first eliminate_k_gradient, src/Driver.cu:142-168, so k-varying metrics would leak in)
        for a in ("metric", "jac"):
            hb.a[a][...] = hb.a[a][:, g:g + 1]
        for c in (2, 5, 6, 7):
            hb.a["metric"][c] = 0.0
        hb.a["metric"][8] = 1.0
        hb.a["bv"][3] = 0.0
        cases.fill_cv_air(hb)
        ci = CHAN_INFLOW
        # T from (p, rho) as the reference's Inflow takes it: pressure * mw / (density * R_u)
        t_in = ci["p"] * cases.MW_AIR / (ci["rho"] * cases.R_U)
        if case["bc"] in ("farfield", "nr"):
            ff = CHAN_FARFIELD
            t_ff = ff["p"] * cases.MW_AIR / (ff["rho"] * cases.R_U)
            st = dict(rho=ff["rho"], u=ff["u"], v=0.0, w=0.0, p=ff["p"], T=t_ff)
            # the subsonic channel's exit: back pressure, or non-reflecting (its upstream wave clipped)
            exit_face = (face(abi.BC_OUTFLOW, 0, 1, (mx - 1, 0, 0), (mx - 1, my - 1, 0), p=CHAN_BACK_PRESSURE)
                         if case["bc"] == "farfield" else
                         face(BC_OUTFLOW_NR, 0, 1, (mx - 1, 0, 0), (mx - 1, my - 1, 0)))
            faces = [face(abi.BC_FARFIELD, 0, -1, (0, 0, 0), (0, my - 1, 0), **st), exit_face,
                     face(abi.BC_WALL, 1, -1, (0, 0, 0), (mx - 1, 0, 0), wall_temperature=CHAN_WALL_T),
                     face(abi.BC_FARFIELD, 1, 1, (0, my - 1, 0), (mx - 1, my - 1, 0), **st)]
        else:
            wall = face(abi.BC_WALL, 1, -1, (0, 0, 0), (mx - 1, 0, 0), wall_temperature=CHAN_WALL_T)
            if case["bc"] == "blow":
                # a blowing wall: the freestream velocity (ux_inf, uy_inf, uz_inf) of the reference
                # state and the blowing window
                wall.u, wall.v, wall.w = p.v_ref, 0.0, 0.0
                wall.blow_shock_wave = 1
                wall.blow_coefficient = CHAN_BLOW["coefficient"]
                wall.blow_start_step, wall.blow_end_step = CHAN_BLOW["start"], CHAN_BLOW["end"]
            faces = [face(abi.BC_INFLOW, 0, -1, (0, 0, 0), (0, my - 1, 0), rho=ci["rho"], u=ci["u"], v=0.0,
                          w=0.0, p=ci["p"], T=t_in),
                     face(abi.BC_OUTFLOW, 0, 1, (mx - 1, 0, 0), (mx - 1, my - 1, 0)), wall,
                     face(abi.BC_SYMMETRY, 1, 1, (0, my - 1, 0), (mx - 1, my - 1, 0))]
        extra = {}
    elif fam == "sod":
        c = cases.sod(mx=case["mx"], my=case["my"], ngg=g, scheme=case["scheme"], reconstruction=case["rec"],
                      cfl=case["cfl"])
        p, hb, faces = c.param, c.blocks[0], c.faces[0]
        extra = {}
    elif fam == "mix":
        m, _ = _mech(fam)
        c = cases.h2_air_box(m, n_nodes=MIX_NODES, ngg=g, seed=case["seed"], scheme=case["scheme"],
                             reconstruction=case["rec"], viscous_order=case["visc"], reaction=bool(case["reaction"]))
        p, hb, faces = c.param, c.blocks[0], c.faces[0]
        if case["bc"] == "catwall":
            faces = catalytic_wall_faces(fam, m, hb)
        if case["bc"] == "nr":  # x faces non-reflecting outflows, the others plain outflows
            faces = box_faces(hb.mx, hb.my, hb.mz,
                              {(d, s_): (BC_OUTFLOW_NR if d == 0 else abi.BC_OUTFLOW) for d in range(3)
                               for s_ in (-1, 1)})
        extra = {"mech": m}
    elif fam == "air5":
        m, tt = _mech(fam)
        c = cases.air5_box_2t(m, tt, n_nodes=MIX_NODES, ngg=g, seed=case["seed"], viscous_order=case["visc"],
                              reaction=bool(case["reaction"]), scheme=case["scheme"], reconstruction=case["rec"])
        p, hb, faces = c.param, c.blocks[0], c.faces[0]
        if case["bc"] == "outflow":
            faces = box_faces(hb.mx, hb.my, hb.mz, {(d, s_): abi.BC_OUTFLOW for d in range(3) for s_ in (-1, 1)})
        if case["bc"] == "catwall":
            faces = catalytic_wall_faces(fam, m, hb)
        extra = {"mech": m, "two_t": tt}
    else:
        raise ValueError(fam)
    p.positive_preserving = case["pp"]
    p.limit_flow = case["limit_flow"]
    p.dt = case["dt"]
    return p, hb, faces, extra


def catalytic_wall_faces(fam, m, hb):
    """A fully catalytic isothermal wall on the low x face, an outflow on the high one, periodic in
    y and z."""
    from cb200.field import face
    t_wall, yw = CAT_WALL[fam]
    y = np.zeros(m.ns)
    for name, v in yw.items():
        y[m.index(name)] = v
    mx, my, mz = hb.mx, hb.my, hb.mz
    faces = [face(abi.BC_WALL, 0, -1, (0, 0, 0), (0, my - 1, mz - 1), sv=y, wall_temperature=t_wall),
             face(abi.BC_OUTFLOW, 0, 1, (mx - 1, 0, 0), (mx - 1, my - 1, mz - 1))]
    faces += box_faces(mx, my, mz, {(d, s_): abi.BC_PERIODIC for d in (1, 2) for s_ in (-1, 1)})
    return faces


def state_arrays(case, hb):
    """The initial arrays state.bin carries, in its order (bv, sv, T_ve, metric, jac)."""
    out = [hb.a["bv"]]
    if "sv" in hb.a:
        out.append(hb.a["sv"])
    if case["family"] == "air5":
        out.append(hb.a["temperature_ve"])
    out += [hb.a["metric"], hb.a["jac"]]
    return out


def state_digest(case, hb):
    """SHA-256 of the initial arrays, and per component their sum, sum of |x| and sum of x^2.  The
    digest records the exact inputs; a test rebuilding them on another machine checks the sums
    (numpy's sin/cos may round differently on another CPU)."""
    h = hashlib.sha256()
    sums = []
    for a in state_arrays(case, hb):
        a = np.ascontiguousarray(a, dtype=np.float64)
        h.update(a.tobytes())
        for c in range(a.shape[0]):
            sums.append([float(a[c].sum()), float(np.abs(a[c]).sum()), float((a[c] ** 2).sum())])
    return {"sha256": h.hexdigest(), "sums": sums}


def same_state(d1, d2, rtol=1e-13):
    """True when two state digests describe the same inputs (up to last-bit rounding)."""
    if d1["sha256"] == d2["sha256"]:
        return True
    a, b = np.array(d1["sums"]), np.array(d2["sums"])
    return a.shape == b.shape and bool(np.all(np.abs(a - b) <= rtol * np.maximum(np.abs(b), 1e-300)))


# ---- the reference's input files -------------------------------------------------------------
def _face_lines(faces, dim):
    """boundary file lines "i1 i2 j1 j2 k1 k2 label" (0-based node ranges, src/Mesh.cpp:837-926)."""
    lines = []
    for f in faces:
        s, e = list(f.range_start), list(f.range_end)
        if dim == 2:
            s[2] = e[2] = 0
        lines.append("%d %d %d %d %d %d %d" % (s[0], e[0], s[1], e[1], s[2], e[2], f.type))
    return lines


BC_NAMES = {abi.BC_OUTFLOW: "outflow", abi.BC_PERIODIC: "periodic", abi.BC_SYMMETRY: "symmetry",
            abi.BC_WALL: "wall", abi.BC_INFLOW: "inflow", abi.BC_FARFIELD: "farfield",
            BC_OUTFLOW_NR: "outflow_nr"}
# the reference's type of each struct (a non-reflecting outflow is an outflow with its own label)
BC_TYPES = {**BC_NAMES, BC_OUTFLOW_NR: "outflow"}


def _coords(case, hb):
    """Node coordinates (interior) for the grid file: the reference computes its own metrics from
    them, which the runner then replaces with state.bin's, so they only need a valid grid."""
    mx, my, mz = hb.mx, hb.my, hb.mz
    if case["family"] in ("air", "chan"):
        n = max(AIR_DIMS if case["family"] == "air" else CHAN_DIMS) - 1
        (x, y, z), _, _ = cases.sine_wave_metrics(n, hb.ngg, 0.05)
        g = hb.ngg
        sl = (slice(g, g + mz), slice(g, g + my), slice(g, g + mx))
        if mz == 1:  # a 2-D grid lies in the plane z = 0
            return x[sl], y[sl], np.zeros_like(z[sl])
        return x[sl], y[sl], z[sl]
    if case["family"] == "sod":
        dx = 1.0 / (mx - 1)
        i = np.arange(mx) * dx
        j = np.arange(my) * 1.0
        Z, Y, X = np.meshgrid([0.0], j, i, indexing="ij")
        return X, Y, Z
    dx = 1e-3 / (mx - 1) if case["family"] == "mix" else 1e-2 / (mx - 1)
    q = np.arange(mx) * dx
    Z, Y, X = np.meshgrid(q, q, q, indexing="ij")
    return X, Y, Z


def write_reference_case(case, case_dir, ref_dir):
    """Writes the reference's input files for `case` into case_dir (data files copied from ref_dir)."""
    p, hb, faces, extra = build(case)
    fam = case["family"]
    dim = 2 if hb.mz == 1 else 3
    os.makedirs(os.path.join(case_dir, "input", "grid"), exist_ok=True)
    os.makedirs(os.path.join(case_dir, "input", "boundary_condition"), exist_ok=True)
    os.makedirs(os.path.join(case_dir, "output", "message"), exist_ok=True)
    x, y, z = _coords(case, hb)
    with open(os.path.join(case_dir, "input", "grid", "grid%4d.grd" % 0), "w") as f:
        f.write("1\n%d %d %d\n" % (hb.mx, hb.my, hb.mz))
        for arr in (x, y, z):
            f.write("\n".join("%.17g" % v for v in np.asarray(arr).ravel()) + "\n")
    with open(os.path.join(case_dir, "input", "boundary_condition", "boundary%4d.txt" % 0), "w") as f:
        lines = _face_lines(faces, dim)
        f.write("%d\n" % len(lines) + "\n".join(lines) + "\n")
    with open(os.path.join(case_dir, "input", "boundary_condition", "inner%4d.txt" % 0), "w") as f:
        f.write("1\n0\n\n")
    labels = sorted({f.type for f in faces})
    s = ["bool parallel = 0", "int gridIsBinary = 0", "int mesh_file_type = 0", "bool steady = 0",
         "int temporal_scheme = 3", "int total_step = 1000000", "int output_screen = 1000000",
         "int inviscid_scheme = %d" % case["scheme"], "int reconstruction = %d" % case["rec"], "int limiter = 0",
         "int viscous_order = %d" % case["visc"], "bool positive_preserving = %d" % case["pp"],
         "bool limit_flow = %d" % case["limit_flow"], "real prandtl_number = 0.72",
         "real entropy_fix_factor = 0.125", "int shock_sensor = 0", "real shockSensor_threshold = 0",
         "real shockSensor_epsilon = -1", "bool gradPInDiffusionFlux = 0",
         # 256-thread viscous blocks: the two-temperature viscous kernels hold too many registers for
         # the default 32 x 8 x 2 on sm_100a; the block shape does not change any result
         "array int viscous_flux_tpb_3d {", " 16 8 2", "}", "array int viscous_derivative_tpb_3d {", " 16 8 2", "}"]
    if fam == "sod":
        s += ["bool fixed_time_step = 0", "real cfl = %r" % case["cfl"],
              "real total_simulation_time = %r" % case["t_end"], "real dt = 1e-8"]
    else:
        s += ["bool fixed_time_step = 1", "real dt = %r" % case["dt"], "real cfl = 0.5"]
    if fam in ("mix", "air5"):
        files = H2_FILES if fam == "mix" else AIR5_FILES
        os.makedirs(os.path.join(case_dir, "input", "chemistry"), exist_ok=True)
        s += ["int species = 1", "int reaction = %d" % case["reaction"], "int chemSrcMethod = 0",
              "int therm_nasa_7_9 = %d" % (7 if fam == "mix" else 9)]
        for key, rel in files.items():
            shutil.copy(os.path.join(ref_dir, rel), os.path.join(case_dir, "input", "chemistry",
                                                                   os.path.basename(rel)))
            s.append("string %s = chemistry/%s" % (key, os.path.basename(rel)))
        if fam == "air5":
            s.append("bool enable_vt_relaxation = 1")
    else:
        s += ["int species = 0", "int reaction = 0"]
    s.append("array string boundary_conditions {")
    s += ["    %s" % BC_NAMES[t] for t in labels]
    s.append("}")
    for t in labels:
        s += ["struct %s {" % BC_NAMES[t], "    string type = %s" % BC_TYPES[t], "    int label = %d" % t]
        if t == BC_OUTFLOW_NR:
            s.append("    int nonReflecting = 1")
        if t == abi.BC_INFLOW:
            ci = CHAN_INFLOW
            s += ["    real density = %r" % ci["rho"], "    real velocity = %r" % ci["u"], "    real u = 1.0",
                  "    real v = 0.0", "    real w = 0.0", "    real pressure = %r" % ci["p"]]
        if t == abi.BC_WALL and case.get("bc") == "catwall":
            t_wall, yw = CAT_WALL[fam]
            s += ["    string thermal_type = isothermal", "    real temperature = %r" % t_wall,
                  "    int catalytic_type = 1"] + ["    real %s = %r" % (n, v) for n, v in yw.items()]
        elif t == abi.BC_WALL:
            s += ["    string thermal_type = isothermal", "    real temperature = %r" % CHAN_WALL_T]
            if case.get("bc") == "blow":
                s += ["    int if_blow_shock_wave = 1",
                      "    real blow_shock_wave_coefficient = %r" % CHAN_BLOW["coefficient"],
                      "    int blow_shock_wave_start_step = %d" % CHAN_BLOW["start"],
                      "    int blow_shock_wave_end_step = %d" % CHAN_BLOW["end"]]
        if t == abi.BC_FARFIELD:
            ff = CHAN_FARFIELD
            s += ["    real density = %r" % ff["rho"], "    real velocity = %r" % ff["u"], "    real u = 1.0",
                  "    real v = 0.0", "    real w = 0.0", "    real pressure = %r" % ff["p"]]
        if t == abi.BC_OUTFLOW and case.get("bc") == "farfield":
            s += ["    int if_backPressure = 1", "    real backPressure = %r" % CHAN_BACK_PRESSURE]
        s.append("}")
    # reference state: (density, velocity, pressure) of the case's reference values; the runner
    # builds the reference's Inflow from it (rho_inf, v_inf, p_inf, speed_of_sound)
    rho_ref, v_ref = p.rho_ref, p.v_ref
    s += ["string reference_state = refstate", "string default_init = refstate", "struct refstate {",
          "    string type = inflow", "    int label = 5", "    real density = %r" % rho_ref,
          "    real velocity = %r" % (v_ref if fam != "sod" else 0.0)]
    if fam in ("air", "sod", "chan"):
        s.append("    real pressure = %r" % 1.0)
    elif fam == "mix":
        s.append("    real pressure = %r" % 101325.0)
        m = extra["mech"]
        for name, yv in zip(m.species, mechmod.stoich_h2_air(m)):
            s.append("    real %s = %r" % (name, float(yv)))
    else:
        s.append("    real pressure = %r" % 2.0e4)
        for name, yv in zip(extra["mech"].species, (0.70, 0.10, 0.05, 0.05, 0.10)):
            s.append("    real %s = %r" % (name, yv))
    s.append("}")
    os.makedirs(os.path.join(case_dir, "input"), exist_ok=True)
    with open(os.path.join(case_dir, "input", "setup.txt"), "w") as f:
        f.write("\n".join(s) + "\n")
    with open(os.path.join(case_dir, "state.bin"), "wb") as f:
        for a in state_arrays(case, hb):
            f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    task = {"mode": "steps" if fam == "sod" else "stages", "stages": case["stages"], "dt": case["dt"],
            "fixed_dt": 0 if fam == "sod" else 1, "mul_constant": 1e-3 if fam in ("air", "chan") else 0.0,
            "load_metric": 1}
    if case.get("plt"):
        task["write_plt"] = 1  # the reference's own flowfield file of the final state
    if fam == "sod":
        task.update(n_steps=100000, t_end=case["t_end"])
    with open(os.path.join(case_dir, "task.txt"), "w") as f:
        f.write("".join("%s %r\n" % (k, v) if not isinstance(v, str) else "%s %s\n" % (k, v)
                        for k, v in task.items()))
    return state_digest(case, hb)


# ---- the runner's dump ------------------------------------------------------------------------
def read_dump(path):
    """Parses out.bin (oracle/ref/ref_stage_runner.cu, write section of run())."""
    with open(path, "rb") as f:
        buf = f.read()
    off = 0

    def ints(n):
        nonlocal off
        v = struct.unpack_from("<%di" % n, buf, off)
        off += 4 * n
        return v

    def dbl(n):
        nonlocal off
        v = np.frombuffer(buf, dtype="<f8", count=n, offset=off).copy()
        off += 8 * n
        return v

    n_block, steps, n_var, n_scalar, two_t, n_dq = ints(6)
    time, dt = dbl(2)
    refs = dbl(4)
    (n_dt,) = ints(1)
    dts = dbl(n_dt)
    blocks = []
    for _ in range(n_block):
        mx, my, mz, g = ints(4)
        npad = (mx + 2 * g) * (my + 2 * g) * (mz + 2 * g)
        shp = lambda c: (c, mz + 2 * g, my + 2 * g, mx + 2 * g)
        blk = {"dims": (mx, my, mz, g), "cv": dbl(npad * n_var).reshape(shp(n_var)),
               "bv": dbl(npad * 6).reshape(shp(6))}
        if n_scalar:
            blk["sv"] = dbl(npad * n_scalar).reshape(shp(n_scalar))
        if two_t:
            blk["temperature_ve"] = dbl(npad).reshape(shp(1))
        blocks.append(blk)
    dqs = []
    for s in range(n_dq):
        mx, my, mz, g = blocks[s % n_block]["dims"]
        dqs.append(dbl(mx * my * mz * n_var).reshape(n_var, mz, my, mx))
    return dict(steps=steps, time=time, dt=dt, rho_inf=refs[0], v_inf=refs[1], p_inf=refs[2],
                speed_of_sound=refs[3], dts=dts, blocks=blocks, dq=dqs)


def interior(a, g):
    return a[(slice(None), slice(g, -g), slice(g, -g), slice(g, -g))] if a.shape[1] > 2 * g else \
        a[(slice(None), slice(g, g + 1), slice(g, -g), slice(g, -g))]


# ---- the multi-block two-temperature square cylinder ("c5") -----------------------------------
C5_MINI = dict(n_side=12, n_normal=10, first=2e-4, half_box=0.03)


def _c5(name, visc=2, pp=1, limit_flow=1, stages=3, dt=1e-8):
    return dict(family="c5", name=name, scheme=52, rec=5, visc=visc, bc="cylinder", stages=stages, dt=dt, seed=0,
                pp=pp, limit_flow=limit_flow, reaction=1)


CASES.append(_c5("c5_air5_cylinder_4blocks"))
# the same grid with 8th-order viscous terms: node fluxes exchanged across the inner faces
CASES.append(_c5("c5_air5_cylinder_4blocks_visc8", visc=8))


def build_multi(case):
    """(param, blocks, faces per block, inner faces per block, extra) of a multi-block case."""
    m, tt = _mech("air5")
    c = cases.square_cylinder_air5(m, tt, ngg=ref_ngg(case["scheme"], case["visc"]), viscous_order=case["visc"],
                                   reaction=bool(case["reaction"]), **C5_MINI)
    p = c.param
    p.positive_preserving = case["pp"]
    p.limit_flow = case["limit_flow"]
    p.dt = case["dt"]
    return p, c.blocks, c.faces, c.meta["inner"], {"mech": m, "two_t": tt, "case": c}


def multi_state_digest(blocks):
    h = hashlib.sha256()
    sums = []
    for hb in blocks:
        d = state_digest({"family": "air5"}, hb)
        h.update(d["sha256"].encode())
        sums += d["sums"]
    return {"sha256": h.hexdigest(), "sums": sums}


def write_reference_multi(case, case_dir, ref_dir):
    """The reference's input files of a multi-block case (grid, boundary and inner-face files of
    every block, setup, state.bin with the blocks in order)."""
    p, blocks, faces, inner, extra = build_multi(case)
    c = extra["case"]
    g = c.meta["grid"]
    fs = c.meta["freestream"]
    nb = len(blocks)
    for d in ("grid", "boundary_condition", "chemistry"):
        os.makedirs(os.path.join(case_dir, "input", d), exist_ok=True)
    os.makedirs(os.path.join(case_dir, "output", "message"), exist_ok=True)
    with open(os.path.join(case_dir, "input", "grid", "grid%4d.grd" % 0), "w") as f:
        f.write("%d\n" % nb)
        for hb in blocks:
            f.write("%d %d %d\n" % (hb.mx, hb.my, hb.mz))
        for (x, y, z) in g["xyz"]:
            for arr in (x, y, z):
                f.write("\n".join("%.17g" % v for v in np.asarray(arr).ravel()) + "\n")
    with open(os.path.join(case_dir, "input", "boundary_condition", "boundary%4d.txt" % 0), "w") as f:
        for fl in g["faces"]:
            f.write("%d\n" % len(fl))
            for line in fl:
                f.write("%d %d %d %d %d %d %d\n" % line)
    with open(os.path.join(case_dir, "input", "boundary_condition", "inner%4d.txt" % 0), "w") as f:
        f.write("%d\n" % sum(len(x) for x in g["inner"]))
        f.write(" ".join("%d" % len(x) for x in g["inner"]) + "\n")
        f.write("iMin iMax jMin jMax kMin kMax id\n")
        for pairs in g["inner"]:
            for a, b in pairs:
                f.write("%d %d %d %d %d %d %d\n" % a)
                f.write("%d %d %d %d %d %d %d\n" % b)
    s = ["bool parallel = 0", "int gridIsBinary = 0", "int mesh_file_type = 0", "bool steady = 0",
         "int temporal_scheme = 3", "int total_step = 1000000", "int output_screen = 1000000",
         "int inviscid_scheme = %d" % case["scheme"], "int reconstruction = 2", "int limiter = 0",
         "int viscous_order = %d" % case["visc"], "bool positive_preserving = %d" % case["pp"],
         "bool limit_flow = %d" % case["limit_flow"], "real prandtl_number = 0.72", "int shock_sensor = 0",
         "real shockSensor_threshold = 0", "real shockSensor_epsilon = -1", "bool gradPInDiffusionFlux = 0",
         "bool fixed_time_step = 1", "real dt = %r" % case["dt"], "real cfl = 0.3",
         "int species = 1", "int reaction = %d" % case["reaction"], "int chemSrcMethod = 0", "int therm_nasa_7_9 = 9",
         "bool enable_vt_relaxation = 1"]
    for key, rel in AIR5_FILES.items():
        shutil.copy(os.path.join(ref_dir, rel), os.path.join(case_dir, "input", "chemistry", os.path.basename(rel)))
        s.append("string %s = chemistry/%s" % (key, os.path.basename(rel)))
    names = extra["mech"].species
    s += ["array string boundary_conditions {", "    freestream outflow wall", "}",
          "struct freestream {", "    string type = inflow", "    int label = 5", "    int inflow_type = 0",
          "    real velocity = %r" % fs["u"], "    real temperature = %r" % fs["T"], "    real Tve = %r" % fs["Tve"],
          "    real pressure = %r" % fs["p"], "    real u = 1.0", "    real v = 0.0", "    real w = 0.0"]
    s += ["    real %s = %r" % (n, float(yv)) for n, yv in zip(names, fs["y"])]
    s += ["}", "struct outflow {", "    string type = outflow", "    int label = 6", "}",
          "struct wall {", "    string type = wall", "    int label = 2", "    string thermal_type = isothermal",
          "    real temperature = 300.0", "    real Tve = 300.0", "}",
          "string reference_state = freestream", "string default_init = freestream"]
    with open(os.path.join(case_dir, "input", "setup.txt"), "w") as f:
        f.write("\n".join(s) + "\n")
    with open(os.path.join(case_dir, "state.bin"), "wb") as f:
        for hb in blocks:
            for a in state_arrays({"family": "air5"}, hb):
                f.write(np.ascontiguousarray(a, dtype=np.float64).tobytes())
    task = {"mode": "stages", "stages": case["stages"], "dt": case["dt"], "fixed_dt": 1, "mul_constant": 0.0,
            "load_metric": 1}
    if case.get("plt"):
        task["write_plt"] = 1  # the reference's own flowfield file of the final state
    with open(os.path.join(case_dir, "task.txt"), "w") as f:
        f.write("".join(("%s %s\n" if isinstance(v, str) else "%s %r\n") % (k, v) for k, v in task.items()))
    return multi_state_digest(blocks)
