"""Device-driven time loop (cb2_rk3_run): one CUDA graph launch whose WHILE node repeats a
captured step.  Its steps must be bitwise identical to as many cb2_rk3_step calls, and its
stop test must match the reference's host loop (physical_time += dt until it reaches
total_simulation_time, src/RK.cuh:240-261)."""
import os

import numpy as np
import pytest

import cb200
from cb200 import abi, cases, mech as mechmod
from cb200.field import DeviceBlock

import helpers

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _pair(p, hb, faces):
    """Two device copies of one host block, each bound to its own context."""
    out = []
    for _ in range(2):
        dev = DeviceBlock(hb)
        ctx = cb200.Context(p)
        ctx.bind(0, dev.view(), faces)
        out.append((dev, ctx))
    return out


def _same(a, b, names):
    ha, hb_ = a.to_host(names), b.to_host(names)
    for n in names:
        assert np.array_equal(ha[n], hb_[n]), n


def test_graph_cfl_steps_match_host_loop(oracle_lib):
    """Sod tube, WENO5-ch, CFL dt computed on the device every step: 40 steps."""
    case = cases.sod(mx=1000)
    b, faces, p = case.blocks[0], case.faces[0], case.param
    oracle_lib.boundary(p, b, faces)
    (d0, c0), (d1, c1) = _pair(p, b, faces)
    t_host, dts = 0.0, []
    for _ in range(40):
        dt = c0.rk3_step(0.0, fixed_dt=False)
        dts.append(dt)
        t_host += dt
    t_dev, steps, dt_last = c1.rk3_run(40)
    assert steps == 40
    assert t_dev == t_host
    assert dt_last == dts[-1]
    _same(d0, d1, ["cv", "bv"])
    # the graph runs the host loop's kernels plus one loop-control kernel per step
    assert c1.launch_count() == c0.launch_count() + 40
    assert c0.read_status() == 0 and c1.read_status() == 0


def test_graph_stops_at_end_time(oracle_lib):
    """The loop ends on the first step whose time reaches t_end, as the host loop does."""
    case = cases.sod(mx=1000)
    b, faces, p = case.blocks[0], case.faces[0], case.param
    oracle_lib.boundary(p, b, faces)
    (d0, c0), (d1, c1) = _pair(p, b, faces)
    t_end = 0.02
    t_host, n_host = 0.0, 0
    while t_host < t_end:
        t_host += c0.rk3_step(0.0, fixed_dt=False)
        n_host += 1
    t_dev, steps, _ = c1.rk3_run(10 ** 6, t_end=t_end)
    assert steps == n_host and t_dev == t_host
    _same(d0, d1, ["cv", "bv"])
    # a second call continues from the time reached; at t >= t_end it takes no step
    assert c1.rk3_run(10, t_end=t_end, time=t_dev)[1] == 0
    t2, s2, _ = c1.rk3_run(5, t_end=1.0, time=t_dev)
    for _ in range(5):
        t_host += c0.rk3_step(0.0, fixed_dt=False)
    assert s2 == 5 and t2 == t_host
    _same(d0, d1, ["cv"])


@pytest.mark.parametrize("scheme,rec,visc", [(abi.INV_AUSMP, abi.REC_WENO7, 8), (abi.INV_WENO7_CH, abi.REC_MUSCL, 0),
                                             (abi.INV_ROE, abi.REC_MUSCL, 0)], ids=["ausm_weno7_visc8", "weno7ch", "roe"])
def test_graph_fixed_dt_matches_host_loop(oracle_lib, scheme, rec, visc):
    p, hb, faces = helpers.curvilinear_air_case(20, 18, 16, scheme=scheme, reconstruction=rec, viscous_order=visc,
                                                bc="periodic", seed=4)
    oracle_lib.boundary(p, hb, faces)
    dt = 0.2 * oracle_lib.cfl_dt(p, hb)
    (d0, c0), (d1, c1) = _pair(p, hb, faces)
    for _ in range(4):
        c0.rk3_step(dt, fixed_dt=True)
    t, steps, dt_last = c1.rk3_run(4, dt=dt, fixed_dt=True)
    assert steps == 4 and dt_last == dt
    assert t == dt + dt + dt + dt
    _same(d0, d1, ["cv", "bv"])


def test_graph_recaptured_after_rebind(oracle_lib):
    """Binding a new block replaces the captured step; switching the dt mode does too."""
    p, hb, faces = helpers.curvilinear_air_case(16, 12, 10, scheme=abi.INV_HLLC, reconstruction=abi.REC_WENO5,
                                                viscous_order=0, bc="periodic", seed=6)
    oracle_lib.boundary(p, hb, faces)
    dt = 0.2 * oracle_lib.cfl_dt(p, hb)
    (d0, c0), (d1, c1) = _pair(p, hb, faces)
    c1.rk3_run(2, dt=dt, fixed_dt=True)
    fresh = DeviceBlock(hb)
    c1.bind(0, fresh.view(), faces)
    c1.rk3_run(3, dt=dt, fixed_dt=True)
    for _ in range(3):
        c0.rk3_step(dt, fixed_dt=True)
    _same(d0, fresh, ["cv"])
    c1.rk3_run(2)  # CFL mode on the same binding
    for _ in range(2):
        c0.rk3_step(0.0, fixed_dt=False)
    _same(d0, fresh, ["cv"])


def test_graph_positivity_limiter_reads_device_dt(oracle_lib):
    """The species positivity limiter takes the step's dt from the device inside the graph."""
    h2 = mechmod.load_json(os.path.join(GOLDEN, "h2_li2004.json"))
    case = cases.h2_air_box(h2, n_nodes=12, scheme=abi.INV_WENO5_CH, reconstruction=abi.REC_WENO5,
                            viscous_order=0, reaction=False)
    p, hb, faces = case.param, case.blocks[0], case.faces[0]
    rng = np.random.default_rng(3)
    sv = hb.a["sv"]
    ih, n2 = h2.index("H"), h2.index("N2")
    y = rng.uniform(0, 2e-3, sv[ih].shape)
    y[rng.uniform(size=y.shape) < 0.4] = 0.0
    sv[ih] = y
    sv[n2] = 1.0 - (sv.sum(axis=0) - sv[n2])
    oracle_lib.cv_from_bv(p, hb)
    oracle_lib.boundary(p, hb, faces)
    oracle_lib.properties(p, hb)
    p.positive_preserving = 1
    (d0, c0), (d1, c1) = _pair(p, hb, faces)
    for _ in range(2):
        c0.rk3_step(5e-9, fixed_dt=True)
    c1.rk3_run(2, dt=5e-9, fixed_dt=True)
    _same(d0, d1, ["cv", "bv", "sv"])
