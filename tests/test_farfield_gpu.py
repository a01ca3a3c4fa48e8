"""The farfield face and the back-pressure outflow (apply_farfield, src/BoundCond.cu:2351-2482;
the back-pressure branch of apply_outflow, :2219-2320) against the FP64 oracle, through the C ABI:
the ghost fill alone and three RK3 steps, on the channel (air: farfield on the inflow and the
far side, back pressure on the outflow, isothermal wall) at its subsonic interior velocity and at
four times it (supersonic: the other branches of both conditions), and on the 9-species H2/air
box with a farfield and a back-pressure face (the mixture gas constant, sound speed and scalars).
The same channel is pinned to the reference's own kernels in tests/test_ref_kernels_gpu.py."""
import numpy as np
import pytest

import cb200
from cb200 import abi, cases
from cb200.field import DeviceBlock, face

import helpers
import refcases

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _sync():
    import torch
    torch.cuda.synchronize()


def _channel(speed, visc):
    name = "chan_farfield_hllc_visc2" if visc else "chan_farfield_weno5ch"
    p, hb, faces, _ = refcases.build(refcases.case_by_name(name))
    for c in (1, 2):
        hb.a["bv"][c] *= speed
    cases.fill_cv_air(hb)
    return p, hb, faces


@pytest.mark.parametrize("speed", [1.0, 4.0], ids=["subsonic", "supersonic"])
def test_farfield_back_pressure_ghost_fill(oracle_lib, speed):
    p, hb, faces = _channel(speed, 0)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    ctx.boundary(0)
    _sync()
    oracle_lib.boundary(p, hb, faces)
    out = dev.to_host(["bv", "cv"])
    assert np.isfinite(out["bv"]).all()
    assert helpers.rel_err(out["bv"], hb.a["bv"]) < 1e-13
    assert helpers.rel_err(out["cv"], hb.a["cv"]) < 1e-13
    ctx.close()


@pytest.mark.parametrize("speed", [1.0, 4.0], ids=["subsonic", "supersonic"])
def test_farfield_back_pressure_rk3(oracle_lib, speed):
    p, hb, faces = _channel(speed, 2)
    oracle_lib.properties(p, hb)
    oracle_lib.boundary(p, hb, faces)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    dt = 0.2 * oracle_lib.cfl_dt(p, hb)
    for _ in range(3):
        ctx.rk3_step(dt, fixed_dt=True)
        oracle_lib.rk3_step(p, [hb], [faces], dt, fixed_dt=True)
    _sync()
    assert ctx.read_status() == 0
    out = dev.to_host(["cv"])
    g = hb.ngg
    sl = (slice(None), slice(None), slice(g, -g), slice(g, -g))
    assert helpers.rel_err(out["cv"][sl], hb.a["cv"][sl]) < 3 * TOL
    ctx.close()


def test_farfield_back_pressure_mixture_rk3(oracle_lib):
    """H2/air box: a farfield (the stoichiometric mixture at 1100 K, 1 atm, 5 m/s along +x) on the
    low x face, a back pressure of 1.02 atm on the high x face, periodic in y and z."""
    import os
    from cb200 import mech as mechmod
    m = mechmod.load_json(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "h2_li2004.json"))
    c = cases.h2_air_box(m, n_nodes=10, scheme=abi.INV_HLLC, reconstruction=abi.REC_MUSCL, viscous_order=2,
                         reaction=False)
    p, hb = c.param, c.blocks[0]
    mx, my, mz = hb.mx, hb.my, hb.mz
    y = mechmod.stoich_h2_air(m)
    mw = 1.0 / sum(y[i] / m.mw[i] for i in range(m.ns))
    T_ff, p_ff = 1100.0, 101325.0
    rho_ff = p_ff * mw / (cases.R_U * T_ff)
    faces = [face(abi.BC_FARFIELD, 0, -1, (0, 0, 0), (0, my - 1, mz - 1), sv=y, rho=rho_ff, u=5.0, v=0.0, w=0.0,
                  p=p_ff, T=T_ff),
             face(abi.BC_OUTFLOW, 0, 1, (mx - 1, 0, 0), (mx - 1, my - 1, mz - 1), p=1.02 * p_ff)]
    faces += [f for f in c.faces[0] if f.face != 0]
    oracle_lib.properties(p, hb)
    oracle_lib.boundary(p, hb, faces)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    for _ in range(3):
        ctx.rk3_step(2e-9, fixed_dt=True)
        oracle_lib.rk3_step(p, [hb], [faces], 2e-9, fixed_dt=True)
    _sync()
    assert ctx.read_status() == 0
    out = dev.to_host(["cv", "bv"])
    g = hb.ngg
    sl = (slice(None), slice(g, -g), slice(g, -g), slice(g, -g))
    assert helpers.rel_err(out["cv"][sl], hb.a["cv"][sl]) < 3 * TOL
    assert helpers.rel_err(out["bv"][sl], hb.a["bv"][sl]) < 3 * TOL
    ctx.close()
