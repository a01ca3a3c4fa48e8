"""The blowing wall (Wall::if_blow_shock_wave, src/BoundCond.cu:3226-3245) against the FP64 oracle,
through the C ABI: on the channel's isothermal wall, the ghost fill and three RK3 steps inside the
blowing window (the wall moving along its inward normal) and the ghost fill after it (the wall at
rest again).  The same channel is pinned to the reference's own kernels in
tests/test_ref_kernels_gpu.py (chan_blow_weno5ch)."""
import numpy as np
import pytest

import cb200
from cb200.field import DeviceBlock

import helpers
import refcases

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _sync():
    import torch
    torch.cuda.synchronize()


@pytest.mark.parametrize("step", [1, 20], ids=["blowing", "after_window"])
def test_blowing_wall_ghost_fill(oracle_lib, step):
    p, hb, faces, extra = refcases.build(refcases.case_by_name("chan_blow_weno5ch"))
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    ctx.set_step(step)
    ctx.boundary(0)
    _sync()
    oracle_lib.set_step(step)
    oracle_lib.boundary(p, hb, faces)
    out = dev.to_host(["bv", "cv"])
    assert helpers.rel_err(out["bv"], hb.a["bv"]) < 1e-13
    assert helpers.rel_err(out["cv"], hb.a["cv"]) < 1e-13
    g = hb.ngg
    wall_v = out["bv"][1:3, g, g, g:-g]  # u, v of the wall's face nodes (j = 0)
    if step <= refcases.CHAN_BLOW["end"]:
        assert np.abs(wall_v).max() > 0
    else:
        assert np.abs(wall_v).max() == 0
    ctx.close()


def test_blowing_wall_rk3(oracle_lib):
    p, hb, faces, extra = refcases.build(refcases.case_by_name("chan_blow_weno5ch"))
    oracle_lib.set_step(0)
    oracle_lib.properties(p, hb)
    oracle_lib.boundary(p, hb, faces)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    ctx.set_step(0)
    dt = 0.2 * oracle_lib.cfl_dt(p, hb)
    for _ in range(3):  # steps 1, 2, 3: inside the window
        ctx.rk3_step(dt, fixed_dt=True)
        oracle_lib.rk3_step(p, [hb], [faces], dt, fixed_dt=True)
    _sync()
    assert ctx.read_status() == 0
    out = dev.to_host(["cv"])
    g = hb.ngg
    sl = (slice(None), slice(None), slice(g, -g), slice(g, -g))
    cv, ref = out["cv"][sl], hb.a["cv"][sl]
    scale = [max(np.abs(ref[c]).max(), 1e-300) for c in range(len(ref))]
    scale[1:4] = [max(scale[1:4])] * 3  # the z momentum of a 2-D channel is rounding noise
    assert max(np.abs(cv[c] - ref[c]).max() / scale[c] for c in range(len(ref))) < 3 * TOL
    ctx.close()
