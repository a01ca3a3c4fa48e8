"""Shock sensor (Ducros / Jameson / jump) and the hybrid linear/WENO weights on the GPU
against the oracle."""
import numpy as np
import pytest

import cb200
from cb200 import abi
from cb200.field import DeviceBlock

import helpers

pytestmark = pytest.mark.gpu


def _sync():
    import torch
    torch.cuda.synchronize()


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_shock_sensor_parity(oracle_lib, kind):
    p, hb, faces = helpers.curvilinear_air_case(20, 18, 16, sensor=(kind, 0.1, 1e-3), bc="outflow")
    oracle_lib.boundary(p, hb, faces)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    ctx.shock_sensor(0)
    oracle_lib.shock_sensor(p, hb)
    _sync()
    s = dev.to_host(["shock_sensor"])["shock_sensor"]
    assert helpers.rel_err(s, hb.a["shock_sensor"]) < 1e-13
    # the pressure-based sensors separate the density/pressure jump from the smooth field
    g = hb.ngg
    inner = hb.a["shock_sensor"][0, g:-g, g:-g, g:-g]
    if kind != 0:
        assert inner.max() > 0.1 and (inner < 0.1).mean() > 0.3


@pytest.mark.parametrize("scheme", [abi.INV_WENO5_CH, abi.INV_WENO7_CH])
def test_hybrid_weno_step_parity(oracle_lib, scheme):
    p, hb, faces = helpers.curvilinear_air_case(20, 18, 16, scheme=scheme, sensor=(1, 0.05, 0.0), seed=4)
    oracle_lib.boundary(p, hb, faces)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    dt = 0.2 * oracle_lib.cfl_dt(p, hb)
    for _ in range(2):
        ctx.rk3_step(dt, fixed_dt=True)
        oracle_lib.rk3_step(p, [hb], [faces], dt, fixed_dt=True)
    _sync()
    out = dev.to_host(["cv"])
    g = hb.ngg
    sl = (slice(None), slice(g, -g), slice(g, -g), slice(g, -g))
    assert helpers.rel_err(out["cv"][sl], hb.a["cv"][sl]) < 3e-12
