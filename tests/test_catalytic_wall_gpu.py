"""The fully catalytic isothermal wall (apply_wall with Wall::catalytic_type 1, src/BoundCond.cu:
3055-3389: the face node and its ghosts take the wall's mass fractions Wall::yk) against the FP64
oracle, through the C ABI: the ghost fill alone and three RK3 steps, on the 9-species H2/air box
and on the two-temperature AIR5 box (the wall's e_ve from yk at its T_ve), each with the wall on
the low x face, an outflow on the high one and periodic y and z faces.  The same boxes are pinned
to the reference's own kernels in tests/test_ref_kernels_gpu.py."""
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


def _setup(name):
    p, hb, faces, extra = refcases.build(refcases.case_by_name(name))
    return p, hb, faces, extra


@pytest.mark.parametrize("name", ["mix_catwall_weno5ch", "air5_catwall_weno5ch"], ids=["h2_air", "air5_2t"])
def test_catalytic_wall_ghost_fill(oracle_lib, name):
    p, hb, faces, extra = _setup(name)
    if "two_t" in extra:
        oracle_lib.cv_from_bv(p, hb)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    ctx.boundary(0)
    _sync()
    oracle_lib.boundary(p, hb, faces)
    out = dev.to_host(["bv", "sv", "cv"])
    for a in ("bv", "sv", "cv"):
        assert np.isfinite(out[a]).all()
        assert helpers.rel_err(out[a], hb.a[a]) < 1e-13, a
    # the wall's face nodes hold the wall's mass fractions
    t_wall, yw = refcases.CAT_WALL["air5" if "two_t" in extra else "mix"]
    m = extra["mech"]
    g = hb.ngg
    for name_, v in yw.items():
        assert np.allclose(out["sv"][m.index(name_), g:-g, g:-g, g], v, rtol=0, atol=1e-15)
    ctx.close()


@pytest.mark.parametrize("name", ["mix_catwall_weno5ch", "air5_catwall_weno5ch"], ids=["h2_air", "air5_2t"])
def test_catalytic_wall_rk3(oracle_lib, name):
    p, hb, faces, extra = _setup(name)
    if "two_t" in extra:
        oracle_lib.cv_from_bv(p, hb)
    oracle_lib.properties(p, hb)
    oracle_lib.boundary(p, hb, faces)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    for _ in range(3):
        ctx.rk3_step(p.dt, fixed_dt=True)
        oracle_lib.rk3_step(p, [hb], [faces], p.dt, fixed_dt=True)
    _sync()
    assert ctx.read_status() == 0
    out = dev.to_host(["cv", "bv"])
    g = hb.ngg
    sl = (slice(None), slice(g, -g), slice(g, -g), slice(g, -g))
    assert helpers.rel_err(out["cv"][sl], hb.a["cv"][sl]) < 3 * TOL
    assert helpers.rel_err(out["bv"][sl], hb.a["bv"][sl]) < 3 * TOL
    ctx.close()
