"""GPU parity of the thermally perfect mixture path (9-species H2/air, reference tables)
against the FP64 oracle: properties/transport, stage update with the Newton temperature,
characteristic WENO with species rows, primitive-reconstruction Riemann solvers, 2nd-order
viscous fluxes with species diffusion, and the finite-rate chemistry source."""
import os

import numpy as np
import pytest

import cb200
from cb200 import abi, cases, mech as mechmod
from cb200.field import DeviceBlock

import helpers

pytestmark = pytest.mark.gpu
TOL = 1e-12
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def h2():
    return mechmod.load_json(os.path.join(GOLDEN, "h2_li2004.json"))


def _sync():
    import torch
    torch.cuda.synchronize()


def _box(oracle, h2, scheme=abi.INV_WENO5_CH, rec=abi.REC_WENO5, visc=2, reaction=True, n=14):
    case = cases.h2_air_box(h2, n_nodes=n, scheme=scheme, reconstruction=rec, viscous_order=visc,
                            reaction=reaction)
    p, hb, faces = case.param, case.blocks[0], case.faces[0]
    oracle.boundary(p, hb, faces)
    oracle.properties(p, hb)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    return p, hb, faces, dev, ctx


def test_properties_parity(oracle_lib, h2):
    p, hb, faces, dev, ctx = _box(oracle_lib, h2)
    for n in ("mul", "thermal_conductivity", "rho_D", "gamma", "acoustic_speed"):
        dev.t[n].zero_()
    ctx.properties(0)
    _sync()
    out = dev.to_host(["mul", "thermal_conductivity", "rho_D", "gamma", "acoustic_speed"])
    for n, v in out.items():
        assert helpers.rel_err(v, hb.a[n]) < 1e-13, n


def test_stage_update_newton_parity(oracle_lib, h2):
    p, hb, faces, dev, ctx = _box(oracle_lib, h2)
    rng = np.random.default_rng(3)
    hb.a["qn"][...] = hb.a["cv"]
    # residuals that change cv by about 1e-3 of its scale over dt/J
    jdt = float(hb.a["jac"].max()) / 2e-9
    hb.a["dq"][...] = 1e-3 * jdt * rng.standard_normal(hb.a["dq"].shape) * np.abs(
        hb.a["cv"][:, 3:-3, 3:-3, 3:-3]).max(axis=(1, 2, 3), keepdims=True)
    hb.a["bv"][5] *= 1.05  # Newton starts from a perturbed temperature
    dev.load(hb, ["qn", "dq", "bv"])
    for rk in range(3):
        ctx.stage_update(0, 2e-9, rk)
        oracle_lib.stage_update(p, hb, 2e-9, rk)
    _sync()
    out = dev.to_host(["cv", "bv", "sv"])
    assert helpers.rel_err(out["cv"], hb.a["cv"]) < 1e-14
    assert helpers.rel_err(out["bv"], hb.a["bv"]) < 1e-12
    assert helpers.rel_err(out["sv"], hb.a["sv"]) < 1e-14


MIX = [("weno5ch", abi.INV_WENO5_CH, abi.REC_WENO5, 0, False),
       ("weno7ch", abi.INV_WENO7_CH, abi.REC_WENO5, 0, False),
       ("hllc_weno5", abi.INV_HLLC, abi.REC_WENO5, 0, False),
       ("ausm_muscl", abi.INV_AUSMP, abi.REC_MUSCL, 0, False),
       ("roe_muscl", abi.INV_ROE, abi.REC_MUSCL, 0, False),
       ("visc2", abi.INV_HLLC, abi.REC_WENO5, 2, False),
       ("chem", abi.INV_HLLC, abi.REC_WENO5, 0, True),
       ("visc8", abi.INV_WENO7_CH, abi.REC_WENO5, 8, False)]


@pytest.mark.parametrize("name,scheme,rec,visc,chem", MIX, ids=[m[0] for m in MIX])
def test_rhs_parity_mixture(oracle_lib, h2, name, scheme, rec, visc, chem):
    n = 16 if scheme == abi.INV_WENO7_CH else 14
    case = cases.h2_air_box(h2, n_nodes=n, ngg=4 if scheme == abi.INV_WENO7_CH else 3, scheme=scheme,
                            reconstruction=rec, viscous_order=visc, reaction=chem)
    p, hb, faces = case.param, case.blocks[0], case.faces[0]
    oracle_lib.boundary(p, hb, faces)
    oracle_lib.properties(p, hb)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    mask = abi.RHS_ALL if not chem else abi.RHS_CHEMISTRY
    ctx.rhs(0, mask)
    oracle_lib.rhs(p, hb, faces, mask)
    _sync()
    dq = dev.to_host(["dq"])["dq"]
    err = helpers.rel_err(dq[:5] if not chem else dq[5:], hb.a["dq"][:5] if not chem else hb.a["dq"][5:])
    assert err < TOL, (name, err)
    # species rows: relative to the largest species residual
    err_s = helpers.rel_err(dq[5:].reshape(1, -1), hb.a["dq"][5:].reshape(1, -1))
    assert err_s < TOL, (name, err_s)
    if chem:
        rts = dev.to_host(["reaction_timeScale"])["reaction_timeScale"]
        g = hb.ngg
        sl = (slice(None), slice(g, -g), slice(g, -g), slice(g, -g))
        assert helpers.rel_err(rts[sl], hb.a["reaction_timeScale"][sl]) < 1e-12


def test_reacting_box_rk3_parity(oracle_lib, h2):
    """Reacting H2-air box in miniature: WENO5 + HLLC, 2nd-order viscous, chemistry, 3 RK3 steps at 2e-9 s."""
    p, hb, faces, dev, ctx = _box(oracle_lib, h2, scheme=abi.INV_HLLC, rec=abi.REC_WENO5, visc=2, reaction=True)
    for _ in range(3):
        ctx.rk3_step(2e-9, fixed_dt=True)
        oracle_lib.rk3_step(p, [hb], [faces], 2e-9, fixed_dt=True)
    _sync()
    out = dev.to_host(["cv", "bv"])
    g = hb.ngg
    sl = (slice(None), slice(g, -g), slice(g, -g), slice(g, -g))
    assert helpers.rel_err(out["cv"][sl], hb.a["cv"][sl]) < 3 * TOL
    assert helpers.rel_err(out["bv"][sl], hb.a["bv"][sl]) < 3 * TOL
    assert ctx.read_status() == 0


def test_positivity_limiter_parity(oracle_lib, h2):
    """Species positivity limiter of the characteristic WENO5 fluxes (positive_preserving): a
    radical with random values and exact zeros, and a step long enough that unlimited fluxes
    would empty cells, so the limiter blends many species fluxes with the first-order flux."""
    p, hb, faces, dev, ctx = _box(oracle_lib, h2, scheme=abi.INV_WENO5_CH, visc=0, reaction=False)
    ctx.close()
    rng = np.random.default_rng(11)
    sv = hb.a["sv"]
    ih, io, n2 = h2.index("H"), h2.index("OH"), h2.index("N2")
    for s in (ih, io):
        y = rng.uniform(0, 2e-3, sv[s].shape)
        y[rng.uniform(size=y.shape) < 0.4] = 0.0
        sv[s] = y
    sv[n2] = 1.0 - (sv.sum(axis=0) - sv[n2])
    oracle_lib.cv_from_bv(p, hb)
    oracle_lib.boundary(p, hb, faces)
    oracle_lib.properties(p, hb)
    p.dt = 4e-7
    p.positive_preserving = 0
    oracle_lib.rhs(p, hb, faces, mask=abi.RHS_INVISCID)
    unlimited = hb.a["dq"].copy()
    p.positive_preserving = 1
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    ctx.rhs(0, mask=abi.RHS_INVISCID)
    _sync()
    oracle_lib.rhs(p, hb, faces, mask=abi.RHS_INVISCID)
    dq = dev.to_host(["dq"])["dq"]
    # the limiter acted: species residuals moved, the flow rows did not
    assert np.abs(hb.a["dq"][5:] - unlimited[5:]).max() > 1e-3 * np.abs(unlimited[5:]).max()
    assert np.array_equal(hb.a["dq"][:5], unlimited[:5])
    assert helpers.rel_err(dq, hb.a["dq"]) < 1e-12
    ctx.close()
