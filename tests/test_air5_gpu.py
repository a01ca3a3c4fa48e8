"""Two-temperature AIR5 on the GPU against the FP64 oracle: the finite-rate chemistry with NASA9
multi-range thermo, Park's control temperatures and the e_ve source, and the stage update with
the two-temperature inversion and VT relaxation on NASA9 thermo.  Tolerance 1e-12 relative per
array component (the same FP64 formulas on both sides; pow/exp/log differ in the last bits
between the host and device libraries)."""
import os

import numpy as np
import pytest

import cb200
from cb200 import abi, cases, mech as mechmod
from cb200.field import DeviceBlock

import helpers
from test_two_temperature_cpu import two_temperature_residual

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL = 1e-12


@pytest.fixture(scope="module")
def air5():
    return mechmod.load_json(os.path.join(GOLD, "air5_park.json"))


@pytest.fixture(scope="module")
def tt():
    return mechmod.load_two_temperature_json(os.path.join(GOLD, "air5_park.json"))


def _sync():
    import torch
    torch.cuda.synchronize()


def _inner(a, g):
    return a[:, g:-g, g:-g, g:-g]


def _setup(oracle, air5, tt, n=10, **kw):
    case = cases.air5_box_2t(air5, tt, n_nodes=n, **kw)
    p, b, faces = case.param, case.blocks[0], case.faces[0]
    oracle.cv_from_bv(p, b)  # cv and e_ve from (bv, Y, T_ve)
    dev = DeviceBlock(b)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    return p, b, faces, dev, ctx


def test_chemistry_two_temperature_parity(oracle_lib, air5, tt):
    p, b, faces, dev, ctx = _setup(oracle_lib, air5, tt)
    ctx.rhs(0, abi.RHS_CHEMISTRY)
    _sync()
    oracle_lib.rhs(p, b, faces, abi.RHS_CHEMISTRY)
    out = dev.to_host(["dq", "reaction_timeScale"])
    assert helpers.rel_err(out["dq"], b.a["dq"]) < TOL
    assert helpers.rel_err(_inner(out["reaction_timeScale"], b.ngg), _inner(b.a["reaction_timeScale"], b.ngg)) < TOL
    # the reactions conserve mass node by node, and the e_ve row carries their energy
    ns = air5.ns
    rows = out["dq"][5:5 + ns]
    assert np.abs(rows.sum(axis=0)).max() <= 1e-12 * np.abs(rows).max()
    assert np.abs(out["dq"][5 + ns]).max() > 0


def test_cv_from_bv_nasa9_parity(oracle_lib, air5, tt):
    case = cases.air5_box_2t(air5, tt, n_nodes=8)
    p, b, faces = case.param, case.blocks[0], case.faces[0]
    dev = DeviceBlock(b)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    ctx.cv_from_bv(0)
    _sync()
    oracle_lib.cv_from_bv(p, b)
    out = dev.to_host(["cv", "sv", "temperature_ve"])
    for n in ("cv", "sv", "temperature_ve"):
        assert helpers.rel_err(out[n], b.a[n]) < 1e-13, n


def test_stage_update_nasa9_two_temperature_parity(oracle_lib, air5, tt):
    p, b, faces, dev, ctx = _setup(oracle_lib, air5, tt, n=8)
    dev.load(b, ["cv", "sv", "temperature_ve"])
    b.a["qn"][...] = b.a["cv"]
    b.a["dq"][...] = two_temperature_residual(b, 1e-8, np.random.default_rng(5))
    dev.load(b, ["qn", "dq"])
    for rk in range(3):
        ctx.stage_update(0, 1e-8, rk)
        oracle_lib.stage_update(p, b, 1e-8, rk)
    _sync()
    g = b.ngg
    out = dev.to_host(["cv", "bv", "sv", "temperature_ve"])
    for n in ("cv", "bv", "sv", "temperature_ve"):
        assert helpers.rel_err(_inner(out[n], g), _inner(b.a[n], g)) < 3 * TOL, n
    assert ctx.read_status() == 0


def _viscous_setup(oracle, air5, tt):
    p, b, faces, dev, ctx = _setup(oracle, air5, tt, n=10, viscous_order=2)
    return p, b, faces, dev, ctx


PROPS = ("gamma", "acoustic_speed", "mach", "mul", "thermal_conductivity", "rho_D", "thermal_conductivity_ve")


def test_properties_two_temperature_parity(oracle_lib, air5, tt):
    p, b, faces, dev, ctx = _viscous_setup(oracle_lib, air5, tt)
    ctx.properties(0)
    _sync()
    oracle_lib.properties(p, b)
    out = dev.to_host(list(PROPS))
    for n in PROPS:
        assert helpers.rel_err(out[n], b.a[n]) < TOL, n
    assert (b.a["thermal_conductivity_ve"] > 0).all()


def test_viscous_two_temperature_parity(oracle_lib, air5, tt):
    """2nd-order viscous fluxes with the e_ve conduction and flux and the T_ve diffusing enthalpy."""
    p, b, faces, dev, ctx = _viscous_setup(oracle_lib, air5, tt)
    oracle_lib.properties(p, b)
    dev.load(b, list(PROPS))
    ctx.rhs(0, abi.RHS_VISCOUS)
    _sync()
    oracle_lib.rhs(p, b, faces, abi.RHS_VISCOUS)
    out = dev.to_host(["dq"])
    assert helpers.rel_err(out["dq"], b.a["dq"]) < 1e-11
    assert np.abs(b.a["dq"][5 + air5.ns]).max() > 0


def test_cfl_two_temperature_parity(oracle_lib, air5, tt):
    p, b, faces, dev, ctx = _viscous_setup(oracle_lib, air5, tt)
    oracle_lib.properties(p, b)
    dev.load(b, list(PROPS))
    dt = ctx.cfl_dt()
    ref = oracle_lib.cfl_dt(p, b)
    assert abs(dt - ref) <= 1e-13 * ref


@pytest.mark.parametrize("scheme,ngg", [(abi.INV_WENO5_CH, 3), (abi.INV_WENO7_CH, 4)], ids=["weno5_ch", "weno7_ch"])
def test_inviscid_char_two_temperature_parity(oracle_lib, air5, tt, scheme, ngg):
    """Characteristic WENO with rho e_ve as a scalar row and the trans-rot Roe-state thermo."""
    p, b, faces, dev, ctx = _setup(oracle_lib, air5, tt, n=10, scheme=scheme, ngg=ngg)
    oracle_lib.properties(p, b)
    dev.load(b, ["gamma", "acoustic_speed", "mach", "mul", "thermal_conductivity", "rho_D"])
    ctx.rhs(0, abi.RHS_INVISCID)
    _sync()
    oracle_lib.rhs(p, b, faces, abi.RHS_INVISCID)
    out = dev.to_host(["dq"])
    assert helpers.rel_err(out["dq"], b.a["dq"]) < 1e-11
    assert np.abs(b.a["dq"][5 + air5.ns]).max() > 0


def test_rk3_step_two_temperature_parity(oracle_lib, air5, tt):
    """Whole SSP-RK3 steps of the two-temperature AIR5 box: WENO5-ch fluxes with the e_ve row,
    2nd-order viscous terms with the e_ve conduction, Park chemistry with the e_ve source, the
    stage update with the VT relaxation, periodic ghost fill and the two-temperature properties."""
    p, b, faces, dev, ctx = _setup(oracle_lib, air5, tt, n=8, viscous_order=2)
    oracle_lib.properties(p, b)
    dev.load(b, list(PROPS))
    dt = 2e-9
    for _ in range(2):
        ctx.rk3_step(dt, fixed_dt=True)
        oracle_lib.rk3_step(p, [b], [faces], dt, True)
    _sync()
    assert ctx.read_status() == 0
    g = b.ngg
    out = dev.to_host(["cv", "bv", "sv", "temperature_ve"])
    for n in ("cv", "bv", "sv", "temperature_ve"):
        assert helpers.rel_err(_inner(out[n], g), _inner(b.a[n], g)) < 1e-10, n


def test_rk3_step_two_temperature_outflow_parity(oracle_lib, air5, tt):
    """The same steps with outflow faces along x (zeroth-order extrapolation of bv and every scalar,
    the ghost T_ve starting its inversion from the face node's)."""
    case = cases.air5_box_2t(air5, tt, n_nodes=8, viscous_order=2)
    p, b, faces = case.param, case.blocks[0], case.faces[0]
    for f in faces:
        if f.face == 0:
            f.type = abi.BC_OUTFLOW
    oracle_lib.cv_from_bv(p, b)
    oracle_lib.properties(p, b)
    dev = DeviceBlock(b)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    for _ in range(2):
        ctx.rk3_step(2e-9, fixed_dt=True)
        oracle_lib.rk3_step(p, [b], [faces], 2e-9, True)
    _sync()
    assert ctx.read_status() == 0
    g = b.ngg
    out = dev.to_host(["cv", "bv", "sv", "temperature_ve"])
    for n in ("cv", "bv", "sv", "temperature_ve"):
        assert helpers.rel_err(_inner(out[n], g), _inner(b.a[n], g)) < 1e-10, n
