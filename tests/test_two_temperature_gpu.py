"""Two-temperature stage operations on the GPU against the FP64 oracle: the conservative fill
with the e_ve / T_ve sync, the stage update with the two-temperature inversion and the VT
relaxation, and the standalone VT step.  Tolerance 1e-12 relative per array, as for the
one-temperature stage update (the same Newton iterations on both sides)."""
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
def h2():
    return mechmod.load_json(os.path.join(GOLD, "h2_li2004.json"))


@pytest.fixture(scope="module")
def tt():
    return mechmod.load_two_temperature_json(os.path.join(GOLD, "h2_two_temperature.json"))


def _sync():
    import torch
    torch.cuda.synchronize()


def _inner(a, g):
    return a[:, g:-g, g:-g, g:-g]


def _setup(oracle, h2, tt, n=8, relaxed_start=True):
    case = cases.h2_air_box_2t(h2, tt, n_nodes=n)
    p, b, faces = case.param, case.blocks[0], case.faces[0]
    if relaxed_start:
        oracle.cv_from_bv(p, b)
    dev = DeviceBlock(b)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    return p, b, faces, dev, ctx


def test_cv_from_bv_two_temperature_parity(oracle_lib, h2, tt):
    p, b, faces, dev, ctx = _setup(oracle_lib, h2, tt, relaxed_start=False)
    ctx.cv_from_bv(0)
    _sync()
    oracle_lib.cv_from_bv(p, b)
    out = dev.to_host(["cv", "sv", "temperature_ve"])
    for n in ("cv", "sv", "temperature_ve"):
        assert helpers.rel_err(out[n], b.a[n]) < 1e-13, n
    assert (b.a["sv"][h2.ns] > 0).all()


def test_stage_update_two_temperature_parity(oracle_lib, h2, tt):
    p, b, faces, dev, ctx = _setup(oracle_lib, h2, tt)
    dev.load(b, ["cv", "sv", "temperature_ve"])
    b.a["qn"][...] = b.a["cv"]
    b.a["dq"][...] = two_temperature_residual(b, 1e-8, np.random.default_rng(11))
    dev.load(b, ["qn", "dq"])
    for rk in range(3):
        ctx.stage_update(0, 1e-8, rk)
        oracle_lib.stage_update(p, b, 1e-8, rk)
    _sync()
    g = b.ngg
    out = dev.to_host(["cv", "bv", "sv", "temperature_ve"])
    for n in ("cv", "bv", "sv", "temperature_ve"):
        assert helpers.rel_err(_inner(out[n], g), _inner(b.a[n], g)) < 3 * TOL, n
    # the step moved T_ve: the relaxation acted
    assert ctx.read_status() == 0


def test_vt_relaxation_parity(oracle_lib, h2, tt):
    p, b, faces, dev, ctx = _setup(oracle_lib, h2, tt)
    dev.load(b, ["cv", "sv", "temperature_ve"])
    before = b.a["temperature_ve"].copy()
    for dt_stage in (2e-8, 5e-7):
        ctx.vt_relaxation(0, dt_stage)
        oracle_lib.vt_relaxation(p, b, dt_stage)
    _sync()
    g = b.ngg
    out = dev.to_host(["cv", "bv", "sv", "temperature_ve"])
    for n in ("cv", "bv", "sv", "temperature_ve"):
        assert helpers.rel_err(_inner(out[n], g), _inner(b.a[n], g)) < TOL, n
    assert np.abs(_inner(b.a["temperature_ve"], g) - _inner(before, g)).max() > 1.0


def test_two_temperature_box_hllc_residual_and_roe_refused(oracle_lib, h2, tt):
    """The H2/air box's two-temperature residual with its WENO5 + HLLC primitive-variable flux
    (e_ve carried as a scalar, the translational-rotational energy and gamma of the states) matches
    the oracle; the Roe flux, which the reference's two-temperature build does not have, is
    refused."""
    p, b, faces, dev, ctx = _setup(oracle_lib, h2, tt)
    oracle_lib.properties(p, b)
    dev.load(b)
    ctx.rhs(0, abi.RHS_INVISCID)
    _sync()
    dq = dev.to_host(["dq"])["dq"]
    oracle_lib.rhs(p, b, faces, abi.RHS_INVISCID)
    assert helpers.rel_err(dq, b.a["dq"]) < TOL
    ctx.close()
    p.inviscid_scheme = abi.INV_ROE
    with pytest.raises(cb200.CB2Error) as e:
        cb200.Context(p)
    assert e.value.code == abi.ERR_UNSUPPORTED
