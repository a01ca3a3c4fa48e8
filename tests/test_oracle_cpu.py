"""CPU checks of the FP64 host oracle against the reference's known answers and against
properties the discretisation must have.  No GPU is used here."""
import math
import os

import numpy as np
import pytest

from cb200 import abi, cases

import helpers

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def run_sod(oracle, mx=1000, scheme=abi.INV_WENO5_CH, t_end=0.2):
    case = cases.sod(mx=mx, scheme=scheme)
    b, faces, p = case.blocks[0], case.faces[0], case.param
    oracle.boundary(p, b, faces)
    t = 0.0
    steps = 0
    # the reference stops when t >= t_end without clipping the last dt (src/RK.cuh:240-264)
    while t < t_end:
        dt = oracle.rk3_step(p, [b], [faces], 0.0, fixed_dt=False)
        t += dt
        steps += 1
    return b, t, steps


def test_sod_against_reference_exact_solution(oracle_lib):
    """Pins the WENO5-ch/SSP-RK3 path of the oracle to the reference's exact Sod data
    (example/sodShockTube/exact.dat, fixture tests/golden/sod_exact.txt)."""
    ex = np.loadtxt(os.path.join(GOLDEN, "sod_exact.txt"))
    b, t, steps = run_sod(oracle_lib)
    x = np.arange(1000) / 999.0
    rho = b.interior("bv", 0)[0, 0, :]
    pr = b.interior("bv", 4)[0, 0, :]
    u = b.interior("bv", 1)[0, 0, :]
    assert abs(t - 0.2) < 1e-3 and steps > 100
    rho_ex = np.interp(x, ex[:, 0], ex[:, 2])
    p_ex = np.interp(x, ex[:, 0], ex[:, 3])
    u_ex = np.interp(x, ex[:, 0], ex[:, 1])
    # L1 errors of a 5th-order shock-capturing scheme on 1000 nodes (first-order at the
    # discontinuities): about 7e-4 here
    assert np.mean(np.abs(rho - rho_ex)) < 1.5e-3
    assert np.mean(np.abs(pr - p_ex)) < 1.2e-3
    assert np.mean(np.abs(u - u_ex)) < 2.5e-3
    # shock position: the density step 0.2656 -> 0.125 is at x = 0.8504 in the exact data
    i_shock = np.argmax(rho < 0.5 * (0.2656 + 0.125))
    assert abs(x[i_shock] - 0.8504) < 3e-3


@pytest.mark.parametrize("scheme,rec", [(abi.INV_WENO7_CH, abi.REC_MUSCL), (abi.INV_AUSMP, abi.REC_MUSCL),
                                        (abi.INV_HLLC, abi.REC_WENO5), (abi.INV_ROE, abi.REC_MUSCL),
                                        (abi.INV_WENO5_CP, abi.REC_MUSCL), (abi.INV_WENO7_CP, abi.REC_MUSCL)])
def test_sod_other_schemes_converge(oracle_lib, scheme, rec):
    ex = np.loadtxt(os.path.join(GOLDEN, "sod_exact.txt"))
    case = cases.sod(mx=400, scheme=scheme, reconstruction=rec)
    b, faces, p = case.blocks[0], case.faces[0], case.param
    oracle_lib.boundary(p, b, faces)
    t = 0.0
    while t < 0.2:
        t += oracle_lib.rk3_step(p, [b], [faces], 0.0, fixed_dt=False)
    x = np.arange(400) / 399.0
    rho = b.interior("bv", 0)[0, 0, :]
    assert np.mean(np.abs(rho - np.interp(x, ex[:, 0], ex[:, 2]))) < 1.2e-2


def test_weno_smooth_advection_order(oracle_lib):
    """1-D periodic density wave advected by u=1: error drops at high order with N."""
    errs = []
    for n in (16, 32):
        m = n + 1
        case = cases.sod(mx=m)  # reuse the 1-D block layout, then overwrite the state
        b, p = case.blocks[0], case.param
        p.inviscid_scheme = abi.INV_WENO5_CH
        faces = [f for f in case.faces[0]]
        for f in faces:
            f.type = abi.BC_PERIODIC if f.face == 0 else abi.BC_OUTFLOW
        dx = 1.0 / n
        b.a["metric"][0] = 1.0 / dx
        b.a["jac"][0] = dx
        x = (np.arange(-3, m + 3)) * dx
        bv = b.a["bv"]
        bv[0] = (1 + 0.2 * np.sin(2 * math.pi * x))[None, None, :]
        bv[1] = 1.0
        bv[4] = 1.0
        bv[5] = bv[4] / (bv[0] * cases.R_AIR)
        cases.fill_cv_air(b)
        p.v_ref = 1.0
        oracle_lib.boundary(p, b, faces)
        t_end, dt = 0.25, 0.2 * dx
        nst = int(round(t_end / dt))
        for _ in range(nst):
            oracle_lib.rk3_step(p, [b], [faces], dt, fixed_dt=True)
        xi = np.arange(m) * dx
        exact = 1 + 0.2 * np.sin(2 * math.pi * (xi - nst * dt))
        errs.append(np.abs(b.interior("bv", 0)[0, 0, :] - exact).max())
    order = math.log2(errs[0] / errs[1])
    assert errs[1] < 1e-4
    assert order > 3.5


def test_stage_update_air_roundtrip(oracle_lib):
    """With dq = 0, stage 0 reproduces cv = qn and the primitive recovery inverts cv_from_bv."""
    p, b, faces = helpers.curvilinear_air_case(mx=10, my=9, mz=8)
    b.a["qn"][...] = b.a["cv"]
    bv0 = b.a["bv"].copy()
    oracle_lib.stage_update(p, b, 1e-3, 0)
    for c in (0, 1, 2, 3, 4):
        np.testing.assert_allclose(b.interior("bv", c), bv0[c][4:-4, 4:-4, 4:-4], rtol=1e-13, atol=1e-14)


def test_rhs_translation_invariance(oracle_lib):
    """A uniform state on a uniform periodic grid has zero residual for every scheme."""
    for scheme, rec in [(abi.INV_WENO5_CH, 2), (abi.INV_WENO7_CH, 2), (abi.INV_AUSMP, 7), (abi.INV_HLLC, 2),
                        (abi.INV_ROE, 3)]:
        p, b, faces = helpers.curvilinear_air_case(mx=12, my=10, mz=9, scheme=scheme, reconstruction=rec,
                                                   jump=False)
        b.a["metric"][...] = 0
        b.a["metric"][0] = b.a["metric"][4] = b.a["metric"][8] = 10.0
        b.a["jac"][0] = 1e-3
        b.a["bv"][0] = 1.3
        b.a["bv"][1:4] = 0.7
        b.a["bv"][4] = 2.0
        b.a["bv"][5] = 2.0 / (1.3 * cases.R_AIR)
        cases.fill_cv_air(b)
        oracle_lib.boundary(p, b, faces)
        oracle_lib.rhs(p, b, faces)
        assert np.abs(b.a["dq"]).max() < 1e-10, scheme
