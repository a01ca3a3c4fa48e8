"""AIR5 two-temperature case: the oracle's NASA9 multi-range thermo and its (T, Tve) chemistry
with the AIR5 control-temperature model against the reference's own host code
(tests/golden/air5_park.json, written through oracle/_ref/dump_air5 by tests/golden/make_mech.py)."""
import json
import os

import numpy as np
import pytest

from cb200 import abi, cases, mech as mechmod

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")


@pytest.fixture(scope="module")
def gold():
    with open(os.path.join(GOLD, "air5_park.json")) as f:
        return json.load(f)


@pytest.fixture(scope="module")
def air5():
    return mechmod.load_json(os.path.join(GOLD, "air5_park.json"))


@pytest.fixture(scope="module")
def tt():
    return mechmod.load_two_temperature_json(os.path.join(GOLD, "air5_park.json"))


def _param(m, tt):
    return cases.make_param(n_var=6 + m.ns, n_spec=m.ns, mech=m.ptr(), two_t=tt.ptr(),
                            inviscid_scheme=abi.INV_WENO5_CH, reconstruction=abi.REC_WENO5)


def _close(a, b, rtol, atol=0.0):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return np.all(np.abs(a - b) <= rtol * np.abs(b) + atol)


def test_fixture_is_the_air5_park_case(gold, air5):
    assert gold["species"] == ["N2", "O2", "NO", "N", "O"]
    assert gold["n_reac"] == 17 and gold["nasa_7_or_9"] == 9
    assert air5.struct.therm_nasa_7_9 == 9 and air5.struct.two_temperature_reaction_temperature == 1
    # dissociation reactions run forward at sqrt(T Tve); the two exchange reactions at T
    assert gold["tcf_a"][:15] == [0.5] * 15 and gold["tcf_b"][:15] == [0.5] * 15
    assert gold["tcf_a"][15:] == [1, 1] and gold["tcf_b"][15:] == [0, 0]


def test_nasa9_thermo_matches_reference(oracle_lib, gold, air5):
    ns = air5.ns
    h_ref = np.asarray(gold["ladder_h"]).reshape(-1, ns)
    cp_ref = np.asarray(gold["ladder_cp"]).reshape(-1, ns)
    g_ref = np.asarray(gold["ladder_gibbs_rt"]).reshape(-1, ns)
    for a, t in enumerate(gold["ladder_T"]):
        h, cp = oracle_lib.nasa7_h_cp(air5, t)
        g = oracle_lib.gibbs_rt(air5, t)
        # h crosses zero for some species: scale the absolute part by the largest |h|
        assert _close(h, h_ref[a], 1e-13, 1e-13 * np.abs(h_ref[a]).max()), (t, h, h_ref[a])
        assert _close(cp, cp_ref[a], 1e-13), (t, cp, cp_ref[a])
        assert _close(g, g_ref[a], 1e-12, 1e-12 * np.abs(g_ref[a]).max()), (t, g, g_ref[a])


def test_species_ve_matches_reference(oracle_lib, gold, air5, tt):
    p = _param(air5, tt)
    ns = air5.ns
    e_ref = np.asarray(gold["ladder_e_ve"]).reshape(-1, ns)
    c_ref = np.asarray(gold["ladder_cv_ve"]).reshape(-1, ns)
    for a, t in enumerate(gold["ladder_T"]):
        e, c = oracle_lib.species_ve(p, t)
        assert _close(e, e_ref[a], 1e-14, 1e-300), (t, e, e_ref[a])
        assert _close(c, c_ref[a], 1e-13, 1e-300), (t, c, c_ref[a])


def test_two_temperature_chemistry_matches_reference(oracle_lib, gold, air5, tt):
    p = _param(air5, tt)
    active = 0
    for s in gold["states"]:
        om, od = oracle_lib.chemistry_source_2t(air5, s["rho"], s["T"], s["Tve"], s["Y"])
        ref, ref_d = np.asarray(s["omega"]), np.asarray(s["omega_d"])
        scale = np.abs(ref_d).max() + 1e-300
        assert _close(om, ref, 1e-11, 1e-12 * scale), (s["T"], s["Tve"], om, ref)
        assert _close(od, ref_d, 1e-11, 1e-12 * scale)
        # e_ve chemical source: sum_l omega_l e_ve,l(Tve)
        e, _ = oracle_lib.species_ve(p, s["Tve"])
        src = float(np.dot(om, e))
        assert abs(src - s["eve_source"]) <= 1e-10 * (np.abs(om * e).sum() + 1e-300), (src, s["eve_source"])
        active += scale > 1e-6
    assert active >= 20


def test_control_temperature_changes_the_rates(oracle_lib, gold, air5):
    """The dissociation rates of a cold-vibration state follow sqrt(T Tve), not T."""
    s = gold["states"][0]
    hot, _ = oracle_lib.chemistry_source_2t(air5, s["rho"], s["T"], s["T"], s["Y"])
    cold, _ = oracle_lib.chemistry_source_2t(air5, s["rho"], s["T"], 300.0, s["Y"])
    assert not np.allclose(hot, cold)


def test_air5_box_oracle_chemistry_rows(oracle_lib, air5, tt):
    """The block chemistry of the AIR5 box: each node's species rows are J omega(T, max(Tve, 1)) and
    its e_ve row J sum_s omega_s e_ve,s(Tve); three stages of an update keep the state finite."""
    case = cases.air5_box_2t(air5, tt, n_nodes=6)
    p, b, faces = case.param, case.blocks[0], case.faces[0]
    oracle_lib.cv_from_bv(p, b)
    ns = air5.ns
    g = b.ngg
    assert (b.a["sv"][ns][g:-g, g:-g, g:-g] > 0).all()
    oracle_lib.rhs(p, b, faces, abi.RHS_CHEMISTRY)
    for (i, j, k) in ((0, 0, 0), (3, 2, 1), (5, 5, 5)):
        bv = b.a["bv"][:, k + g, j + g, i + g]
        y = b.a["sv"][:ns, k + g, j + g, i + g]
        tve = b.a["temperature_ve"][0, k + g, j + g, i + g]
        jac = b.a["jac"][0, k + g, j + g, i + g]
        om, _ = oracle_lib.chemistry_source_2t(air5, bv[0], bv[5], max(tve, 1.0), y)
        e, _ = oracle_lib.species_ve(p, tve)
        dq = b.a["dq"][:, k, j, i]
        assert _close(dq[5:5 + ns], jac * om, 1e-14, 1e-14 * np.abs(jac * om).max())
        assert abs(dq[5 + ns] - jac * np.dot(om, e)) <= 1e-12 * jac * np.abs(om * e).sum()
    b.a["qn"][...] = b.a["cv"]
    for rk in range(3):
        oracle_lib.stage_update(p, b, 1e-9, rk)
    assert np.isfinite(b.a["bv"][:, g:-g, g:-g, g:-g]).all()
    assert (b.a["temperature_ve"][0][g:-g, g:-g, g:-g] > 0).all()


def test_air5_box_oracle_viscous_two_temperature(oracle_lib, air5, tt):
    """Properties (gamma of the trans-rot mode, kappa_ve = kappa cv_ve / cp) and the 2nd-order
    viscous residual with the e_ve rows on the AIR5 box: finite, and the e_ve conduction acts."""
    case = cases.air5_box_2t(air5, tt, n_nodes=6, viscous_order=2)
    p, b, faces = case.param, case.blocks[0], case.faces[0]
    oracle_lib.cv_from_bv(p, b)
    oracle_lib.properties(p, b)
    g = b.ngg
    inner = (slice(None), slice(g, -g), slice(g, -g), slice(g, -g))
    kve, kap = b.a["thermal_conductivity_ve"][inner], b.a["thermal_conductivity"][inner]
    assert (kve > 0).all() and (kve < kap).all()
    # the trans-rot gamma of partly dissociated air: near 1.4 (diatomic; the NASA9 cp is not
    # exactly the harmonic-oscillator split) and below 5/3 (atoms)
    gam = b.a["gamma"][inner]
    assert (gam > 1.35).all() and (gam < 1.67).all()
    oracle_lib.rhs(p, b, faces, abi.RHS_VISCOUS)
    assert np.isfinite(b.a["dq"]).all()
    assert np.abs(b.a["dq"][5 + air5.ns]).max() > 0
    dt = oracle_lib.cfl_dt(p, b)
    assert 0 < dt < 1e-3


def test_air5_box_oracle_step_two_temperature(oracle_lib, air5, tt):
    """A whole oracle step of the AIR5 box with every two-temperature term: finite and T_ve moves
    towards T (the VT relaxation and the e_ve conduction act)."""
    case = cases.air5_box_2t(air5, tt, n_nodes=6, viscous_order=2)
    p, b, faces = case.param, case.blocks[0], case.faces[0]
    oracle_lib.cv_from_bv(p, b)
    oracle_lib.properties(p, b)
    g = b.ngg
    inner = (0, slice(g, -g), slice(g, -g), slice(g, -g))
    gap0 = (b.a["bv"][5] - b.a["temperature_ve"][0])[inner[1:]]
    for _ in range(3):
        oracle_lib.rk3_step(p, [b], [faces], 2e-9, True)
    assert np.isfinite(b.a["cv"]).all()
    gap = (b.a["bv"][5] - b.a["temperature_ve"][0])[inner[1:]]
    assert np.abs(gap).mean() < np.abs(gap0).mean()
