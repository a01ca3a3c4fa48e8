"""Flowfield files (cb2_write_flowfield / cb2_read_flowfield) against the reference's own: the files
under tests/golden/plt/ are the reference's output/flowfield.plt, written by its FieldIO after the
runner's three stages of the case (tests/golden/make_ref_kernels.py; an air channel, the 9-species
H2/air box and the two-temperature AIR5 box).  The library reads them back into a block (the
restart), writes the same state again byte for byte, and round-trips its own files with ghost
layers.  tests/plt.py is an independent reader of the format."""
import json
import os

import numpy as np
import pytest

import cb200
from cb200.field import DeviceBlock

import plt
import refcases

HERE = os.path.dirname(os.path.abspath(__file__))
PLT_DIR = os.path.join(HERE, "golden", "plt")
FIXTURE = os.path.join(HERE, "golden", "ref_kernels.npz")
CASES = ["chan_nr_weno5ch", "mix_catwall_weno5ch", "air5_catwall_weno5ch"]


def _golden(name):
    path = os.path.join(PLT_DIR, name + ".plt")
    if not os.path.exists(path):
        pytest.skip("no reference flowfield file for " + name)
    return path


def _species(extra):
    m = extra.get("mech")
    return list(m.species) if m is not None else []


def _expected_names(extra):
    two_t = "two_t" in extra
    return (["x", "y", "z", "density", "u", "v", "w", "pressure", "temperature"] + _species(extra) +
            (["Eve"] if two_t else []) + ["mach"] + (["Tve"] if two_t else []))


@pytest.mark.parametrize("name", CASES)
def test_reference_flowfield_holds_the_reference_state(name):
    """The reference's file, read by tests/plt.py: its variables, zone and (min, max) pairs, and its
    density and temperature equal to the reference's dumped state (ref_kernels.npz) bit for bit."""
    path = _golden(name)
    p, hb, faces, extra = refcases.build(refcases.case_by_name(name))
    f = plt.read(path)
    assert f["title"] == "Solution file" and f["file_type"] == 0
    assert f["names"] == _expected_names(extra)
    (z,) = f["zones"]
    assert z["name"] == "zone 0" and z["dims"] == (hb.mx, hb.my, hb.mz)
    for (lo, hi), v in zip(z["minmax"], f["names"]):
        assert lo == z["data"][v].min() and hi == z["data"][v].max(), v
    ref = np.load(FIXTURE)
    assert np.array_equal(z["data"]["density"], ref[name + "/cv"][0])
    assert np.array_equal(z["data"]["temperature"], ref[name + "/T"])


def _padded(hb, interior):
    """A padded (ghost ngg) array with `interior` in its nodes."""
    g = hb.ngg
    a = np.zeros((hb.mz + 2 * g, hb.my + 2 * g, hb.mx + 2 * g))
    a[g:g + hb.mz, g:g + hb.my, g:g + hb.mx] = interior
    return a


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_restart_from_reference_file_and_write_it_again(name, tmp_path):
    import torch
    path = _golden(name)
    f = plt.read(path)
    (zf,) = f["zones"]
    p, hb, faces, extra = refcases.build(refcases.case_by_name(name))
    species = _species(extra)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    t = ctx.read_flowfield(path, species)
    torch.cuda.synchronize()
    assert t == zf["time"]
    g = hb.ngg
    inner = (slice(g, g + hb.mz), slice(g, g + hb.my), slice(g, g + hb.mx))
    out = dev.to_host(["bv"] + (["sv"] if "sv" in dev.t else []) +
                      (["temperature_ve"] if "temperature_ve" in dev.t else []))
    for c, v in enumerate(["density", "u", "v", "w", "pressure", "temperature"]):
        assert np.array_equal(out["bv"][c][inner], zf["data"][v]), v
    for s_, v in enumerate(species + (["Eve"] if "two_t" in extra else [])):
        assert np.array_equal(out["sv"][s_][inner], zf["data"][v]), v
    if "two_t" in extra:
        assert np.array_equal(out["temperature_ve"][0][inner], zf["data"]["Tve"])
    # the same state written again: mach as the reference had it, coordinates from its file
    dev.t["mach"][0][inner] = torch.from_numpy(zf["data"]["mach"]).cuda()
    xyz = [tuple(_padded(hb, zf["data"][c]) for c in ("x", "y", "z"))]
    mine = tmp_path / "flowfield.plt"
    ctx.write_flowfield(mine, xyz, species, ngg_out=0, solution_time=zf["time"])
    with open(path, "rb") as a, open(mine, "rb") as b:
        assert a.read() == b.read()
    ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["mix_catwall_weno5ch", "air5_catwall_weno5ch"])
def test_flowfield_round_trip_with_ghost_layers(name, tmp_path):
    """A block's state written with all its ghost layers and read into a second block, whose fields
    started at zero, comes back bit for bit, ghosts included."""
    import torch
    p, hb, faces, extra = refcases.build(refcases.case_by_name(name))
    species = _species(extra)
    rng = np.random.default_rng(5)
    hb.a["mach"][...] = rng.uniform(0.1, 3.0, hb.a["mach"].shape)
    dev = DeviceBlock(hb)
    ctx = cb200.Context(p)
    ctx.bind(0, dev.view(), faces)
    g = hb.ngg
    shp = hb.a["bv"].shape[1:]
    xyz = [tuple(rng.uniform(-1, 1, shp) for _ in range(3))]
    path = tmp_path / "flowfield.plt"
    ctx.write_flowfield(path, xyz, species, ngg_out=g, solution_time=1.25e-6)
    f = plt.read(path)
    assert f["zones"][0]["dims"] == (hb.mx + 2 * g, hb.my + 2 * g, hb.mz + 2 * g)
    assert np.array_equal(f["zones"][0]["data"]["x"], xyz[0][0])
    hb2 = type(hb)(hb.mx, hb.my, hb.mz, hb.ngg, hb.specs)
    for k in hb.a:
        hb2.a[k][...] = hb.a[k]
    for k in ("bv", "sv", "temperature_ve"):
        if k in hb2.a:
            hb2.a[k][...] = 0.0
    dev2 = DeviceBlock(hb2)
    ctx2 = cb200.Context(p)
    ctx2.bind(0, dev2.view(), faces)
    assert ctx2.read_flowfield(path, species) == 1.25e-6
    torch.cuda.synchronize()
    a, b = dev.to_host(), dev2.to_host()
    for k in ("bv", "sv", "temperature_ve"):
        if k in a:
            assert np.array_equal(a[k], b[k]), k
    ctx.close()
    ctx2.close()
