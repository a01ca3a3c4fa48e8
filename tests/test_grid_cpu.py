"""The host grid module (cb200.grid) against the reference's own grid stage: the metrics and
Jacobian that the reference's Mesh computed for the four-block square cylinder of the fixture
tests/golden/ref_kernels.npz (dumped by the reference-kernel runner before it loads the case's
own), and the inner-face registration that the reference's exchange then used."""
import json
import os

import numpy as np
import pytest

from cb200 import grid

import refcases

FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_kernels.npz")


def test_square_cylinder_metrics_match_reference_mesh():
    if not os.path.exists(FIXTURE):
        pytest.skip("fixture not generated")
    z = np.load(FIXTURE)
    meta = json.loads(bytes(z["meta"]).decode())
    name = "c5_air5_cylinder_4blocks"
    if name + "/ref_metric" not in z:
        pytest.skip("no reference metrics in the fixture")
    p, blocks, faces, inner, extra = refcases.build_multi(meta[name]["case"])
    c = extra["case"]
    ref = z[name + "/ref_metric"]
    off = 0
    for b, hb in enumerate(blocks):
        npad = hb.a["jac"][0].size
        rm = ref[off:off + 9 * npad].reshape(hb.a["metric"].shape)
        rj = ref[off + 9 * npad:off + 10 * npad].reshape(hb.a["jac"][0].shape)
        off += 10 * npad
        m, j = grid.metrics(c.meta["padded"][b], c.meta["g1"], hb.ngg)
        scale = np.abs(rm).max()
        assert np.abs(m - rm).max() <= 1e-13 * scale, b
        assert np.abs(j - rj).max() <= 1e-13 * np.abs(rj).max(), b
    assert off == ref.size


def test_inner_face_registration_maps_coincident_nodes():
    """Every registered inner face of the cylinder maps its face layer onto nodes with the same
    coordinates in the neighbour block, and its ghosts onto the neighbour's interior."""
    c = refcases.build_multi(refcases.case_by_name("c5_air5_cylinder_4blocks"))[4]["case"]
    xyz = c.meta["grid"]["xyz"]
    for b, faces in enumerate(c.meta["inner"]):
        for f in faces:
            t = f.target_block
            for n1 in range(f.n_point[1]):
                for n0 in range(f.n_point[0]):
                    n = (n0, n1, 0)
                    d = [f.loop_dir[a] * n[a] for a in range(3)]
                    idx = [f.range_start[a] + d[a] for a in range(3)]
                    it = [f.target_start[a] + f.target_loop_dir[a] * d[f.src_tar[a]] for a in range(3)]
                    layer = f.range_start[f.face] if f.direction > 0 else f.range_end[f.face]
                    assert 0 <= it[0] < xyz[t][0].shape[2] and 0 <= it[1] < xyz[t][0].shape[1]
                    if idx[f.face] == layer:
                        for a in range(2):
                            assert xyz[b][a][0, idx[1], idx[0]] == xyz[t][a][0, it[1], it[0]]
