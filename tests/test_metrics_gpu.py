"""cb2_metrics (the metrics and Jacobian of a block on the device) against the host computation of
cb200/grid.py, which tests/test_grid_cpu.py pins to the reference's own Mesh (1e-13): the four
body-fitted blocks of the square-cylinder grid (2-D, ghost coordinates from the inner faces and
the physical boundaries) and a perturbed curvilinear 3-D grid."""
import numpy as np
import pytest
import torch

from cb200 import cases, grid, lib
from cb200.lib import CB2Error

pytestmark = pytest.mark.gpu
TOL = 1e-13


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _check(padded, g1, ngg, mx, my, mz):
    X, Y, Z = padded
    m_ref, j_ref = grid.metrics(padded, g1, ngg)
    metric = torch.zeros((9,) + j_ref.shape, dtype=torch.float64, device="cuda")
    jac = torch.zeros(j_ref.shape, dtype=torch.float64, device="cuda")
    lib.metrics(_dev(X), _dev(Y), _dev(Z), mx, my, mz, g1, ngg, metric, jac)
    torch.cuda.synchronize()
    m, j = metric.cpu().numpy(), jac.cpu().numpy()
    assert np.abs(j - j_ref).max() <= TOL * np.abs(j_ref).max()
    for c in range(9):
        scale = max(np.abs(m_ref).max(), 1e-300)
        assert np.abs(m[c] - m_ref[c]).max() <= TOL * scale, c


def test_device_metrics_square_cylinder_blocks():
    ngg = 3
    g = grid.square_cylinder(24, 16, first=2e-4, half_box=0.03)
    inner = [[grid.register_inner_face(a, b, 2, ngg) for a, b in faces] for faces in g["inner"]]
    padded, g1 = grid.extend_coordinates(g["xyz"], inner, ngg)
    for b in range(4):
        _check(padded[b], g1, ngg, 24, 16, 1)


def test_device_metrics_curvilinear_3d():
    n, ngg = 20, 4
    (X, Y, Z), _, _ = cases.sine_wave_metrics(n, ngg + 1, 0.05)
    _check((X, Y, Z), ngg + 1, ngg, n + 1, n + 1, n + 1)


def test_non_positive_jacobian_is_reported():
    """A left-handed block (x mirrored) has J < 0 everywhere: the call reports it."""
    n, ngg = 8, 2
    (X, Y, Z), _, _ = cases.sine_wave_metrics(n, ngg + 1, 0.0)
    m = n + 1
    metric = torch.zeros((9, m + 2 * ngg, m + 2 * ngg, m + 2 * ngg), dtype=torch.float64, device="cuda")
    jac = torch.zeros(metric.shape[1:], dtype=torch.float64, device="cuda")
    with pytest.raises(CB2Error):
        lib.metrics(_dev(-X), _dev(Y), _dev(Z), m, m, m, ngg + 1, ngg, metric, jac)
