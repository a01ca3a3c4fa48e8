"""Synthetic inputs of the benchmark configurations (seeded, no external data).

Each builder returns a `Case`: the scalar settings (ParamView), one HostBlock per grid block
with initial bv/sv/cv and metrics, and the face boundary conditions.  Metrics are the exact
derivatives of the analytic grid map (computational coordinates = node indices), so they
are periodic-consistent; the library consumes metric/jac as given, as the reference's hot
path does.
"""
import math
from dataclasses import dataclass, field as dfield

import numpy as np

from . import abi
from .field import HostBlock, array_specs, box_faces

R_U = 8314.462618
MW_AIR = 28.9647
R_AIR = R_U / MW_AIR
GAMMA_AIR = 1.4


@dataclass
class Case:
    name: str
    param: abi.ParamView
    blocks: list
    faces: list  # list (per block) of lists of FaceBC
    meta: dict = dfield(default_factory=dict)

    @property
    def n_nodes(self):
        return sum(b.mx * b.my * b.mz for b in self.blocks)


def make_param(n_var=5, n_spec=0, dim=3, inviscid_scheme=abi.INV_WENO5_CH, reconstruction=abi.REC_MUSCL,
               viscous_order=0, Pr=0.72, cfl=0.5, rho_ref=1.0, v_ref=1.0, mu_constant=0.0,
               entropy_fix_factor=0.125, mech=None, precision=abi.PREC_FP64):
    p = abi.ParamView()
    p.abi_version = abi.ABI_VERSION
    p.dim = dim
    p.n_var = n_var
    p.n_spec = n_spec
    p.n_scalar = n_spec
    p.n_scalar_transported = n_spec
    p.inviscid_scheme = inviscid_scheme
    p.reconstruction = reconstruction
    p.limiter = 0
    p.viscous_order = viscous_order
    p.positive_preserving = 0
    p.gradP_in_diffusion_flux = 0
    p.reaction = 0
    p.shock_sensor = 0
    p.sensor_eps = 0.0
    p.sensor_threshold = 0.0
    p.entropy_fix_factor = entropy_fix_factor
    p.Pr = Pr
    p.cfl = cfl
    p.rho_ref = rho_ref
    p.v_ref = v_ref
    p.mu_constant = mu_constant
    p.precision = precision
    p.mech = mech
    return p


def fill_cv_air(b: HostBlock):
    """cv from bv for air over the whole padded block (compute_cv_from_bv<Air>)."""
    bv, cv = b.a["bv"], b.a["cv"]
    rho = bv[0]
    cv[0] = rho
    cv[1] = rho * bv[1]
    cv[2] = rho * bv[2]
    cv[3] = rho * bv[3]
    cv[4] = 0.5 * (bv[1] ** 2 + bv[2] ** 2 + bv[3] ** 2) * rho + bv[4] / (GAMMA_AIR - 1)


def _node_coords(n, g):
    return np.arange(-g, n + g, dtype=np.float64)


def sod(mx=1000, my=1, ngg=3, scheme=abi.INV_WENO5_CH, reconstruction=abi.REC_MUSCL, cfl=0.5):
    """Sod shock tube: x in [0,1] on mx nodes (x_i = i/(mx-1)), (rho,u,p) = (1,0,1) for
    x <= 0.5 and (0.125,0,0.1) beyond, outflow on every face, calorically perfect air."""
    mz = 1
    specs = array_specs(mx, my, mz, ngg, 5, 0, roe=(scheme == abi.INV_ROE))
    b = HostBlock(mx, my, mz, ngg, specs)
    dx = 1.0 / (mx - 1)
    x = _node_coords(mx, ngg) * dx
    left = x <= 0.5
    rho = np.where(left, 1.0, 0.125)
    pr = np.where(left, 1.0, 0.1)
    bv = b.a["bv"]
    bv[0] = rho[None, None, :]
    bv[4] = pr[None, None, :]
    bv[5] = bv[4] / (bv[0] * R_AIR)
    m = b.a["metric"]
    m[0] = 1.0 / dx
    m[4] = 1.0
    m[8] = 1.0
    b.a["jac"][0] = dx
    fill_cv_air(b)
    faces = box_faces(mx, my, mz, {(0, -1): abi.BC_OUTFLOW, (0, 1): abi.BC_OUTFLOW,
                                   (1, -1): abi.BC_OUTFLOW, (1, 1): abi.BC_OUTFLOW})
    c = math.sqrt(GAMMA_AIR * 1.0 / 1.0)
    p = make_param(dim=2, inviscid_scheme=scheme, reconstruction=reconstruction, cfl=cfl,
                   rho_ref=1.0, v_ref=c)  # |u| < 1 -> v_inf = c (src/BoundCond.cpp:335-340)
    return Case("sod", p, [b], [faces], {"t_end": 0.2, "dx": dx})


def sine_wave_metrics(n, ngg, amp=0.05):
    """Analytic map x = xi + a sin(2 pi eta) sin(2 pi zeta) (cyclic in y, z) on the unit cube
    with n intervals; returns (coords[3], metric[9], jac) on the padded node lattice."""
    s = 1.0 / n
    q = _node_coords(n + 1, ngg) * s  # xi, eta, zeta of each node
    Z, Y, X = np.meshgrid(q, q, q, indexing="ij")  # arrays indexed [k, j, i]
    tp = 2 * math.pi
    a = amp
    sx, cx = np.sin(tp * X), np.cos(tp * X)
    sy, cy = np.sin(tp * Y), np.cos(tp * Y)
    sz, cz = np.sin(tp * Z), np.cos(tp * Z)
    x = X + a * sy * sz
    y = Y + a * sz * sx
    z = Z + a * sx * sy
    # d(x,y,z)/d(i,j,k) = s * d(x,y,z)/d(xi,eta,zeta)
    J = np.empty((3, 3) + X.shape)
    J[0, 0] = 1.0
    J[0, 1] = a * tp * cy * sz
    J[0, 2] = a * tp * sy * cz
    J[1, 0] = a * tp * sz * cx
    J[1, 1] = 1.0
    J[1, 2] = a * tp * cz * sx
    J[2, 0] = a * tp * cx * sy
    J[2, 1] = a * tp * sx * cy
    J[2, 2] = 1.0
    J *= s
    Jm = np.moveaxis(J, (0, 1), (-2, -1))
    inv = np.linalg.inv(Jm)  # [..., a, b] = d(i,j,k)_a / d(x,y,z)_b
    det = np.linalg.det(Jm)
    metric = np.empty((9,) + X.shape)
    for r in range(3):
        for c in range(3):
            metric[3 * r + c] = inv[..., r, c]
    return (x, y, z), metric, det


def sine_wave(n=256, ngg=4, amp=0.05, mu=1e-4, scheme=abi.INV_AUSMP, reconstruction=abi.REC_WENO7,
              viscous_order=8):
    """3-D sine-wave advection on the perturbed periodic curvilinear grid of (n+1)^3 nodes:
    rho = 1 + 0.2 sin(2 pi (x+y+z)), u = v = w = 1, p = 1, constant mu, Pr = 0.72."""
    m = n + 1
    specs = array_specs(m, m, m, ngg, 5, 0, viscous_order=viscous_order, roe=(scheme == abi.INV_ROE))
    b = HostBlock(m, m, m, ngg, specs)
    (x, y, z), metric, det = sine_wave_metrics(n, ngg, amp)
    b.a["metric"][...] = metric
    b.a["jac"][0] = det
    bv = b.a["bv"]
    bv[0] = 1.0 + 0.2 * np.sin(2 * math.pi * (x + y + z))
    bv[1] = 1.0
    bv[2] = 1.0
    bv[3] = 1.0
    bv[4] = 1.0
    bv[5] = bv[4] / (bv[0] * R_AIR)
    b.a["mul"][0] = mu
    fill_cv_air(b)
    faces = box_faces(m, m, m, {(d, s): abi.BC_PERIODIC for d in range(3) for s in (-1, 1)})
    p = make_param(dim=3, inviscid_scheme=scheme, reconstruction=reconstruction, viscous_order=viscous_order,
                   cfl=0.5, rho_ref=1.0, v_ref=math.sqrt(3.0), mu_constant=mu)
    return Case("sine_wave", p, [b], [faces], {"n": n, "amp": amp})
