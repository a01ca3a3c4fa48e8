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
from . import mech as mechmod
from .field import HostBlock, array_specs, box_faces
from .mech import stoich_h2_air

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
               entropy_fix_factor=0.125, mech=None, precision=abi.PREC_FP64, two_t=None):
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
    p.limit_flow = 0
    p.p_ref = 0.0
    p.c_ref = 0.0
    p.dt = 0.0
    if two_t is not None:
        # e_ve is the scalar after the species (i_eve = n_spec, src/Parameter.cpp:647-656)
        p.two_t = two_t
        p.n_scalar = n_spec + 1
        p.n_scalar_transported = n_spec + 1
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
    # x + y + z of every node: the exact solution is rho = 1 + 0.2 sin(2 pi (x + y + z - 3 t))
    return Case("sine_wave", p, [b], [faces], {"n": n, "amp": amp, "xyz_sum": x + y + z})


# ---- thermally perfect mixtures ------------------------------------------------------------
def nasa7_h(mech, t):
    """h_k(T) [J/kg] on an array of temperatures (NASA7 two-range, linear extension outside)."""
    d = mech.d
    ns = mech.ns
    lo = np.asarray(d["low_temp_coeff"]).reshape(ns, 7)
    hi = np.asarray(d["high_temp_coeff"]).reshape(ns, 7)
    tl, tm, th = (np.asarray(d[k]) for k in ("t_low", "t_mid", "t_high"))
    out = np.empty((ns,) + np.shape(t))
    for s in range(ns):
        tt = np.clip(t, tl[s], th[s])
        c = np.where((tt < tm[s])[None], lo[s][:, None].reshape((7,) + (1,) * np.ndim(t)),
                     hi[s][:, None].reshape((7,) + (1,) * np.ndim(t)))
        h = c[0] * tt + 0.5 * c[1] * tt ** 2 + c[2] * tt ** 3 / 3 + 0.25 * c[3] * tt ** 4 + 0.2 * c[4] * tt ** 5 + c[5]
        cp = c[0] + c[1] * tt + c[2] * tt ** 2 + c[3] * tt ** 3 + c[4] * tt ** 4
        h = h + cp * (t - tt)
        out[s] = h * R_U / mech.mw[s]
    return out


def fill_mixture_state(b: HostBlock, mech, rho, u, v, w, p, t, y):
    """bv, sv and cv of a thermally perfect mixture on the whole padded block."""
    bv, sv, cv = b.a["bv"], b.a["sv"], b.a["cv"]
    bv[0], bv[1], bv[2], bv[3], bv[4], bv[5] = rho, u, v, w, p, t
    for s in range(mech.ns):
        sv[s] = y[s]
    h = nasa7_h(mech, bv[5])
    E = 0.5 * (bv[1] ** 2 + bv[2] ** 2 + bv[3] ** 2)
    for s in range(mech.ns):
        E = E + h[s] * sv[s]
    cv[0] = bv[0]
    cv[1], cv[2], cv[3] = bv[0] * bv[1], bv[0] * bv[2], bv[0] * bv[3]
    cv[4] = E * bv[0] - bv[4]
    for s in range(mech.ns):
        cv[5 + s] = bv[0] * sv[s]


def _mix_r(mech, y):
    return sum(y[s] * R_U / mech.mw[s] for s in range(mech.ns))


def turbulence_field(n, u_rms, k_max=8, k0=4.0, seed=1234):
    """Divergence-free random-phase velocity on an n^3 periodic lattice with the spectrum
    E(k) ~ k^4 exp(-2 k^2/k0^2) for |k| <= k_max, scaled to the given u_rms."""
    rng = np.random.default_rng(seed)
    kk = np.fft.fftfreq(n, 1.0 / n)
    KZ, KY, KX = np.meshgrid(kk, kk, kk, indexing="ij")
    K = np.sqrt(KX ** 2 + KY ** 2 + KZ ** 2)
    mask = (K > 0) & (K <= k_max)
    amp = np.zeros_like(K)
    Ek = K[mask] ** 4 * np.exp(-2 * K[mask] ** 2 / k0 ** 2)
    amp[mask] = np.sqrt(Ek / (4 * math.pi * K[mask] ** 2))
    comps = []
    for _ in range(3):
        ph = rng.uniform(0, 2 * math.pi, K.shape)
        comps.append(amp * np.exp(1j * ph))
    # project onto the plane normal to k
    kd = [KX, KY, KZ]
    K2 = np.where(K > 0, K ** 2, 1.0)
    dot = (kd[0] * comps[0] + kd[1] * comps[1] + kd[2] * comps[2]) / K2
    vel = [np.real(np.fft.ifftn(comps[a] - kd[a] * dot)) for a in range(3)]
    rms = math.sqrt(sum(np.mean(v_ ** 2) for v_ in vel) / 3)
    return [v_ * (u_rms / rms) for v_ in vel]


def h2_air_box(mech, n_nodes=192, ngg=3, length=1e-3, seed=2024, scheme=abi.INV_HLLC,
               reconstruction=abi.REC_WENO5, viscous_order=2, reaction=True):
    """Reacting H2/air box: n_nodes^3 uniform periodic grid (node 0 == node n-1) with sides L,
    divergence-free random-phase velocity (|k| <= 8, k^4 exp(-2k^2/k0^2), k0 = 4,
    u_rms = 10 m/s), T = 1200 K + five 300 K Gaussian hot spots of radius 0.05 mm at seeded
    positions, p = 1 atm, stoichiometric premixed H2/air."""
    m = n_nodes
    nper = m - 1  # periodic intervals
    dx = length / nper
    specs = array_specs(m, m, m, ngg, 5 + mech.ns, mech.ns, viscous_order=viscous_order,
                        roe=(scheme == abi.INV_ROE), reaction=reaction)
    b = HostBlock(m, m, m, ngg, specs)
    idx = (np.arange(-ngg, m + ngg)) % nper  # periodic image of every padded node
    u, v, w = turbulence_field(nper, 10.0, seed=seed)
    U = [f[np.ix_(idx, idx, idx)] for f in (u, v, w)]  # arrays indexed [k, j, i]
    rng = np.random.default_rng(seed + 1)
    centres = rng.uniform(0, length, (5, 3))
    q = idx * dx
    Z, Y, X = np.meshgrid(q, q, q, indexing="ij")
    T = np.full(X.shape, 1200.0)
    r0 = 0.05e-3
    for c in centres:
        d2 = 0
        for coord, cc in zip((X, Y, Z), c):
            dd = np.abs(coord - cc)
            dd = np.minimum(dd, length - dd)
            d2 = d2 + dd ** 2
        T += 300.0 * np.exp(-d2 / r0 ** 2)
    y = stoich_h2_air(mech)
    p = np.full(X.shape, 101325.0)
    rho = p / (_mix_r(mech, y) * T)
    fill_mixture_state(b, mech, rho, U[0], U[1], U[2], p, T, [np.full(X.shape, ys) for ys in y])
    mt = b.a["metric"]
    mt[0] = mt[4] = mt[8] = 1.0 / dx
    b.a["jac"][0] = dx ** 3
    faces = box_faces(m, m, m, {(d, s): abi.BC_PERIODIC for d in range(3) for s in (-1, 1)})
    c0 = math.sqrt(1.4 * 101325.0 / float(rho.mean()))
    par = make_param(n_var=5 + mech.ns, n_spec=mech.ns, dim=3, inviscid_scheme=scheme,
                     reconstruction=reconstruction, viscous_order=viscous_order, cfl=0.5,
                     rho_ref=float(rho.mean()), v_ref=c0, mech=mech.ptr())
    par.reaction = 1 if reaction else 0
    return Case("h2_air_box", par, [b], [faces], {"dt": 2e-9, "mech": mech, "dx": dx})


def h2_air_box_2t(mech, tt, n_nodes=10, ngg=3, length=1e-3, seed=77, t_ve_ratio=0.6):
    """Two-temperature H2/air box out of vibrational equilibrium: the reacting box's state
    (velocity field, hot spots, 1 atm, stoichiometric mixture with 2 % of it moved to H, O and
    OH) with T_ve = t_ve_ratio * T + 300 K at every node.  e_ve is left at zero, so a
    cv-from-bv pass fills it from T_ve (sync_two_temperature_state_from_sv)."""
    base = h2_air_box(mech, n_nodes=n_nodes, ngg=ngg, length=length, seed=seed, viscous_order=0, reaction=False)
    hb0 = base.blocks[0]
    m = n_nodes
    ns = mech.ns
    specs = array_specs(m, m, m, ngg, 6 + ns, ns + 1)
    specs["temperature_ve"] = (1, ngg)
    b = HostBlock(m, m, m, ngg, specs)
    for name in ("bv", "metric", "jac", "mul", "mach", "thermal_conductivity", "acoustic_speed", "gamma"):
        if name in hb0.a and name in b.a:
            b.a[name][...] = hb0.a[name]
    y = hb0.a["sv"].copy()
    rng = np.random.default_rng(seed + 5)
    moved = 0.02 * y[mech.index("O2")]
    for name, share in (("H", 0.2), ("O", 0.3), ("OH", 0.5)):
        y[mech.index(name)] += share * moved * rng.uniform(0.5, 1.5, moved.shape)
    y[mech.index("O2")] -= moved
    y /= y.sum(axis=0, keepdims=True)
    b.a["sv"][:ns] = y
    b.a["sv"][ns] = 0.0
    b.a["temperature_ve"][0] = t_ve_ratio * b.a["bv"][5] + 300.0
    par = make_param(n_var=6 + ns, n_spec=ns, dim=3, inviscid_scheme=abi.INV_HLLC, reconstruction=abi.REC_WENO5,
                     cfl=0.5, rho_ref=base.param.rho_ref, v_ref=base.param.v_ref, mech=mech.ptr(), two_t=tt.ptr())
    return Case("h2_air_box_2t", par, [b], base.faces, {"mech": mech, "two_t": tt, "dx": base.meta["dx"]})


def air5_box_2t(mech, tt, n_nodes=10, ngg=3, length=1e-2, seed=91, viscous_order=0, reaction=True,
                scheme=abi.INV_WENO5_CH, reconstruction=abi.REC_WENO5):
    """Two-temperature AIR5 periodic box with the post-shock conditions of a Mach-10 body: a
    uniform n_nodes^3 grid with sides L, random-phase velocity (u_rms = 400 m/s), T = 6000 K +
    three 2500 K Gaussian spots, T_ve = 0.45 T + 600 K (vibration lagging), p = 20 kPa, and
    partly dissociated air (N2 0.70, O2 0.10, NO 0.05, N 0.05, O 0.10 by mass, +-30 % seeded
    noise, renormalised).  bv, sv, T_ve and the geometry are set; cv and e_ve are left to a
    cv-from-bv pass."""
    m = n_nodes
    nper = m - 1
    dx = length / nper
    ns = mech.ns
    specs = array_specs(m, m, m, ngg, 6 + ns, ns + 1, viscous_order=viscous_order, reaction=reaction)
    specs["temperature_ve"] = (1, ngg)
    if viscous_order:
        specs["thermal_conductivity_ve"] = (1, ngg)
    b = HostBlock(m, m, m, ngg, specs)
    idx = (np.arange(-ngg, m + ngg)) % nper
    u, v, w = turbulence_field(nper, 400.0, k_max=3, k0=2.0, seed=seed)
    U = [f[np.ix_(idx, idx, idx)] for f in (u, v, w)]
    rng = np.random.default_rng(seed + 1)
    q = idx * dx
    Z, Y, X = np.meshgrid(q, q, q, indexing="ij")
    T = np.full(X.shape, 6000.0)
    for c in rng.uniform(0, length, (3, 3)):
        d2 = 0
        for coord, cc in zip((X, Y, Z), c):
            dd = np.abs(coord - cc)
            dd = np.minimum(dd, length - dd)
            d2 = d2 + dd ** 2
        T += 2500.0 * np.exp(-d2 / (0.2 * length) ** 2)
    base = {"N2": 0.70, "O2": 0.10, "NO": 0.05, "N": 0.05, "O": 0.10}
    y = np.stack([base[n] * (1 + 0.3 * rng.uniform(-1, 1, X.shape)) for n in mech.species])
    y /= y.sum(axis=0, keepdims=True)
    p = np.full(X.shape, 2.0e4)
    rho = p / ((y * (8314.462618 / mech.mw)[:, None, None, None]).sum(axis=0) * T)
    bv = b.a["bv"]
    bv[0], bv[1], bv[2], bv[3], bv[4], bv[5] = rho, U[0], U[1], U[2], p, T
    b.a["sv"][:ns] = y
    b.a["sv"][ns] = 0.0
    b.a["temperature_ve"][0] = 0.45 * T + 600.0
    mt = b.a["metric"]
    mt[0] = mt[4] = mt[8] = 1.0 / dx
    b.a["jac"][0] = dx ** 3
    faces = box_faces(m, m, m, {(d, s): abi.BC_PERIODIC for d in range(3) for s in (-1, 1)})
    c0 = math.sqrt(1.3 * 2.0e4 / float(rho.mean()))
    par = make_param(n_var=6 + ns, n_spec=ns, dim=3, inviscid_scheme=scheme, reconstruction=reconstruction,
                     viscous_order=viscous_order, cfl=0.3, rho_ref=float(rho.mean()), v_ref=c0, mech=mech.ptr(),
                     two_t=tt.ptr())
    par.reaction = 1 if reaction else 0
    return Case("air5_box_2t", par, [b], [faces], {"mech": mech, "two_t": tt, "dx": dx})


def reactive_shock_tube(mech, n_nodes=400, ngg=3, length=0.1, scheme=abi.INV_HLLC,
                        reconstruction=abi.REC_WENO5, reaction=True):
    """1-D reactive shock tube, stoichiometric H2/air: (T, p) = (1500 K, 5 atm) left of
    x = L/2 and (300 K, 1 atm) right of it, outflow faces."""
    mx, my, mz = n_nodes, 1, 1
    specs = array_specs(mx, my, mz, ngg, 5 + mech.ns, mech.ns, roe=(scheme == abi.INV_ROE), reaction=reaction)
    b = HostBlock(mx, my, mz, ngg, specs)
    dx = length / (mx - 1)
    x = np.arange(-ngg, mx + ngg) * dx
    left = x <= 0.5 * length
    shape = b.a["bv"][0].shape
    T = np.broadcast_to(np.where(left, 1500.0, 300.0)[None, None, :], shape).copy()
    p = np.broadcast_to(np.where(left, 5 * 101325.0, 101325.0)[None, None, :], shape).copy()
    y = stoich_h2_air(mech)
    rho = p / (_mix_r(mech, y) * T)
    z0 = np.zeros(shape)
    fill_mixture_state(b, mech, rho, z0, z0, z0, p, T, [np.full(shape, ys) for ys in y])
    mt = b.a["metric"]
    mt[0] = 1.0 / dx
    mt[4] = mt[8] = 1.0
    b.a["jac"][0] = dx
    faces = box_faces(mx, my, mz, {(0, -1): abi.BC_OUTFLOW, (0, 1): abi.BC_OUTFLOW,
                                   (1, -1): abi.BC_OUTFLOW, (1, 1): abi.BC_OUTFLOW})
    rho_l = float(rho[0, 0, 0])
    c_l = math.sqrt(1.4 * 5 * 101325.0 / rho_l)
    par = make_param(n_var=5 + mech.ns, n_spec=mech.ns, dim=2, inviscid_scheme=scheme,
                     reconstruction=reconstruction, cfl=0.5, rho_ref=rho_l, v_ref=c_l, mech=mech.ptr())
    par.reaction = 1 if reaction else 0
    return Case("reactive_shock_tube", par, [b], [faces], {"t_end": 50e-6, "mech": mech, "dx": dx})


# ---- the two-temperature AIR5 square cylinder (four body-fitted blocks) --------------------
def air5_freestream(mech, tt, mach=10.0, T=250.0, Tve=250.0, p=500.0, y=(0.767, 0.233, 0.0, 0.0, 0.0)):
    """Freestream state of the AIR5 cylinder as the reference's Inflow builds it from
    (mach, temperature, Tve, pressure, Y) (src/BoundCond.cpp:214-300): mw from Y, rho =
    p mw / (R_u T), e_ve at Tve, and the speed of sound of the translational-rotational gas, so
    the velocity is mach * c along +x."""
    ns = mech.ns
    yk = np.asarray(y, dtype=np.float64)
    mw = 0.0
    for i in range(ns):
        mw += yk[i] / mech.mw[i]
    mw = 1.0 / mw
    rho = p * mw / (R_U * T)
    # cp of the translational-rotational modes: 5/2 R (molecules) and 3/2 R (atoms) plus R
    geom = np.asarray(mech.d["geometry"])
    cv_tr = sum(yk[i] * (R_U / mech.mw[i]) * (1.5 if geom[i] == 0 else 2.5) for i in range(ns))
    r_mix = R_U / mw
    gamma = (cv_tr + r_mix) / cv_tr
    c = math.sqrt(gamma * r_mix * T)
    e_ve = mechmod.mixture_ve_energy(tt, mech.mw, Tve, yk)
    sv = np.concatenate([yk, [e_ve]])
    return dict(rho=rho, u=mach * c, v=0.0, w=0.0, p=p, T=T, Tve=Tve, y=yk, sv=sv, c=c, mw=mw)


def square_cylinder_air5(mech, tt, n_side=256, n_normal=512, ngg=3, side=0.01, half_box=0.04, first=1e-6,
                         mach=10.0, T_inf=250.0, p_inf=500.0, T_wall=300.0, viscous_order=2, reaction=True,
                         scheme=abi.INV_WENO5_CH, cfl=0.3):
    """Mach-10 two-temperature AIR5 flow over a square cylinder of side D on four body-fitted
    blocks of n_side x n_normal nodes (grid.square_cylinder): freestream inflow on the box except
    its downstream side (outflow), an isothermal 300 K wall (T_ve too), metrics and Jacobian from
    the grid as the reference's Mesh computes them.  Initial state: the freestream with the
    velocity damped and T, T_ve blended to the wall values over a 0.05 D layer at the body
    (an impulsive start that the first steps turn into the bow shock)."""
    from . import grid as gridmod
    from .field import face
    ns = mech.ns
    g = gridmod.square_cylinder(n_side, n_normal, side=side, half_box=half_box, first=first)
    inner = [[gridmod.register_inner_face(a, b, 2, ngg) for a, b in faces] for faces in g["inner"]]
    padded, g1 = gridmod.extend_coordinates(g["xyz"], inner, ngg)
    fs = air5_freestream(mech, tt, mach=mach, T=T_inf, Tve=T_inf, p=p_inf)
    blocks, faces = [], []
    h = 0.5 * side
    for b in range(4):
        X, Y, Z = padded[b]
        met, jac = gridmod.metrics(padded[b], g1, ngg)
        mx, my, mz = n_side, n_normal, 1
        specs = array_specs(mx, my, mz, ngg, 6 + ns, ns + 1, viscous_order=viscous_order, reaction=reaction)
        specs["temperature_ve"] = (1, ngg)
        if viscous_order:
            specs["thermal_conductivity_ve"] = (1, ngg)
        hb = HostBlock(mx, my, mz, ngg, specs)
        s = (slice(g1 - ngg, g1 + mz + ngg), slice(g1 - ngg, g1 + my + ngg), slice(g1 - ngg, g1 + mx + ngg))
        x, y = X[s], Y[s]
        d = np.sqrt(np.maximum(np.abs(x) - h, 0.0) ** 2 + np.maximum(np.abs(y) - h, 0.0) ** 2)
        blend = np.exp(-d / (0.05 * side))
        T = fs["T"] + (T_wall - fs["T"]) * blend
        bv = hb.a["bv"]
        bv[0] = fs["p"] / ((R_U / fs["mw"]) * T)
        bv[1] = fs["u"] * (1.0 - blend)
        bv[2] = 0.0
        bv[3] = 0.0
        bv[4] = fs["p"]
        bv[5] = T
        for i in range(ns):
            hb.a["sv"][i] = fs["y"][i]
        hb.a["sv"][ns] = 0.0  # e_ve from T_ve by the first cv-from-bv pass
        hb.a["temperature_ve"][0] = T
        hb.a["metric"][...] = met
        hb.a["jac"][0] = jac
        blocks.append(hb)
        fl = []
        for (i1, i2, j1, j2, k1, k2, lab) in g["faces"][b]:
            if lab == abi.BC_WALL:
                fl.append(face(abi.BC_WALL, 1, -1, (i1, j1, k1), (i2, j2, k2), wall_temperature=T_wall,
                               wall_temperature_ve=T_wall))
            elif lab == abi.BC_INFLOW:
                fl.append(face(abi.BC_INFLOW, 1, 1, (i1, j1, k1), (i2, j2, k2), sv=fs["sv"], rho=fs["rho"],
                               u=fs["u"], v=0.0, w=0.0, p=fs["p"], T=fs["T"]))
            else:
                fl.append(face(abi.BC_OUTFLOW, 1, 1, (i1, j1, k1), (i2, j2, k2)))
        faces.append(fl)
    par = make_param(n_var=6 + ns, n_spec=ns, dim=2, inviscid_scheme=scheme, reconstruction=abi.REC_WENO5,
                     viscous_order=viscous_order, cfl=cfl, rho_ref=fs["rho"], v_ref=fs["u"], mech=mech.ptr(),
                     two_t=tt.ptr())
    par.reaction = 1 if reaction else 0
    par.p_ref, par.c_ref = fs["p"], fs["c"]
    return Case("square_cylinder_air5", par, blocks, faces,
                {"mech": mech, "two_t": tt, "inner": inner, "grid": g, "freestream": fs, "padded": padded,
                 "g1": g1})
