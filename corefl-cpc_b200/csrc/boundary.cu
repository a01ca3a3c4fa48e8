// Ghost-layer fill of bv/sv/cv from the face boundary conditions of a block.
//
// Faces are applied one launch per face in the reference's priority order
// (farfield < outflow < inflow < symmetry < wall < periodic, src/BoundCond.cu:3846-3998), so
// the edges and corners shared by two faces end with the same values the reference gets.
//   outflow  : zeroth-order extrapolation (apply_outflow without back pressure,
//              src/BoundCond.cu:2204-2350)
//   periodic : average of the coincident end nodes, then ghost copy from the far side
//              (apply_periodic, src/BoundCond.cu:3390-3440)
//   symmetry : mirror with the normal velocity reflected (apply_symmetry, src/BoundCond.cu:2130-2202)
//   inflow   : fixed supersonic state on the face node and all ghost layers (the constant
//              state of apply_inflow, src/BoundCond.cu:2484; its profile, subsonic and
//              turbulent-fluctuation branches are not built)
//   wall     : no-slip, non-catalytic, adiabatic or isothermal (apply_wall,
//              src/BoundCond.cu:3055-3389)
// Every filled node gets its cv recomputed (compute_cv_from_bv_1_point, FieldOperation.cuh:163).
#include "point.cuh"
#include "launch.h"
#include "boundary.cuh"

namespace cb2 {

__device__ __forceinline__ bool face_point_at(const FaceBC &f, long long t, int &i, int &j, int &k) {
  const int n0 = f.end[0] - f.start[0] + 1, n1 = f.end[1] - f.start[1] + 1, n2 = f.end[2] - f.start[2] + 1;
  if (t >= (long long)n0 * n1 * n2) return false;
  i = f.start[0] + (int)(t % n0);
  j = f.start[1] + (int)((t / n0) % n1);
  k = f.start[2] + (int)(t / ((long long)n0 * n1));
  return true;
}

__device__ __forceinline__ bool face_point(const FaceBC &f, int &i, int &j, int &k) {
  return face_point_at(f, (long long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k);
}

// One thread per (face node, layer): consecutive threads take consecutive nodes of one layer.
// The layers of a face node are independent of one another in the outflow, inflow, symmetry and
// wall fills (each reads only interior nodes or the face's own constants), so every layer's cv
// rebuild -- the costly part with two temperatures -- runs in its own thread.
__device__ __forceinline__ bool face_layer_point(const FaceBC &f, int n_layer, int &i, int &j, int &k, int &l) {
  const long long n = (long long)(f.end[0] - f.start[0] + 1) * (f.end[1] - f.start[1] + 1) * (f.end[2] - f.start[2] + 1);
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n * n_layer) return false;
  l = (int)(t / n);
  return face_point_at(f, t - l * n, i, j, k);
}

// gamma = cp / (cp - R) of the node's mixture at its T (the back-pressure outflow's sound speed).
template <int NS>
__device__ __forceinline__ double node_gamma(const Zone &z, const Param &p, idx_t g) {
  if constexpr (NS == 0) {
    return kGammaAir;
  } else {
    const idx_t sz = z.L.sz;
    double cp[NS];
    species_cp<NS>(z.bv[g + 5 * sz], p.mech, cp);
    double cpm = 0, r = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      cpm += z.sv[g + l * sz] * cp[l];
      r += z.sv[g + l * sz] * __ldg(p.mech.gas_const + l);
    }
    return cpm / (cpm - r);
  }
}

template <int NS>
__global__ void k_bc_outflow(Zone z, Param p, FaceBC f) {
  int i, j, k, gl;
  if (!face_layer_point(f, z.ngg, i, j, k, gl)) return;
  ++gl;  // ghost layers 1..ngg
  int d[3] = {0, 0, 0};
  d[f.face] = f.direction;
  const idx_t sz = z.L.sz;
  const idx_t gb = z.L.at(i, j, k);
  if (f.p > 0) {
    // back pressure (Outflow::if_backPressure, src/BoundCond.cu:2219-2320): where the face node's
    // normal Mach number is below 1 the face state takes the back pressure along the acoustic
    // invariant of the node inside, and the ghosts are reflected about it; the face node itself
    // keeps its values
    const double *M = z.metric + (idx_t)(3 * f.face) * sz;
    double nx = M[gb], ny = M[gb + sz], nz = M[gb + 2 * sz];
    const double gni = f.direction / sqrt(nx * nx + ny * ny + nz * nz);
    nx *= gni; ny *= gni; nz *= gni;
    double u_b = z.bv[gb + sz], v_b = z.bv[gb + 2 * sz], w_b = z.bv[gb + 3 * sz];
    const double u_face = nx * u_b + ny * v_b + nz * w_b;
    double p_b = z.bv[gb + 4 * sz], rho_b = z.bv[gb];
    const double a_b = sqrt(node_gamma<NS>(z, p, gb) * p_b / rho_b);
    const idx_t gg = z.L.at(i + gl * d[0], j + gl * d[1], k + gl * d[2]);
    const idx_t gi = z.L.at(i - gl * d[0], j - gl * d[1], k - gl * d[2]);
    if (fabs(u_face / a_b) < 1) {
      p_b = f.p;
      const idx_t g1 = z.L.at(i - d[0], j - d[1], k - d[2]);
      const double d1 = z.bv[g1], u1 = z.bv[g1 + sz], v1 = z.bv[g1 + 2 * sz], w1 = z.bv[g1 + 3 * sz],
                   p1 = z.bv[g1 + 4 * sz];
      const double c1 = sqrt(node_gamma<NS>(z, p, g1) * p1 / d1);
      const double temp = (p_b - p1) / c1;
      rho_b = d1 + temp / c1;
      u_b = u1 - nx * temp / d1;
      v_b = v1 - ny * temp / d1;
      w_b = w1 - nz * temp / d1;
      const double p_g = 2 * p_b - z.bv[gi + 4 * sz], rho_g = 2 * rho_b - z.bv[gi];
      z.bv[gg] = rho_g;
      z.bv[gg + sz] = 2 * u_b - z.bv[gi + sz];
      z.bv[gg + 2 * sz] = 2 * v_b - z.bv[gi + 2 * sz];
      z.bv[gg + 3 * sz] = 2 * w_b - z.bv[gi + 3 * sz];
      z.bv[gg + 4 * sz] = p_g;
      for (int l = 0; l < p.n_scalar; ++l) z.sv[gg + l * sz] = 2 * z.sv[gb + l * sz] - z.sv[gi + l * sz];
      double R = kRAir;
      if constexpr (NS > 0) {
        R = 0;
        for (int l = 0; l < NS; ++l) R += z.sv[gg + l * sz] * __ldg(p.mech.gas_const + l);
      }
      z.bv[gg + 5 * sz] = p_g / (rho_g * R);
      if (NS > 0 && p.i_eve >= 0) {
        const double tve_b = z.tve[gb] > 0.0 ? z.tve[gb] : z.bv[gb + 5 * sz];
        const double tve_i = z.tve[gi] > 0.0 ? z.tve[gi] : z.bv[gi + 5 * sz];
        z.tve[gg] = fmax(2 * tve_b - tve_i, 1.0);
      }
    } else {
      z.bv[gg] = rho_b;
      z.bv[gg + sz] = u_b;
      z.bv[gg + 2 * sz] = v_b;
      z.bv[gg + 3 * sz] = w_b;
      z.bv[gg + 4 * sz] = p_b;
      z.bv[gg + 5 * sz] = z.bv[gb + 5 * sz];
      for (int l = 0; l < p.n_scalar; ++l) z.sv[gg + l * sz] = z.sv[gb + l * sz];
      if (p.i_eve >= 0) z.tve[gg] = z.tve[gb] > 0.0 ? z.tve[gb] : z.bv[gb + 5 * sz];
    }
    cv_point<NS>(z, p, gg);
    return;
  }
  {
    const idx_t gg = z.L.at(i + gl * d[0], j + gl * d[1], k + gl * d[2]);
    for (int l = 0; l < 6; ++l) z.bv[gg + l * sz] = z.bv[gb + l * sz];
    for (int l = 0; l < p.n_scalar; ++l) z.sv[gg + l * sz] = z.sv[gb + l * sz];
    // two-temperature: the ghost T_ve (the starting guess of its inversion from e_ve) is the
    // face node's, or its T when unset (src/BoundCond.cu:2339-2345)
    if (p.i_eve >= 0) z.tve[gg] = z.tve[gb] > 0.0 ? z.tve[gb] : z.bv[gb + 5 * sz];
    cv_point<NS>(z, p, gg);
  }
}

template <int NS>
__global__ void k_bc_periodic(Zone z, Param p, FaceBC f) {
  int i, j, k;
  if (!face_point(f, i, j, k)) return;
  int d[3] = {0, 0, 0};
  d[f.face] = f.direction;
  int o[3] = {i, j, k};
  const int ext[3] = {z.mx, z.my, z.mz};
  o[f.face] = f.direction < 0 ? ext[f.face] - 1 : 0;
  const idx_t sz = z.L.sz;
  const idx_t gb = z.L.at(i, j, k), go = z.L.at(o[0], o[1], o[2]);
  for (int l = 0; l < 6; ++l) {
    const double ave = 0.5 * (z.bv[gb + l * sz] + z.bv[go + l * sz]);
    z.bv[gb + l * sz] = ave;
    z.bv[go + l * sz] = ave;
  }
  for (int l = 0; l < p.n_scalar; ++l) {
    const double ave = 0.5 * (z.sv[gb + l * sz] + z.sv[go + l * sz]);
    z.sv[gb + l * sz] = ave;
    z.sv[go + l * sz] = ave;
  }
  cv_point<NS>(z, p, gb);
  for (int gl = 1; gl <= z.ngg; ++gl) {
    const idx_t gg = z.L.at(i + gl * d[0], j + gl * d[1], k + gl * d[2]);
    const idx_t gs = z.L.at(o[0] + gl * d[0], o[1] + gl * d[1], o[2] + gl * d[2]);
    for (int l = 0; l < 6; ++l) z.bv[gg + l * sz] = z.bv[gs + l * sz];
    for (int l = 0; l < p.n_scalar; ++l) z.sv[gg + l * sz] = z.sv[gs + l * sz];
    cv_point<NS>(z, p, gg);
  }
}

// Symmetry (apply_symmetry, src/BoundCond.cu:2130-2202): the face node takes the tangential
// velocity and the rho, p, T, Y of its inner neighbour; ghosts mirror the interior with the
// normal velocity reflected.
template <int NS>
__global__ void k_bc_symmetry(Zone z, Param p, FaceBC f) {
  int i, j, k, gl;
  if (!face_layer_point(f, z.ngg + 1, i, j, k, gl)) return;
  int d[3] = {0, 0, 0};
  d[f.face] = f.direction;
  const idx_t sz = z.L.sz;
  const idx_t gb = z.L.at(i, j, k);
  const idx_t g1 = z.L.at(i - d[0], j - d[1], k - d[2]);
  const double *M = z.metric + (idx_t)(3 * f.face) * sz;
  double kx = M[gb], ky = M[gb + sz], kz = M[gb + 2 * sz];
  const double km = sqrt(kx * kx + ky * ky + kz * kz);
  kx /= km; ky /= km; kz /= km;
  if (gl == 0) {
    const double u1 = z.bv[g1 + sz], v1 = z.bv[g1 + 2 * sz], w1 = z.bv[g1 + 3 * sz];
    const double uk = kx * u1 + ky * v1 + kz * w1;
    z.bv[gb + sz] = u1 - kx * uk;
    z.bv[gb + 2 * sz] = v1 - ky * uk;
    z.bv[gb + 3 * sz] = w1 - kz * uk;
    z.bv[gb] = z.bv[g1];
    z.bv[gb + 4 * sz] = z.bv[g1 + 4 * sz];
    z.bv[gb + 5 * sz] = z.bv[g1 + 5 * sz];
    for (int l = 0; l < p.n_scalar; ++l) z.sv[gb + l * sz] = z.sv[g1 + l * sz];
    if (p.i_eve >= 0) z.tve[gb] = z.tve[g1];
    cv_point<NS>(z, p, gb);
  } else {
    const idx_t gg = z.L.at(i + gl * d[0], j + gl * d[1], k + gl * d[2]);
    const idx_t gi = z.L.at(i - gl * d[0], j - gl * d[1], k - gl * d[2]);
    z.bv[gg] = z.bv[gi];
    const double u = z.bv[gi + sz], v = z.bv[gi + 2 * sz], w = z.bv[gi + 3 * sz];
    const double uk = kx * u + ky * v + kz * w;
    z.bv[gg + sz] = u - 2 * uk * kx;
    z.bv[gg + 2 * sz] = v - 2 * uk * ky;
    z.bv[gg + 3 * sz] = w - 2 * uk * kz;
    z.bv[gg + 4 * sz] = z.bv[gi + 4 * sz];
    z.bv[gg + 5 * sz] = z.bv[gi + 5 * sz];
    for (int l = 0; l < p.n_scalar; ++l) z.sv[gg + l * sz] = z.sv[gi + l * sz];
    if (p.i_eve >= 0) z.tve[gg] = z.tve[gi];
    cv_point<NS>(z, p, gg);
  }
}

// Constant inflow state on the face node and every ghost layer, scalars (Y_k, then e_ve) from
// the face's state (Inflow::sv); rebuilding cv brings T_ve into agreement with e_ve, starting
// its inversion from the node's T_ve as the reference does.
template <int NS>
__global__ void k_bc_inflow(Zone z, Param p, FaceBC f) {
  int i, j, k, gl;
  if (!face_layer_point(f, z.ngg + 1, i, j, k, gl)) return;
  int d[3] = {0, 0, 0};
  d[f.face] = f.direction;
  const idx_t sz = z.L.sz;
  {
    const idx_t gg = z.L.at(i + gl * d[0], j + gl * d[1], k + gl * d[2]);
    z.bv[gg] = f.rho;
    z.bv[gg + sz] = f.u;
    z.bv[gg + 2 * sz] = f.v;
    z.bv[gg + 3 * sz] = f.w;
    z.bv[gg + 4 * sz] = f.p;
    z.bv[gg + 5 * sz] = f.T;
    for (int l = 0; l < p.n_scalar; ++l) z.sv[gg + l * sz] = f.sv[l];
    cv_point<NS>(z, p, gg);
  }
}

// Index of the interior node a wall reads, moved off any physical boundary of the block
// (project_to_interior in apply_wall, src/BoundCond.cu:3070-3088).  The face flags exist for
// face nodes only; a tangential index in the ghost range (extended face ranges) reads no
// flag here, where the reference's flag lookup would leave the array.
__device__ __forceinline__ bool flag_at(const int *f, int a, int na, int b, int nb) {
  return a >= 0 && a < na && b >= 0 && b < nb && f[a + b * na] != 0;
}

__device__ __forceinline__ void project_to_interior(const Zone &z, int &i, int &j, int &k) {
  if (i <= 0 && flag_at(z.bt.il, j, z.my, k, z.mz)) i = 1;
  else if (i >= z.mx - 1 && flag_at(z.bt.ir, j, z.my, k, z.mz)) i = z.mx - 2;
  if (j <= 0 && flag_at(z.bt.jl, i, z.mx, k, z.mz)) j = 1;
  else if (j >= z.my - 1 && flag_at(z.bt.jr, i, z.mx, k, z.mz)) j = z.my - 2;
  if (z.mz > 1) {
    if (k <= 0 && flag_at(z.bt.kl, i, z.mx, j, z.my)) k = 1;
    else if (k >= z.mz - 1 && flag_at(z.bt.kr, i, z.mx, j, z.my)) k = z.mz - 2;
  }
}

// Farfield (apply_farfield, src/BoundCond.cu:2351-2482): from the normal Mach number of the node
// inside, a supersonic inflow takes the farfield state, a subsonic inflow blends it with the
// interior along the acoustic invariant (the pressure averaged, density and velocity shifted by
// the pressure jump), a subsonic outflow imposes the farfield pressure the same way, and a
// supersonic outflow keeps the interior state; the scalars come from the farfield on inflow and
// from the interior on outflow.  Subsonic ghosts are reflected about the face state, supersonic
// ones equal it.  One thread per (face node, layer): every layer reads interior nodes only.
template <int NS>
__global__ void k_bc_farfield(Zone z, Param p, FaceBC f) {
  int i, j, k, gl;
  if (!face_layer_point(f, z.ngg + 1, i, j, k, gl)) return;
  int d[3] = {0, 0, 0};
  d[f.face] = f.direction;
  const idx_t sz = z.L.sz;
  int ii = i - d[0], ij = j - d[1], ik = k - d[2];
  project_to_interior(z, ii, ij, ik);
  const idx_t gin = z.L.at(ii, ij, ik), gf = z.L.at(i, j, k);
  const double *M = z.metric + (idx_t)(3 * f.face) * sz;
  double nx = M[gf], ny = M[gf + sz], nz = M[gf + 2 * sz];
  const double gni = f.direction / sqrt(nx * nx + ny * ny + nz * nz);
  nx *= gni; ny *= gni; nz *= gni;
  const double rho_in = z.bv[gin], u_in = z.bv[gin + sz], v_in = z.bv[gin + 2 * sz], w_in = z.bv[gin + 3 * sz];
  const double p_in = z.bv[gin + 4 * sz], t_in = z.bv[gin + 5 * sz];
  double c_in;
  if constexpr (NS == 0) c_in = sqrt(fmax(kGammaAir * kRAir * t_in, 1e-12));
  else c_in = fmax(z.acoustic[gin], 1e-12);
  const double rho_c_in = fmax(rho_in * c_in, 1e-12);
  const double mn_in = (u_in * nx + v_in * ny + w_in * nz) / c_in;
  const bool tt = NS > 0 && p.i_eve >= 0;
  constexpr int NSC = NS + 1;  // species and, with two temperatures, e_ve
  double sv_b[NSC];
  auto r_mix = [&]() {
    if constexpr (NS == 0) {
      return kRAir;
    } else {
      double r = 0;
#pragma unroll
      for (int l = 0; l < NS; ++l) r += sv_b[l] * __ldg(p.mech.gas_const + l);
      return fmax(r, 1e-12);
    }
  };
  double rho_b = rho_in, u_b = u_in, v_b = v_in, w_b = w_in, p_b = p_in, t_b = t_in;
  double tve_b = t_in;
  if (tt) tve_b = z.tve[gin] > 0.0 ? z.tve[gin] : t_in;
  if (mn_in < 0.0) {
    for (int l = 0; l < p.n_scalar; ++l) sv_b[l] = f.sv[l];
    if (mn_in <= -1.0) {
      rho_b = f.rho; u_b = f.u; v_b = f.v; w_b = f.w; p_b = f.p; t_b = f.T;
    } else {
      const double du_n = (f.u - u_in) * nx + (f.v - v_in) * ny + (f.w - w_in) * nz;
      p_b = 0.5 * (p_in + f.p - rho_in * c_in * du_n);
      p_b = fmax(p_b, 0.1 * fmax(f.p, 1.0));
      rho_b = f.rho + (p_b - f.p) / (c_in * c_in);
      rho_b = fmax(rho_b, 0.1 * fmax(f.rho, 1e-12));
      u_b = f.u - (p_b - f.p) * nx / rho_c_in;
      v_b = f.v - (p_b - f.p) * ny / rho_c_in;
      w_b = f.w - (p_b - f.p) * nz / rho_c_in;
      t_b = p_b / fmax(rho_b * r_mix(), 1e-12);
    }
    if (tt) tve_b = f.wall_Tve > 0.0 ? f.wall_Tve : t_b;
  } else {
    for (int l = 0; l < p.n_scalar; ++l) sv_b[l] = z.sv[gin + l * sz];
    if (mn_in < 1.0) {
      p_b = f.p;
      const double dp = p_b - p_in;
      rho_b = rho_in + dp / (c_in * c_in);
      rho_b = fmax(rho_b, 0.1 * fmax(rho_in, 1e-12));
      u_b = u_in - dp * nx / rho_c_in;
      v_b = v_in - dp * ny / rho_c_in;
      w_b = w_in - dp * nz / rho_c_in;
      t_b = p_b / fmax(rho_b * r_mix(), 1e-12);
    }
  }
  double st[6] = {rho_b, u_b, v_b, w_b, p_b, t_b};
  double tve_s = tve_b;
  idx_t gw = gf;
  if (gl > 0) {
    int ai = i - gl * d[0], aj = j - gl * d[1], ak = k - gl * d[2];
    project_to_interior(z, ai, aj, ak);
    const idx_t gi = z.L.at(ai, aj, ak);
    gw = z.L.at(i + gl * d[0], j + gl * d[1], k + gl * d[2]);
    if (mn_in > -1.0 && mn_in < 1.0) {
      double rho_g = 2 * rho_b - z.bv[gi], p_g = 2 * p_b - z.bv[gi + 4 * sz];
      rho_g = fmax(rho_g, 0.1 * fmax(rho_b, 1e-12));
      p_g = fmax(p_g, 0.1 * fmax(p_b, 1.0));
      st[0] = rho_g;
      st[1] = 2 * u_b - z.bv[gi + sz];
      st[2] = 2 * v_b - z.bv[gi + 2 * sz];
      st[3] = 2 * w_b - z.bv[gi + 3 * sz];
      st[4] = p_g;
      st[5] = p_g / fmax(rho_g * r_mix(), 1e-12);
    }
  }
  // set_boundary_state (src/BoundCond.cu:55-76)
#pragma unroll
  for (int l = 0; l < 6; ++l) z.bv[gw + l * sz] = st[l];
  for (int l = 0; l < p.n_scalar; ++l) z.sv[gw + l * sz] = sv_b[l];
  if (tt) z.tve[gw] = fmax(tve_s, 1.0);
  cv_point<NS>(z, p, gw);
}

// No-slip, non-catalytic wall, isothermal (wall_T > 0) or adiabatic (apply_wall,
// src/BoundCond.cu:3055-3389, without jets, blowing or wall fluctuations): the wall node takes
// p and Y of the first interior node and T_wall; ghosts mirror the interior velocity and, for
// an isothermal wall, T_ghost = 2 T_wall - T_inner (floored at T_wall when it drops below
// 0.1 T_wall; at 0.1 T_wall with two temperatures).  Two temperatures: the wall's T_ve is the
// given wall_Tve (else T_wall) on an isothermal wall and the interior's on an adiabatic one; the
// ghost T_ve mirrors it like T (floored at 0.1 max(T_ve,wall, 1)); e_ve of the wall node and of
// every ghost is the mixture's at that T_ve.
template <int NS>
__global__ void k_bc_wall(Zone z, Param p, FaceBC f) {
  int i, j, k, gl;
  if (!face_layer_point(f, z.ngg + 1, i, j, k, gl)) return;
  int d[3] = {0, 0, 0};
  d[f.face] = f.direction;
  const idx_t sz = z.L.sz;
  const idx_t gb = z.L.at(i, j, k);
  int ii = i - d[0], ij = j - d[1], ik = k - d[2];
  project_to_interior(z, ii, ij, ik);
  const idx_t g1 = z.L.at(ii, ij, ik);
  const bool iso = f.wall_T > 0;
  const bool tt = NS > 0 && p.i_eve >= 0;
  const double t_wall = iso ? f.wall_T : z.bv[g1 + 5 * sz];
  double tve_wall = t_wall;
  if (tt) {
    const double tve_in = z.tve[g1] > 0.0 ? z.tve[g1] : z.bv[g1 + 5 * sz];
    tve_wall = !iso ? tve_in : (f.wall_Tve > 0.0 ? f.wall_Tve : t_wall);
  }
  // a fully catalytic wall (Wall::catalytic_type 1) gives its face node and ghosts the wall's
  // mass fractions f.sv (Wall::yk); a non-catalytic one copies them from the interior
  const bool cat = NS > 0 && f.sv != nullptr;
  // the wall's velocity: at rest, or blowing along its inward normal while the step lies in the
  // blowing window (src/BoundCond.cu:3226-3245): blow_coefficient x max(the inner node's normal
  // velocity towards the wall, and for steps <= 50 the freestream's (f.u, f.v, f.w))
  double wu = 0, wv = 0, ww = 0;
  if (f.blow && p.step >= f.blow_start && p.step <= f.blow_end) {
    const double *Mf = z.metric + (idx_t)(3 * f.face) * sz;
    double nx = Mf[gb], ny = Mf[gb + sz], nz = Mf[gb + 2 * sz];
    const double ninv = f.direction / fmax(sqrt(nx * nx + ny * ny + nz * nz), 1e-30);
    nx *= ninv; ny *= ninv; nz *= ninv;
    const double vn_local = nx * z.bv[g1 + sz] + ny * z.bv[g1 + 2 * sz] + nz * z.bv[g1 + 3 * sz];
    const double vn_inf = nx * f.u + ny * f.v + nz * f.w;
    const double seed = p.step <= 50 ? fmax(vn_inf, 0.0) : 0.0;
    const double blow = fmax(f.blow_coef, 0.0) * fmax(fmax(vn_local, 0.0), seed);
    wu = -blow * nx;
    wv = -blow * ny;
    ww = -blow * nz;
  }
  double R = kRAir;
  if (gl == 0) {
    const double pw = z.bv[g1 + 4 * sz];
    if constexpr (NS > 0) {
      R = 0;
      for (int s = 0; s < NS; ++s) {
        z.sv[gb + s * sz] = cat ? f.sv[s] : z.sv[g1 + s * sz];
        R += z.sv[gb + s * sz] * __ldg(p.mech.gas_const + s);
      }
    }
    z.bv[gb] = pw / (t_wall * R);
    z.bv[gb + sz] = wu;
    z.bv[gb + 2 * sz] = wv;
    z.bv[gb + 3 * sz] = ww;
    z.bv[gb + 4 * sz] = pw;
    z.bv[gb + 5 * sz] = t_wall;
    if constexpr (NS > 0) {
      if (tt) {
        double y[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) y[s] = z.sv[gb + s * sz];
        z.tve[gb] = tve_wall;
        z.sv[gb + p.i_eve * sz] = mixture_ve_energy<NS>(tve_wall, y, p.mech, nullptr);
      }
    }
    cv_point<NS>(z, p, gb);
  } else {
    int ai = i - gl * d[0], aj = j - gl * d[1], ak = k - gl * d[2];
    project_to_interior(z, ai, aj, ak);
    const idx_t gi = z.L.at(ai, aj, ak);
    const idx_t gg = z.L.at(i + gl * d[0], j + gl * d[1], k + gl * d[2]);
    const double p_i = z.bv[gi + 4 * sz], t_i = z.bv[gi + 5 * sz];
    double t_g = t_i;
    if (iso) {
      t_g = 2 * t_wall - t_i;
      if (t_g <= 0.1 * t_wall) t_g = tt ? 0.1 * t_wall : t_wall;
    }
    double tve_g = t_g;
    if (tt) {
      const double tve_i = z.tve[gi] > 0.0 ? z.tve[gi] : t_i;
      tve_g = tve_i;
      if (iso) {
        tve_g = 2 * tve_wall - tve_i;
        const double floor_ve = 0.1 * fmax(tve_wall, 1.0);
        if (tve_g <= floor_ve) tve_g = floor_ve;
      }
    }
    if constexpr (NS > 0) {
      R = 0;
      for (int s = 0; s < NS; ++s) {
        // catalytic: R of the face node, which holds the wall's mass fractions
        const double y = cat ? f.sv[s] : z.sv[gi + s * sz];
        z.sv[gg + s * sz] = y;
        R += y * __ldg(p.mech.gas_const + s);
      }
    }
    z.bv[gg] = p_i / (t_g * R);
    z.bv[gg + sz] = 2 * wu - z.bv[gi + sz];
    z.bv[gg + 2 * sz] = 2 * wv - z.bv[gi + 2 * sz];
    z.bv[gg + 3 * sz] = 2 * ww - z.bv[gi + 3 * sz];
    z.bv[gg + 4 * sz] = p_i;
    z.bv[gg + 5 * sz] = t_g;
    if constexpr (NS > 0) {
      if (tt) {
        double y[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) y[s] = z.sv[gg + s * sz];
        z.tve[gg] = tve_g;
        z.sv[gg + p.i_eve * sz] = mixture_ve_energy<NS>(tve_g, y, p.mech, nullptr);
      }
    }
    cv_point<NS>(z, p, gg);
  }
}

// Exchange across one inner face of a multi-block grid (inner_communication,
// src/DataCommunication.cu:36-124), one thread per node of the registered face range (the face
// layer and its ngg ghost layers): the node index in the target block follows the registered
// orientation (src_tar, loop directions).  On the coincident face layer the two blocks' values
// are averaged into both, except that a node at rest in the target block (a wall corner) is
// copied from there when this block's node moves; ghost nodes take the target block's values.
// cv of every written node is rebuilt (the two-temperature sync included).
template <int NS>
__global__ void k_inner_exchange(Zone z, Zone zt, Param p, cb2_inner_face f) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n01 = (long long)f.n_point[0] * f.n_point[1];
  if (t >= n01 * f.n_point[2]) return;
  int n[3];
  n[0] = (int)(t % f.n_point[0]);
  n[1] = (int)((t / f.n_point[0]) % f.n_point[1]);
  n[2] = (int)(t / n01);
  int idx[3], it[3], d_idx[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    d_idx[a] = f.loop_dir[a] * n[a];
    idx[a] = f.range_start[a] + d_idx[a];
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) it[a] = f.target_start[a] + f.target_loop_dir[a] * d_idx[f.src_tar[a]];
  const idx_t sz = z.L.sz, szt = zt.L.sz;
  const idx_t g = z.L.at(idx[0], idx[1], idx[2]), gt = zt.L.at(it[0], it[1], it[2]);
  const int face_layer = f.direction > 0 ? f.range_start[f.face] : f.range_end[f.face];
  if (idx[f.face] == face_layer) {
    const double u_this = norm3d(z.bv[g + sz], z.bv[g + 2 * sz], z.bv[g + 3 * sz]);
    if (fabs(u_this) > 1e-15) {
      const double u_that = norm3d(zt.bv[gt + szt], zt.bv[gt + 2 * szt], zt.bv[gt + 3 * szt]);
      if (fabs(u_that) < 1e-15) {
        for (int l = 0; l < 6; ++l) z.bv[g + l * sz] = zt.bv[gt + l * szt];
        for (int l = 0; l < p.n_scalar; ++l) z.sv[g + l * sz] = zt.sv[gt + l * szt];
        if (p.i_eve >= 0) z.tve[g] = zt.tve[gt];
      } else {
        for (int l = 0; l < 6; ++l) {
          const double ave = 0.5 * (zt.bv[gt + l * szt] + z.bv[g + l * sz]);
          z.bv[g + l * sz] = ave;
          zt.bv[gt + l * szt] = ave;
        }
        for (int l = 0; l < p.n_scalar; ++l) {
          const double ave = 0.5 * (zt.sv[gt + l * szt] + z.sv[g + l * sz]);
          z.sv[g + l * sz] = ave;
          zt.sv[gt + l * szt] = ave;
        }
        if (p.i_eve >= 0) {
          const double ave = 0.5 * (zt.tve[gt] + z.tve[g]);
          z.tve[g] = ave;
          zt.tve[gt] = ave;
        }
        cv_point<NS>(zt, p, gt);
      }
    }
  } else {
    for (int l = 0; l < 6; ++l) z.bv[g + l * sz] = zt.bv[gt + l * szt];
    for (int l = 0; l < p.n_scalar; ++l) z.sv[g + l * sz] = zt.sv[gt + l * szt];
    if (p.i_eve >= 0) z.tve[g] = zt.tve[gt];
  }
  cv_point<NS>(z, p, g);
}

int launch_inner_exchange(const Zone &z, const Zone &zt, const Param &p, const cb2_inner_face &f, cudaStream_t s,
                          int &nl) {
  const long long np = (long long)f.n_point[0] * f.n_point[1] * f.n_point[2];
  if (np <= 0) return CB2_OK;
  const unsigned blocks = (unsigned)((np + 127) / 128);
  ProfScope prof("inner_exchange", s);
  switch (p.n_spec) {
    case 0: k_inner_exchange<0><<<blocks, 128, 0, s>>>(z, zt, p, f); break;
    case 5: k_inner_exchange<5><<<blocks, 128, 0, s>>>(z, zt, p, f); break;
    case 9: k_inner_exchange<9><<<blocks, 128, 0, s>>>(z, zt, p, f); break;
    default: return CB2_ERR_UNSUPPORTED;
  }
  ++nl;
  return check_launch();
}

// The 8th-order node fluxes across one inner face (exchange_value task 1 -> inner_exchange,
// src/DataCommunication.cu:437-527): on the coincident face layer the two blocks' fluxes are
// averaged into both, every component of fFlux, gFlux and hFlux; on the ghost layers this block
// takes the neighbour's.  E: double, or float for the mixed form's FP32 node fluxes.
template <typename E>
__global__ void k_inner_flux_exchange(Zone z, Zone zt, int n_var, cb2_inner_face f) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n01 = (long long)f.n_point[0] * f.n_point[1];
  if (t >= n01 * f.n_point[2]) return;
  int n[3];
  n[0] = (int)(t % f.n_point[0]);
  n[1] = (int)((t / f.n_point[0]) % f.n_point[1]);
  n[2] = (int)(t / n01);
  int idx[3], it[3], d_idx[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    d_idx[a] = f.loop_dir[a] * n[a];
    idx[a] = f.range_start[a] + d_idx[a];
  }
#pragma unroll
  for (int a = 0; a < 3; ++a) it[a] = f.target_start[a] + f.target_loop_dir[a] * d_idx[f.src_tar[a]];
  const idx_t sz = z.L.sz, szt = zt.L.sz;
  const idx_t g = z.L.at(idx[0], idx[1], idx[2]), gt = zt.L.at(it[0], it[1], it[2]);
  E *F[3], *Ft[3];
  if constexpr (sizeof(E) == 4) {
    F[0] = z.fF32; F[1] = z.gF32; F[2] = z.hF32;
    Ft[0] = zt.fF32; Ft[1] = zt.gF32; Ft[2] = zt.hF32;
  } else {
    F[0] = z.fF; F[1] = z.gF; F[2] = z.hF;
    Ft[0] = zt.fF; Ft[1] = zt.gF; Ft[2] = zt.hF;
  }
  const int face_layer = f.direction > 0 ? f.range_start[f.face] : f.range_end[f.face];
  const bool coincident = idx[f.face] == face_layer;
  for (int l = 0; l < n_var; ++l)
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const E that = Ft[a][gt + l * szt];
      if (coincident) {
        const E ave = E(0.5) * (F[a][g + l * sz] + that);
        F[a][g + l * sz] = ave;
        Ft[a][gt + l * szt] = ave;
      } else {
        F[a][g + l * sz] = that;
      }
    }
}

int launch_inner_flux_exchange(const Zone &z, const Zone &zt, const Param &p, const cb2_inner_face &f,
                               cudaStream_t s, int &nl) {
  const long long np = (long long)f.n_point[0] * f.n_point[1] * f.n_point[2];
  if (np <= 0) return CB2_OK;
  const unsigned blocks = (unsigned)((np + 127) / 128);
  ProfScope prof("inner_flux_exchange", s);
  if (visc8_f32(p)) k_inner_flux_exchange<float><<<blocks, 128, 0, s>>>(z, zt, p.n_var, f);
  else k_inner_flux_exchange<double><<<blocks, 128, 0, s>>>(z, zt, p.n_var, f);
  ++nl;
  return check_launch();
}

// 2-D blocks: copy the k = 0 plane into every k ghost plane (eliminate_k_gradient_point).
__global__ void k_eliminate_k_gradient(Zone z, Param p) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x - z.ngg;
  const int j = blockIdx.y - z.ngg;
  if (i >= z.mx + z.ngg) return;
  eliminate_k_gradient_point(z, p, i, j);
}

// Periodic exchange of the 8th-order viscous node fluxes (periodic_exchange task 1,
// src/DataCommunication.cu:665-712).
// The node-flux arrays the periodic exchange works on: the caller's FP64 arrays, or the
// mixed form's FP32 copies.
template <typename F>
__device__ __forceinline__ void flux_arrays(const Zone &z, F *arr[3]) {
  if constexpr (sizeof(F) == 4) {
    arr[0] = z.fF32; arr[1] = z.gF32; arr[2] = z.hF32;
  } else {
    arr[0] = z.fF; arr[1] = z.gF; arr[2] = z.hF;
  }
}

template <typename F>
__global__ void k_periodic_flux(Zone z, Param p, FaceBC f) {
  int i, j, k;
  if (!face_point(f, i, j, k)) return;
  int d[3] = {0, 0, 0};
  d[f.face] = f.direction;
  int o[3] = {i, j, k};
  const int ext[3] = {z.mx, z.my, z.mz};
  o[f.face] = f.direction < 0 ? ext[f.face] - 1 : 0;
  const idx_t sz = z.L.sz;
  const idx_t gb = z.L.at(i, j, k), go = z.L.at(o[0], o[1], o[2]);
  F *arr[3];
  flux_arrays<F>(z, arr);
  for (int l = 0; l < p.n_var; ++l)
    for (int a = 0; a < 3; ++a) {
      const F ave = F(0.5) * (arr[a][gb + l * sz] + arr[a][go + l * sz]);
      arr[a][gb + l * sz] = ave;
      arr[a][go + l * sz] = ave;
    }
  for (int gl = 1; gl <= z.ngg; ++gl) {
    const idx_t gg = z.L.at(i + gl * d[0], j + gl * d[1], k + gl * d[2]);
    const idx_t gs = z.L.at(o[0] + gl * d[0], o[1] + gl * d[1], o[2] + gl * d[2]);
    for (int l = 0; l < p.n_var; ++l)
      for (int a = 0; a < 3; ++a) arr[a][gg + l * sz] = arr[a][gs + l * sz];
  }
}

static inline long long face_points(const FaceBC &f) {
  return (long long)(f.end[0] - f.start[0] + 1) * (f.end[1] - f.start[1] + 1) * (f.end[2] - f.start[2] + 1);
}

template <int NS>
__global__ void k_bc_periodic_pair(Zone z, Param p, FaceBC f) {
  bc_periodic_pair_item<NS>(z, p, f, (long long)blockIdx.x * blockDim.x + threadIdx.x);
}

// The same pairing for the 8th-order viscous node fluxes (components 1..n_var-1 of the three
// flux arrays; component 0 carries no viscous flux and is never read).
template <typename F>
__global__ void k_periodic_flux_pair(Zone z, Param p, FaceBC f) {
  PairItem it;
  const int g = z.ngg;
  if (!pair_item(f, g, (long long)blockIdx.x * blockDim.x + threadIdx.x, it)) return;
  const int m = f.face == 0 ? z.mx : (f.face == 1 ? z.my : z.mz);
  const idx_t sz = z.L.sz;
  F *arr[3];
  flux_arrays<F>(z, arr);
  if (it.p == 0) {
    const idx_t ga = along(z.L, f.face, it.i, it.j, it.k, 0), gb = along(z.L, f.face, it.i, it.j, it.k, m - 1);
    for (int l = 1; l < p.n_var; ++l)
      for (int a = 0; a < 3; ++a) {
        const F ave = F(0.5) * (arr[a][ga + l * sz] + arr[a][gb + l * sz]);
        arr[a][ga + l * sz] = ave;
        arr[a][gb + l * sz] = ave;
      }
    return;
  }
  const bool left = it.p <= g;
  const int dst = left ? -it.p : m - 1 + (it.p - g);
  const int src = left ? m - 1 - it.p : it.p - g;
  const idx_t gg = along(z.L, f.face, it.i, it.j, it.k, dst), gs = along(z.L, f.face, it.i, it.j, it.k, src);
  for (int l = 1; l < p.n_var; ++l)
    for (int a = 0; a < 3; ++a) arr[a][gg + l * sz] = arr[a][gs + l * sz];
}

// If periodic face f and the next periodic face in list order are the two faces of one
// direction that can be applied together, return the index of the left one (direction -1),
// else -1.  *next receives the index of the partner.
static int periodic_pair(const Zone &z, const FaceBC *faces, int n, int f, int *next) {
  int q = f + 1;
  while (q < n && faces[q].type != CB2_BC_PERIODIC) ++q;
  if (q >= n) return -1;
  const FaceBC &a = faces[f], &b = faces[q];
  if (a.face != b.face || a.direction == b.direction) return -1;
  const int d = a.face;
  for (int c = 0; c < 3; ++c)
    if (c != d && (a.start[c] != b.start[c] || a.end[c] != b.end[c])) return -1;
  const int m = d == 0 ? z.mx : (d == 1 ? z.my : z.mz);
  if (m < z.ngg + 2) return -1;
  const FaceBC &l = a.direction < 0 ? a : b;
  if (l.start[d] != 0 || l.end[d] != 0) return -1;
  const FaceBC &r = a.direction < 0 ? b : a;
  if (r.start[d] != m - 1 || r.end[d] != m - 1) return -1;
  *next = q;
  return a.direction < 0 ? f : q;
}

// Small CTAs: a face has few nodes, and spreading them over more SMs shortens the launch.
constexpr int kFaceThreads = 64;

template <int NS>
static int launch_bc_ns(const Zone &z, const Param &p, const FaceBC *faces, int n, cudaStream_t s, int &nl) {
  // priority order of the reference
  const int order[6] = {CB2_BC_FARFIELD, CB2_BC_OUTFLOW, CB2_BC_INFLOW, CB2_BC_SYMMETRY, CB2_BC_WALL,
                        CB2_BC_PERIODIC};
  for (int t : order) {
    for (int f = 0; f < n; ++f) {
      if (faces[f].type != t) continue;
      // Two temperatures: face by face, as the reference.  Rebuilding cv syncs e_ve and T_ve
      // (sync_two_temperature_state_from_sv), and the reference's order of those syncs -- the low
      // face's nodes and ghosts first, then the high face averaging with the synced low nodes --
      // decides T_ve wherever e_ve and T_ve disagree on entry (an e_ve left at zero).
      if (t == CB2_BC_PERIODIC && p.i_eve < 0) {
        int q = -1;
        const int lf = periodic_pair(z, faces, n, f, &q);
        if (lf >= 0) {
          const long long np = face_points(faces[lf]) * (2 * z.ngg + 1);
          ProfScope prof("boundary_face", s);
          k_bc_periodic_pair<NS><<<(unsigned)((np + 127) / 128), 128, 0, s>>>(z, p, faces[lf]);
          ++nl;
          CB2_TRY(check_launch());
          f = q;  // the partner is done
          continue;
        }
      }
      const long long np = face_points(faces[f]);
      if (np == 0) continue;
      // threads per face node: one per ghost layer (outflow), one per layer including the face
      // node (inflow, symmetry, wall), one per line (periodic)
      const int layers = t == CB2_BC_OUTFLOW ? z.ngg : (t == CB2_BC_PERIODIC ? 1 : z.ngg + 1);
      const unsigned blocks = (unsigned)((np * layers + kFaceThreads - 1) / kFaceThreads);
      ProfScope prof("boundary_face", s);
      switch (t) {
        case CB2_BC_FARFIELD: k_bc_farfield<NS><<<blocks, kFaceThreads, 0, s>>>(z, p, faces[f]); break;
        case CB2_BC_OUTFLOW: k_bc_outflow<NS><<<blocks, kFaceThreads, 0, s>>>(z, p, faces[f]); break;
        case CB2_BC_INFLOW: k_bc_inflow<NS><<<blocks, kFaceThreads, 0, s>>>(z, p, faces[f]); break;
        case CB2_BC_SYMMETRY: k_bc_symmetry<NS><<<blocks, kFaceThreads, 0, s>>>(z, p, faces[f]); break;
        case CB2_BC_WALL: k_bc_wall<NS><<<blocks, kFaceThreads, 0, s>>>(z, p, faces[f]); break;
        case CB2_BC_PERIODIC: k_bc_periodic<NS><<<blocks, kFaceThreads, 0, s>>>(z, p, faces[f]); break;
      }
      ++nl;
      CB2_TRY(check_launch());
    }
  }
  return CB2_OK;
}

// Non-reflecting outflow (DBoundCond::nonReflectingBoundary -> apply_outflow_nr_conserv,
// src/BoundCond.cu:3580-3845; called after the inviscid flux, src/RK.cuh:190-193): at every node
// of the face, the conservative variables' normal derivative (one-sided, second order, into the
// block) is split into the acoustic, entropy/vorticity and species waves along the unit face
// normal; the waves that travel into the block are dropped (their speeds clipped at zero), and
// the outgoing ones are added back to dq as -J (R Lambda L) dQ/dn.  The wave speeds are
// u.n - c|grad k|, u.n, u.n + c|grad k| with n the unit normal, as the reference takes them.  The
// mixture's gamma = cp / (cp - R) at the node's T; the species rows carry Y_k, and in two
// temperatures the e_ve row takes no correction.  One thread per face node; the face's nodes
// only (the reference also visits the tangential ghost nodes of an extended face, whose writes
// land on other nodes of the ghost-free dq array).
template <int NS>
__global__ void k_outflow_nonreflecting(Zone z, Param p, FaceBC f) {
  const int n0 = f.end[0] - f.start[0] + 1, n1 = f.end[1] - f.start[1] + 1;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n0 * n1 * (f.end[2] - f.start[2] + 1)) return;
  const int i = f.start[0] + (int)(t % n0), j = f.start[1] + (int)((t / n0) % n1),
            k = f.start[2] + (int)(t / ((long long)n0 * n1));
  const idx_t sz = z.L.sz;
  const int sgn = f.direction == -1 ? 1 : -1;  // into the block
  idx_t step;
  if (f.face == 0) step = 1;
  else if (f.face == 1) step = z.L.disp2;
  else step = z.L.disp1;
  step *= sgn;
  const idx_t g = z.L.at(i, j, k);
  // dQ/dn: sgn * (-3/2 Q0 + 2 Q1 - 1/2 Q2), summed in the reference's order
  const double cc[3] = {-1.5, 2.0, -0.5};
  double dQ[5 + NS];
#pragma unroll
  for (int v = 0; v < 5 + NS; ++v) dQ[v] = 0;
#pragma unroll
  for (int l = 0; l <= 2; ++l) {
    const double c = sgn * cc[l];
    const idx_t gl = g + l * step;
#pragma unroll
    for (int v = 0; v < 5 + NS; ++v) dQ[v] += c * z.cv[gl + v * sz];
  }
  const double r = z.bv[g], u = z.bv[g + sz], v = z.bv[g + 2 * sz], w = z.bv[g + 3 * sz], pr = z.bv[g + 4 * sz];
  const double *M = z.metric + (idx_t)(3 * f.face) * sz;
  double kx = M[g], ky = M[g + sz], kz = M[g + 2 * sz];
  const double gki = 1 / norm3d(kx, ky, kz);
  kx *= gki; ky *= gki; kz *= gki;
  const double Uk = u * kx + v * ky + w * kz;
  double gam = kGammaAir;
  double h[NS > 0 ? NS : 1], Y[NS > 0 ? NS : 1];
  const double T = z.bv[g + 5 * sz];
  if constexpr (NS > 0) {
    double cp[NS];
    species_h_cp<NS>(T, p.mech, h, cp);
    double cpm = 0, cvm = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      Y[l] = z.sv[g + l * sz];
      cpm += Y[l] * cp[l];
      cvm += Y[l] * (cp[l] - __ldg(p.mech.gas_const + l));
    }
    gam = cpm / cvm;
  }
  const double c2 = gam * pr / r, c = sqrt(c2), ic2 = 1 / c2, cgk = c / gki;
  double lam0 = Uk - cgk, lam1 = Uk, lam2 = Uk + cgk;
  if (f.direction == -1) {
    lam0 = fmin(lam0, 0.0); lam1 = fmin(lam1, 0.0); lam2 = fmin(lam2, 0.0);
  } else {
    lam0 = fmax(lam0, 0.0); lam1 = fmax(lam1, 0.0); lam2 = fmax(lam2, 0.0);
  }
  const double ek = 0.5 * (u * u + v * v + w * w), gm1 = gam - 1, alpha = gm1 * ek;
  double aY = 0, al[NS > 0 ? NS : 1];
  if constexpr (NS > 0) {
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      al[l] = gam * __ldg(p.mech.gas_const + l) * T - gm1 * h[l];
      aY += al[l] * dQ[5 + l];
    }
  }
  // wave amplitudes
  const double L0 = lam0 * 0.5 * ic2 *
                    ((alpha + Uk * c) * dQ[0] - (gm1 * u + kx * c) * dQ[1] - (gm1 * v + ky * c) * dQ[2] -
                     (gm1 * w + kz * c) * dQ[3] + gm1 * dQ[4] + aY);
  double tk = gm1 * kx;
  const double L1 = lam1 * ic2 *
                    ((kx * (c2 - alpha) - c * (kz * v - ky * w)) * dQ[0] + (tk * u) * dQ[1] + (tk * v + kz * c) * dQ[2] +
                     (tk * w - ky * c) * dQ[3] - tk * dQ[4] - kx * aY);
  tk = gm1 * ky;
  const double L2 = lam1 * ic2 *
                    ((ky * (c2 - alpha) - c * (kx * w - kz * u)) * dQ[0] + (tk * u - kz * c) * dQ[1] + (tk * v) * dQ[2] +
                     (tk * w + kx * c) * dQ[3] - tk * dQ[4] - ky * aY);
  tk = gm1 * kz;
  const double L3 = lam1 * ic2 *
                    ((kz * (c2 - alpha) - c * (ky * u - kx * v)) * dQ[0] + (tk * u + ky * c) * dQ[1] +
                     (tk * v - kx * c) * dQ[2] + (tk * w) * dQ[3] - tk * dQ[4] - kz * aY);
  const double L4 = lam2 * 0.5 * ic2 *
                    ((alpha - Uk * c) * dQ[0] - (gm1 * u - kx * c) * dQ[1] - (gm1 * v - ky * c) * dQ[2] -
                     (gm1 * w - kz * c) * dQ[3] + gm1 * dQ[4] + aY);
  // back to conservative increments
  const double hh = (z.cv[g + 4 * sz] + pr) / r, igm1 = 1 / gm1;
  const double sum = L0 + kx * L1 + ky * L2 + kz * L3 + L4;
  double d[5];
  d[0] = sum;
  d[1] = u * sum + c * (kx * (L4 - L0) - kz * L2 + ky * L3);
  d[2] = v * sum + c * (ky * (L4 - L0) + kz * L1 - kx * L3);
  d[3] = w * sum + c * (kz * (L4 - L0) - ky * L1 + kx * L2);
  d[4] = hh * sum + c * (Uk * (L4 - L0) + (kz * v - ky * w - kx * c * igm1) * L1 +
                         (kx * w - kz * u - ky * c * igm1) * L2 + (ky * u - kx * v - kz * c * igm1) * L3);
  const double mj = -z.jac[g];
  const idx_t g0 = z.L0.at(i, j, k), sz0 = z.L0.sz;
  if constexpr (NS > 0) {
    double add = 0;
#pragma unroll
    for (int l = 0; l < NS; ++l) {
      const double Ls = lam1 * (dQ[5 + l] - Y[l] * dQ[0]);
      z.dq[g0 + (5 + l) * sz0] += mj * (Ls + Y[l] * sum);
      add += al[l] * Ls;
    }
    d[4] -= add * igm1;
  }
#pragma unroll
  for (int l = 0; l < 5; ++l) z.dq[g0 + l * sz0] += mj * d[l];
}

template <int NS>
static int launch_nr_ns(const Zone &z, const Param &p, const FaceBC *faces, int n_faces, cudaStream_t s, int &nl) {
  const int ext[3] = {z.mx, z.my, z.mz};
  for (int fi = 0; fi < n_faces; ++fi) {
    if (!faces[fi].nonreflecting) continue;
    FaceBC f = faces[fi];
    for (int a = 0; a < 3; ++a) {  // the face's own nodes
      if (a == f.face) continue;
      f.start[a] = max(f.start[a], 0);
      f.end[a] = min(f.end[a], ext[a] - 1);
    }
    const long long n = (long long)max(f.end[0] - f.start[0] + 1, 0) * max(f.end[1] - f.start[1] + 1, 0) *
                        max(f.end[2] - f.start[2] + 1, 0);
    if (n == 0) continue;
    ProfScope prof("outflow_nonreflecting", s);
    k_outflow_nonreflecting<NS><<<(unsigned)((n + 127) / 128), 128, 0, s>>>(z, p, f);
    ++nl;
    CB2_TRY(check_launch());
  }
  return CB2_OK;
}

int launch_nonreflecting(const Zone &z, const Param &p, const FaceBC *faces, int n_faces, cudaStream_t s,
                         int &n_launch) {
  switch (p.n_spec) {
    case 0: return launch_nr_ns<0>(z, p, faces, n_faces, s, n_launch);
    case 5: return launch_nr_ns<5>(z, p, faces, n_faces, s, n_launch);
    case 9: return launch_nr_ns<9>(z, p, faces, n_faces, s, n_launch);
    default: return CB2_ERR_UNSUPPORTED;
  }
}

int launch_eliminate_k_gradient(const Zone &z, const Param &p, cudaStream_t s, int &nl) {
  const int g = z.ngg;
  dim3 grid((z.mx + 2 * g + 127) / 128, z.my + 2 * g, 1);
  ProfScope prof("eliminate_k_gradient", s);
  k_eliminate_k_gradient<<<grid, 128, 0, s>>>(z, p);
  ++nl;
  return check_launch();
}

int launch_boundary(const Zone &z, const Param &p, const FaceBC *faces, int n_faces, cudaStream_t s,
                    int &n_launch) {
  switch (p.n_spec) {
    case 0: return launch_bc_ns<0>(z, p, faces, n_faces, s, n_launch);
    case 5: return launch_bc_ns<5>(z, p, faces, n_faces, s, n_launch);
    case 9: return launch_bc_ns<9>(z, p, faces, n_faces, s, n_launch);
    default: return CB2_ERR_UNSUPPORTED;
  }
}

int launch_periodic_flux_exchange(const Zone &z, const Param &p, const FaceBC *faces, int n_faces, cudaStream_t s,
                                  int &n_launch) {
  for (int f = 0; f < n_faces; ++f) {
    if (faces[f].type != CB2_BC_PERIODIC) continue;
    int q = -1;
    const int lf = periodic_pair(z, faces, n_faces, f, &q);
    if (lf >= 0) {
      const long long np = face_points(faces[lf]) * (2 * z.ngg + 1);
      ProfScope prof("periodic_flux_exchange", s);
      if (visc8_f32(p))
        k_periodic_flux_pair<float><<<(unsigned)((np + 127) / 128), 128, 0, s>>>(z, p, faces[lf]);
      else
        k_periodic_flux_pair<double><<<(unsigned)((np + 127) / 128), 128, 0, s>>>(z, p, faces[lf]);
      ++n_launch;
      CB2_TRY(check_launch());
      f = q;
      continue;
    }
    const long long np = face_points(faces[f]);
    const unsigned blocks = (unsigned)((np + 127) / 128);
    if (!blocks) continue;
    ProfScope prof("periodic_flux_exchange", s);
    if (visc8_f32(p)) k_periodic_flux<float><<<blocks, 128, 0, s>>>(z, p, faces[f]);
    else k_periodic_flux<double><<<blocks, 128, 0, s>>>(z, p, faces[f]);
    ++n_launch;
    CB2_TRY(check_launch());
  }
  return CB2_OK;
}

}  // namespace cb2
