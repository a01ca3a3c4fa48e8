// Viscous fluxes.
//
// Order 8 (compute_viscous_flux_collocated<mix,8>, src/ViscousScheme.cu:470-585;
// compute_viscous_flux_derivative<8>, :790-834; stencils d_dXi/d_dEta/d_dZeta, :140-468):
//   node gradients of u,v,w,T with 8th-order central differences (one-sided closures on the
//   four nodes next to a physical boundary), collocated node fluxes into fFlux/gFlux/hFlux,
//   periodic exchange of the node fluxes, then dq += J (dF/dxi + dG/deta + dH/dzeta).
// Order 2 (compute_{fv,gv,hv}_2nd_order, src/ViscousScheme.cu:836-1512; compute_dFv_dx etc.,
//   :86-138): face fluxes from face-averaged metrics/coefficients and compact differences,
//   mixture species diffusion with the correction velocity and the h_k J_k energy term;
//   the face difference is taken in the same kernel as the face flux through shared memory.
#include <type_traits>
#include "common.cuh"
#include "thermo.cuh"
#include "thermo_2t.cuh"
#include "launch.h"
#include "stencil8.cuh"

namespace cb2 {

// 8th-order node fluxes: one thread per node, CTAs of kVisTI (i) x kVisTJ (j) nodes of one
// k-plane, so the j-neighbours of a stencil are mostly lines the same CTA brought into L1.
constexpr int kVisTI = 32, kVisTJ = 8, kVisThreads = kVisTI * kVisTJ;

// Node fluxes of the momentum and energy equations (air); comps 1..4 of fFlux/gFlux/hFlux.
// T is the arithmetic type (double: plain form; float: mixed form, FP64 arrays read and
// written, the stencils, stresses and fluxes evaluated in FP32).
template <typename T>
__device__ __forceinline__ void visc8_node_flux_air(const Zone &z, const Param &p) {
  const int i = blockIdx.x * kVisTI + threadIdx.x, j = blockIdx.y * kVisTJ + threadIdx.y, k = blockIdx.z;
  if (i >= z.mx || j >= z.my) return;
  const Layout &L = z.L;
  const idx_t sz = L.sz, g = L.at(i, j, k);
  const BFlags b = bflags(z, i, j, k);
  const idx_t si = 1, sj = L.disp2, sk = L.disp1;
  // the mixed form reads the FP32 copies of bv, the metric and J
  using Src = std::conditional_t<sizeof(T) == 4, const float *, const double *>;
  Src BV, M;
  if constexpr (sizeof(T) == 4) {
    BV = z.bv32;
    M = z.met32 + g;
  } else {
    BV = z.bv;
    M = z.metric + g;
  }
  auto der = [&](int comp, T &dxi, T &deta, T &dzeta) {
    const Src f = BV + comp * sz + g;
    dxi = d8<T>([&](int m) { return T(f[m * si]); }, i, z.mx, b.il, b.ir);
    deta = d8<T>([&](int m) { return T(f[m * sj]); }, j, z.my, b.jl, b.jr);
    dzeta = d8<T>([&](int m) { return T(f[m * sk]); }, k, z.mz, b.kl, b.kr);
  };
  T u_xi, u_eta, u_zeta, v_xi, v_eta, v_zeta, w_xi, w_eta, w_zeta, t_xi, t_eta, t_zeta;
  der(1, u_xi, u_eta, u_zeta);
  der(2, v_xi, v_eta, v_zeta);
  der(3, w_xi, w_eta, w_zeta);
  der(5, t_xi, t_eta, t_zeta);
  const T xi_x = T(M[0]), xi_y = T(M[sz]), xi_z = T(M[2 * sz]);
  const T eta_x = T(M[3 * sz]), eta_y = T(M[4 * sz]), eta_z = T(M[5 * sz]);
  const T zeta_x = T(M[6 * sz]), zeta_y = T(M[7 * sz]), zeta_z = T(M[8 * sz]);
  const T u_x = u_xi * xi_x + u_eta * eta_x + u_zeta * zeta_x;
  const T u_y = u_xi * xi_y + u_eta * eta_y + u_zeta * zeta_y;
  const T u_z = u_xi * xi_z + u_eta * eta_z + u_zeta * zeta_z;
  const T v_x = v_xi * xi_x + v_eta * eta_x + v_zeta * zeta_x;
  const T v_y = v_xi * xi_y + v_eta * eta_y + v_zeta * zeta_y;
  const T v_z = v_xi * xi_z + v_eta * eta_z + v_zeta * zeta_z;
  const T w_x = w_xi * xi_x + w_eta * eta_x + w_zeta * zeta_x;
  const T w_y = w_xi * xi_y + w_eta * eta_y + w_zeta * zeta_y;
  const T w_z = w_xi * xi_z + w_eta * eta_z + w_zeta * zeta_z;
  const T mu = T(z.mul[g]);
  const T txx = mu * (4 * u_x - 2 * v_y - 2 * w_z) / 3;
  const T tyy = mu * (4 * v_y - 2 * u_x - 2 * w_z) / 3;
  const T tzz = mu * (4 * w_z - 2 * u_x - 2 * v_y) / 3;
  const T txy = mu * (u_y + v_x), txz = mu * (u_z + w_x), tyz = mu * (v_z + w_y);
  const T t_x = t_xi * xi_x + t_eta * eta_x + t_zeta * zeta_x;
  const T t_y = t_xi * xi_y + t_eta * eta_y + t_zeta * zeta_y;
  const T t_z = t_xi * xi_z + t_eta * eta_z + t_zeta * zeta_z;
  const T cp = T(kGammaAir * kRAir / (kGammaAir - 1));
  const T kap = mu / T(p.Pr) * cp;
  const T u = T(BV[g + sz]), v = T(BV[g + 2 * sz]), w = T(BV[g + 3 * sz]);
  const T Ex = u * txx + v * txy + w * txz + kap * t_x;
  const T Ey = u * txy + v * tyy + w * tyz + kap * t_y;
  const T Ez = u * txz + v * tyz + w * tzz + kap * t_z;
  // node fluxes: the caller's FP64 arrays, or the FP32 copies the mixed form's divergence reads
  T *FF, *GF, *HF;
  if constexpr (sizeof(T) == 4) {
    FF = z.fF32; GF = z.gF32; HF = z.hF32;
  } else {
    FF = z.fF; GF = z.gF; HF = z.hF;
  }
  FF[g + sz] = xi_x * txx + xi_y * txy + xi_z * txz;
  FF[g + 2 * sz] = xi_x * txy + xi_y * tyy + xi_z * tyz;
  FF[g + 3 * sz] = xi_x * txz + xi_y * tyz + xi_z * tzz;
  GF[g + sz] = eta_x * txx + eta_y * txy + eta_z * txz;
  GF[g + 2 * sz] = eta_x * txy + eta_y * tyy + eta_z * tyz;
  GF[g + 3 * sz] = eta_x * txz + eta_y * tyz + eta_z * tzz;
  HF[g + sz] = zeta_x * txx + zeta_y * txy + zeta_z * txz;
  HF[g + 2 * sz] = zeta_x * txy + zeta_y * tyy + zeta_z * tyz;
  HF[g + 3 * sz] = zeta_x * txz + zeta_y * tyz + zeta_z * tzz;
  FF[g + 4 * sz] = xi_x * Ex + xi_y * Ey + xi_z * Ez;
  GF[g + 4 * sz] = eta_x * Ex + eta_y * Ey + eta_z * Ez;
  HF[g + 4 * sz] = zeta_x * Ex + zeta_y * Ey + zeta_z * Ez;
}

__global__ void __launch_bounds__(kVisThreads) k_visc8_node_flux_air_f64(Zone z, Param p) {
  visc8_node_flux_air<double>(z, p);
}
// bounded to 64 registers: four CTAs of 256 threads per SM
__global__ void __launch_bounds__(kVisThreads, 4) k_visc8_node_flux_air_f32(Zone z, Param p) {
  visc8_node_flux_air<float>(z, p);
}

// Node fluxes of a thermally perfect mixture (compute_viscous_flux_collocated<Mixture,8> followed
// by compute_viscous_flux_collocated_scalar<8>, src/ViscousScheme.cu:470-788), FP64: the stresses
// and the conduction kappa grad T as for air (kappa from the property kernel), in two temperatures
// kappa_ve grad T_ve added to the energy flux, then per species the mixture-averaged diffusion flux
// J_k = rho D_k (grad Y_k - Y_k W grad(1/W)-term [+ the pressure term]) - Y_k V_c with the
// correction velocity V_c, its enthalpy h_k J_k (two temperatures: h_k with e_ve at T_ve) added to
// the energy flux, and in two temperatures the e_ve flux kappa_ve grad T_ve + sum e_ve,k J_k.
// Every flux is projected on the node's grad xi / grad eta / grad zeta, as the reference stores
// them; additions into the energy flux follow the reference's order (the collocated kernel's
// stresses and conduction, then species by species).
template <int NS, bool TT>
__global__ void __launch_bounds__(kVisThreads) k_visc8_node_flux_mix(Zone z, Param p) {
  const int i = blockIdx.x * kVisTI + threadIdx.x, j = blockIdx.y * kVisTJ + threadIdx.y, k = blockIdx.z;
  if (i >= z.mx || j >= z.my) return;
  const Layout &L = z.L;
  const idx_t sz = L.sz, g = L.at(i, j, k);
  const BFlags b = bflags(z, i, j, k);
  const idx_t si = 1, sj = L.disp2, sk = L.disp1;
  const double *M = z.metric + g;
  auto der = [&](const double *f0, double &dxi, double &deta, double &dzeta) {
    const double *f = f0 + g;
    dxi = d8<double>([&](int m) { return f[m * si]; }, i, z.mx, b.il, b.ir);
    deta = d8<double>([&](int m) { return f[m * sj]; }, j, z.my, b.jl, b.jr);
    dzeta = d8<double>([&](int m) { return f[m * sk]; }, k, z.mz, b.kl, b.kr);
  };
  const double xi_x = M[0], xi_y = M[sz], xi_z = M[2 * sz];
  const double eta_x = M[3 * sz], eta_y = M[4 * sz], eta_z = M[5 * sz];
  const double zeta_x = M[6 * sz], zeta_y = M[7 * sz], zeta_z = M[8 * sz];
  double *FF = z.fF, *GF = z.gF, *HF = z.hF;
  double F4, G4, H4;
  {
    double u_xi, u_eta, u_zeta, v_xi, v_eta, v_zeta, w_xi, w_eta, w_zeta, t_xi, t_eta, t_zeta;
    der(z.bv + sz, u_xi, u_eta, u_zeta);
    der(z.bv + 2 * sz, v_xi, v_eta, v_zeta);
    der(z.bv + 3 * sz, w_xi, w_eta, w_zeta);
    der(z.bv + 5 * sz, t_xi, t_eta, t_zeta);
    const double u_x = u_xi * xi_x + u_eta * eta_x + u_zeta * zeta_x;
    const double u_y = u_xi * xi_y + u_eta * eta_y + u_zeta * zeta_y;
    const double u_z = u_xi * xi_z + u_eta * eta_z + u_zeta * zeta_z;
    const double v_x = v_xi * xi_x + v_eta * eta_x + v_zeta * zeta_x;
    const double v_y = v_xi * xi_y + v_eta * eta_y + v_zeta * zeta_y;
    const double v_z = v_xi * xi_z + v_eta * eta_z + v_zeta * zeta_z;
    const double w_x = w_xi * xi_x + w_eta * eta_x + w_zeta * zeta_x;
    const double w_y = w_xi * xi_y + w_eta * eta_y + w_zeta * zeta_y;
    const double w_z = w_xi * xi_z + w_eta * eta_z + w_zeta * zeta_z;
    const double mu = z.mul[g];
    const double txx = mu * (4 * u_x - 2 * v_y - 2 * w_z) / 3.0;
    const double tyy = mu * (4 * v_y - 2 * u_x - 2 * w_z) / 3.0;
    const double tzz = mu * (4 * w_z - 2 * u_x - 2 * v_y) / 3.0;
    const double txy = mu * (u_y + v_x), txz = mu * (u_z + w_x), tyz = mu * (v_z + w_y);
    FF[g + sz] = xi_x * txx + xi_y * txy + xi_z * txz;
    FF[g + 2 * sz] = xi_x * txy + xi_y * tyy + xi_z * tyz;
    FF[g + 3 * sz] = xi_x * txz + xi_y * tyz + xi_z * tzz;
    GF[g + sz] = eta_x * txx + eta_y * txy + eta_z * txz;
    GF[g + 2 * sz] = eta_x * txy + eta_y * tyy + eta_z * tyz;
    GF[g + 3 * sz] = eta_x * txz + eta_y * tyz + eta_z * tzz;
    HF[g + sz] = zeta_x * txx + zeta_y * txy + zeta_z * txz;
    HF[g + 2 * sz] = zeta_x * txy + zeta_y * tyy + zeta_z * tyz;
    HF[g + 3 * sz] = zeta_x * txz + zeta_y * tyz + zeta_z * tzz;
    const double t_x = t_xi * xi_x + t_eta * eta_x + t_zeta * zeta_x;
    const double t_y = t_xi * xi_y + t_eta * eta_y + t_zeta * zeta_y;
    const double t_z = t_xi * xi_z + t_eta * eta_z + t_zeta * zeta_z;
    const double kap = z.kappa[g];
    const double u = z.bv[g + sz], v = z.bv[g + 2 * sz], w = z.bv[g + 3 * sz];
    const double Ex = u * txx + v * txy + w * txz + kap * t_x;
    const double Ey = u * txy + v * tyy + w * tyz + kap * t_y;
    const double Ez = u * txz + v * tyz + w * tzz + kap * t_z;
    F4 = xi_x * Ex + xi_y * Ey + xi_z * Ez;
    G4 = eta_x * Ex + eta_y * Ey + eta_z * Ez;
    H4 = zeta_x * Ex + zeta_y * Ey + zeta_z * Ez;
  }
  double efx = 0, efy = 0, efz = 0;
  if constexpr (TT) {
    double v_xi, v_eta, v_zeta;
    der(z.tve, v_xi, v_eta, v_zeta);
    const double v_x = v_xi * xi_x + v_eta * eta_x + v_zeta * zeta_x;
    const double v_y = v_xi * xi_y + v_eta * eta_y + v_zeta * zeta_y;
    const double v_z = v_xi * xi_z + v_eta * eta_z + v_zeta * zeta_z;
    const double kve = z.kappa_ve[g];
    efx = kve * (xi_x * v_x + xi_y * v_y + xi_z * v_z);
    efy = kve * (eta_x * v_x + eta_y * v_y + eta_z * v_z);
    efz = kve * (zeta_x * v_x + zeta_y * v_y + zeta_z * v_z);
    F4 += efx;
    G4 += efy;
    H4 += efz;
  }
  // species diffusion (the scalar kernel)
  const Mech &m = p.mech;
  double dif[NS], yk[NS], fx[NS], fy[NS], fz[NS];
  double swx = 0, swy = 0, swz = 0, cx = 0, cy = 0, cz = 0, mwt = 0, srdy = 0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    yk[s] = z.sv[g + s * sz];
    dif[s] = z.rhoD[g + s * sz];
    double y_xi, y_eta, y_zeta;
    der(z.sv + s * sz, y_xi, y_eta, y_zeta);
    const double y_x = y_xi * xi_x + y_eta * eta_x + y_zeta * zeta_x;
    const double y_y = y_xi * xi_y + y_eta * eta_y + y_zeta * zeta_y;
    const double y_z = y_xi * xi_z + y_eta * eta_z + y_zeta * zeta_z;
    fx[s] = xi_x * y_x + xi_y * y_y + xi_z * y_z;
    fy[s] = eta_x * y_x + eta_y * y_y + eta_z * y_z;
    fz[s] = zeta_x * y_x + zeta_y * y_y + zeta_z * y_z;
    cx += dif[s] * fx[s];
    cy += dif[s] * fy[s];
    cz += dif[s] * fz[s];
    const double iw = __ldg(m.imw + s);
    swx += fx[s] * iw;
    swy += fy[s] * iw;
    swz += fz[s] * iw;
    mwt += yk[s] * iw;
    srdy += dif[s] * yk[s];
  }
  mwt = 1.0 / mwt;
  cx -= mwt * srdy * swx;
  cy -= mwt * srdy * swy;
  cz -= mwt * srdy * swz;
  if (p.gradP) {
    double p_xi, p_eta, p_zeta;
    der(z.bv + 4 * sz, p_xi, p_eta, p_zeta);
    const double p_x = p_xi * xi_x + p_eta * eta_x + p_zeta * zeta_x;
    const double p_y = p_xi * xi_y + p_eta * eta_y + p_zeta * zeta_y;
    const double p_z = p_xi * xi_z + p_eta * eta_z + p_zeta * zeta_z;
    const double pg = z.bv[g + 4 * sz];
    const double gpx = (xi_x * p_x + xi_y * p_y + xi_z * p_z) / pg;
    const double gpy = (eta_x * p_x + eta_y * p_y + eta_z * p_z) / pg;
    const double gpz = (zeta_x * p_x + zeta_y * p_y + zeta_z * p_z) / pg;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double co = (mwt * __ldg(m.imw + s) - 1) * yk[s];
      fx[s] += co * gpx;
      fy[s] += co * gpy;
      fz[s] += co * gpz;
      cx += co * gpx * dif[s];
      cy += co * gpy * dif[s];
      cz += co * gpz * dif[s];
    }
  }
  double h[NS];
  const double tm = z.bv[g + 5 * sz];
  species_h<NS>(tm, m, h);
  const double tve_m = TT ? z.tve[g] : tm;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    double hd = h[s], ev = 0;
    if constexpr (TT) {
      hd = h[s] - ve_energy(s, tm, m, nullptr) + ve_energy(s, tve_m, m, nullptr);
      ev = ve_energy(s, tve_m, m, nullptr);
    }
    double jd = dif[s] * (fx[s] - mwt * yk[s] * swx) - yk[s] * cx;
    FF[g + (5 + s) * sz] = jd;
    F4 += hd * jd;
    if constexpr (TT) efx += ev * jd;
    jd = dif[s] * (fy[s] - mwt * yk[s] * swy) - yk[s] * cy;
    GF[g + (5 + s) * sz] = jd;
    G4 += hd * jd;
    if constexpr (TT) efy += ev * jd;
    jd = dif[s] * (fz[s] - mwt * yk[s] * swz) - yk[s] * cz;
    HF[g + (5 + s) * sz] = jd;
    H4 += hd * jd;
    if constexpr (TT) efz += ev * jd;
  }
  FF[g + 4 * sz] = F4;
  GF[g + 4 * sz] = G4;
  HF[g + 4 * sz] = H4;
  if constexpr (TT) {
    FF[g + (5 + NS) * sz] = efx;
    GF[g + (5 + NS) * sz] = efy;
    HF[g + (5 + NS) * sz] = efz;
  }
}

// The divergence reads each flux array along one direction only; rows of kVisRow i-nodes
// measured faster than 2-D tiles for it.
constexpr int kVisRow = 128;

// ASSIGN: the divergence is the first term of the residual, so it writes dq (the mass row
// gets zero) instead of adding to a zeroed dq.
template <typename T, bool ASSIGN>
__device__ __forceinline__ void visc8_divergence_row(const Zone &z, const Param &p) {
  const int i = blockIdx.x * kVisRow + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= z.mx) return;
  const Layout &L = z.L;
  const idx_t sz = L.sz, g = L.at(i, j, k);
  const BFlags b = bflags(z, i, j, k);
  const idx_t sj = L.disp2, sk = L.disp1;
  const T jac = T(z.jac[g]);
  const idx_t g0 = z.L0.at(i, j, k), sz0 = z.L0.sz;
  if (ASSIGN) z.dq[g0] = 0.0;
  using Src = std::conditional_t<sizeof(T) == 4, const float *, const double *>;
  Src F0, G0, H0;
  if constexpr (sizeof(T) == 4) {
    F0 = z.fF32; G0 = z.gF32; H0 = z.hF32;
  } else {
    F0 = z.fF; G0 = z.gF; H0 = z.hF;
  }
#pragma unroll 1
  for (int l = 1; l < p.n_var; ++l) {
    const Src f = F0 + l * sz + g, gg = G0 + l * sz + g, h = H0 + l * sz + g;
    const T d = d8<T>([&](int m) { return T(f[m]); }, i, z.mx, b.il, b.ir) +
                d8<T>([&](int m) { return T(gg[m * sj]); }, j, z.my, b.jl, b.jr) +
                d8<T>([&](int m) { return T(h[m * sk]); }, k, z.mz, b.kl, b.kr);
    if (ASSIGN) z.dq[g0 + l * sz0] = double(d * jac);
    else z.dq[g0 + l * sz0] += double(d * jac);
  }
}

// Both sums fit in 32 registers (16 rows of 128 threads per SM); the FP32 one needs the bound.
template <bool ASSIGN>
__global__ void __launch_bounds__(kVisRow) k_visc8_divergence_f64(Zone z, Param p) {
  visc8_divergence_row<double, ASSIGN>(z, p);
}
template <bool ASSIGN>
__global__ void __launch_bounds__(kVisRow, 16) k_visc8_divergence_f32(Zone z, Param p) {
  visc8_divergence_row<float, ASSIGN>(z, p);
}

// ---- 2nd-order face fluxes ----------------------------------------------------------------
// Face between node (i,j,k) and its +1 neighbour along DIR.  The compact difference is taken
// along DIR and the two transverse derivatives are averaged over the two nodes (4-point).
template <int NS, int DIR, bool TT = false>
__device__ __forceinline__ void visc2_face(const Zone &z, const Param &p, int i, int j, int k, double *fv) {
  const Layout &L = z.L;
  const idx_t sz = L.sz;
  const idx_t st[3] = {1, L.disp2, L.disp1};
  const idx_t g = L.at(i, j, k), gn = g + st[DIR];
  const double *M = z.metric;
  double mtr[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) mtr[c] = 0.5 * (M[g + c * sz] + M[gn + c * sz]);
  // derivatives of a field along xi, eta, zeta at the face
  auto grad = [&](const double *f, double &dxi, double &deta, double &dzeta) {
    double d[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (a == DIR) d[a] = f[gn] - f[g];
      else d[a] = 0.25 * (f[g + st[a]] - f[g - st[a]] + f[gn + st[a]] - f[gn - st[a]]);
    }
    dxi = d[0]; deta = d[1]; dzeta = d[2];
  };
  double u_xi, u_eta, u_zeta, v_xi, v_eta, v_zeta, w_xi, w_eta, w_zeta, t_xi, t_eta, t_zeta;
  grad(z.bv + sz, u_xi, u_eta, u_zeta);
  grad(z.bv + 2 * sz, v_xi, v_eta, v_zeta);
  grad(z.bv + 3 * sz, w_xi, w_eta, w_zeta);
  grad(z.bv + 5 * sz, t_xi, t_eta, t_zeta);
  const double xi_x = mtr[0], xi_y = mtr[1], xi_z = mtr[2], eta_x = mtr[3], eta_y = mtr[4], eta_z = mtr[5];
  const double zeta_x = mtr[6], zeta_y = mtr[7], zeta_z = mtr[8];
  const double u_x = u_xi * xi_x + u_eta * eta_x + u_zeta * zeta_x;
  const double u_y = u_xi * xi_y + u_eta * eta_y + u_zeta * zeta_y;
  const double u_z = u_xi * xi_z + u_eta * eta_z + u_zeta * zeta_z;
  const double v_x = v_xi * xi_x + v_eta * eta_x + v_zeta * zeta_x;
  const double v_y = v_xi * xi_y + v_eta * eta_y + v_zeta * zeta_y;
  const double v_z = v_xi * xi_z + v_eta * eta_z + v_zeta * zeta_z;
  const double w_x = w_xi * xi_x + w_eta * eta_x + w_zeta * zeta_x;
  const double w_y = w_xi * xi_y + w_eta * eta_y + w_zeta * zeta_y;
  const double w_z = w_xi * xi_z + w_eta * eta_z + w_zeta * zeta_z;
  const double mu = 0.5 * (z.mul[g] + z.mul[gn]);
  const double txx = mu * (4 * u_x - 2 * v_y - 2 * w_z) / 3.0;
  const double tyy = mu * (4 * v_y - 2 * u_x - 2 * w_z) / 3.0;
  const double tzz = mu * (4 * w_z - 2 * u_x - 2 * v_y) / 3.0;
  const double txy = mu * (u_y + v_x), txz = mu * (u_z + w_x), tyz = mu * (v_z + w_y);
  const double *Md = M + (idx_t)(3 * DIR) * sz;
  const double jl = z.jac[g], jr = z.jac[gn];
  const double kxj = 0.5 * (Md[g] * jl + Md[gn] * jr);
  const double kyj = 0.5 * (Md[g + sz] * jl + Md[gn + sz] * jr);
  const double kzj = 0.5 * (Md[g + 2 * sz] * jl + Md[gn + 2 * sz] * jr);
  fv[0] = kxj * txx + kyj * txy + kzj * txz;
  fv[1] = kxj * txy + kyj * tyy + kzj * tyz;
  fv[2] = kxj * txz + kyj * tyz + kzj * tzz;
  const double um = 0.5 * (z.bv[g + sz] + z.bv[gn + sz]);
  const double vm = 0.5 * (z.bv[g + 2 * sz] + z.bv[gn + 2 * sz]);
  const double wm = 0.5 * (z.bv[g + 3 * sz] + z.bv[gn + 3 * sz]);
  const double t_x = t_xi * xi_x + t_eta * eta_x + t_zeta * zeta_x;
  const double t_y = t_xi * xi_y + t_eta * eta_y + t_zeta * zeta_y;
  const double t_z = t_xi * xi_z + t_eta * eta_z + t_zeta * zeta_z;
  double kap;
  if constexpr (NS == 0) {
    const double cp = kGammaAir * kRAir / (kGammaAir - 1);
    kap = mu / p.Pr * cp;
  } else {
    kap = 0.5 * (z.kappa[g] + z.kappa[gn]);
  }
  fv[3] = um * fv[0] + vm * fv[1] + wm * fv[2] + kap * (kxj * t_x + kyj * t_y + kzj * t_z);
  if constexpr (NS > 0) {
    const Mech &m = p.mech;
    double dif[NS], yk[NS], force[NS];
    double sum_gy_w = 0, sum_rdy = 0, corr = 0, mwt = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double *ys = z.sv + s * sz;
      yk[s] = 0.5 * (ys[g] + ys[gn]);
      dif[s] = 0.5 * (z.rhoD[g + s * sz] + z.rhoD[gn + s * sz]);
      double y_xi, y_eta, y_zeta;
      grad(ys, y_xi, y_eta, y_zeta);
      const double y_x = y_xi * xi_x + y_eta * eta_x + y_zeta * zeta_x;
      const double y_y = y_xi * xi_y + y_eta * eta_y + y_zeta * zeta_y;
      const double y_z = y_xi * xi_z + y_eta * eta_z + y_zeta * zeta_z;
      const double gdy = kxj * y_x + kyj * y_y + kzj * y_z;
      force[s] = gdy;
      corr += dif[s] * gdy;
      sum_gy_w += gdy * __ldg(m.imw + s);
      mwt += yk[s] * __ldg(m.imw + s);
      sum_rdy += dif[s] * yk[s];
    }
    mwt = 1.0 / mwt;
    corr -= mwt * sum_rdy * sum_gy_w;
    if (p.gradP) {
      double p_xi, p_eta, p_zeta;
      grad(z.bv + 4 * sz, p_xi, p_eta, p_zeta);
      const double p_x = p_xi * xi_x + p_eta * eta_x + p_zeta * zeta_x;
      const double p_y = p_xi * xi_y + p_eta * eta_y + p_zeta * zeta_y;
      const double p_z = p_xi * xi_z + p_eta * eta_z + p_zeta * zeta_z;
      const double gp = (kxj * p_x + kyj * p_y + kzj * p_z) / (0.5 * (z.bv[gn + 4 * sz] + z.bv[g + 4 * sz]));
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        force[s] += (mwt * __ldg(m.imw + s) - 1) * yk[s] * gp;
        corr += (mwt * __ldg(m.imw + s) - 1) * yk[s] * gp * dif[s];
      }
    }
    double h[NS];
    const double tm = 0.5 * (z.bv[g + 5 * sz] + z.bv[gn + 5 * sz]);
    species_h<NS>(tm, m, h);
    const double tve_m = TT ? 0.5 * (z.tve[g] + z.tve[gn]) : tm;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const double jd = dif[s] * (force[s] - mwt * yk[s] * sum_gy_w) - yk[s] * corr;
      fv[4 + s] = jd;
      // two-temperature: the diffusing enthalpy carries e_ve at T_ve
      // (compute_nonequilibrium_diffusion_enthalpy, src/Thermo.cuh:43-47)
      const double hd = TT ? h[s] - ve_energy(s, tm, m, nullptr) + ve_energy(s, tve_m, m, nullptr) : h[s];
      fv[3] += hd * jd;
    }
    if constexpr (TT) {
      // e_ve conduction kappa_ve grad T_ve in the energy flux, and the e_ve flux
      // (src/ViscousScheme.cu:1024-1039)
      double v_xi, v_eta, v_zeta;
      grad(z.tve, v_xi, v_eta, v_zeta);
      const double v_x = v_xi * xi_x + v_eta * eta_x + v_zeta * zeta_x;
      const double v_y = v_xi * xi_y + v_eta * eta_y + v_zeta * zeta_y;
      const double v_z = v_xi * xi_z + v_eta * eta_z + v_zeta * zeta_z;
      const double kve = 0.5 * (z.kappa_ve[g] + z.kappa_ve[gn]);
      const double cond_ve = kve * (kxj * v_x + kyj * v_y + kzj * v_z);
      fv[3] += cond_ve;
      double ef = cond_ve;
#pragma unroll
      for (int s = 0; s < NS; ++s) ef += ve_energy(s, tve_m, m, nullptr) * fv[4 + s];
      fv[4 + NS] = ef;
    }
  }
}

constexpr int kV2TI = 16, kV2TS = 16;  // tile of 16 transverse x 16 faces along the direction

// Face fluxes of a tile and their difference: a CTA owns kV2TS faces along DIR (the first
// one is the left face of the first node) for kV2TI positions of the transverse index.  The
// thread index runs fastest along i in every direction (along the faces for x, along the
// transverse index for y/z), so a warp's loads are contiguous.
template <int NS, int DIR, bool TT = false>
__device__ __forceinline__ void visc2_tile(const Zone &z, const Param &p) {
  constexpr int NF = 4 + NS + (TT ? 1 : 0);
  constexpr int kPrev = DIR == 0 ? 1 : kV2TI;  // thread of the previous face along DIR
  __shared__ double sfv[NF][kV2TI * kV2TS];
  const int tid = threadIdx.x;
  const int tt = DIR == 0 ? tid / kV2TS : tid % kV2TI, ts = DIR == 0 ? tid % kV2TS : tid / kV2TI;
  int i, j, k, n;
  const int s0 = blockIdx.y * (kV2TS - 1);
  n = s0 - 1 + ts;  // face n + 1/2 along DIR
  if (DIR == 0) { i = n; j = blockIdx.x * kV2TI + tt; k = blockIdx.z; }
  else if (DIR == 1) { i = blockIdx.x * kV2TI + tt; j = n; k = blockIdx.z; }
  else { i = blockIdx.x * kV2TI + tt; j = blockIdx.z; k = n; }
  const int ext[3] = {z.mx, z.my, z.mz};
  const int tr = DIR == 0 ? j : i;
  const int trmax = DIR == 0 ? z.my : z.mx;
  const bool valid = tr < trmax && n <= ext[DIR] - 1;
  if (valid) {
    double fv[NF];
    visc2_face<NS, DIR, TT>(z, p, i, j, k, fv);
#pragma unroll
    for (int c = 0; c < NF; ++c) sfv[c][tid] = fv[c];
  }
  __syncthreads();
  if (valid && ts >= 1 && n >= 0) {
    const idx_t g0 = z.L0.at(i, j, k), sz0 = z.L0.sz;
#pragma unroll
    for (int c = 0; c < NF; ++c) z.dq[g0 + (c + 1) * sz0] += sfv[c][tid] - sfv[c][tid - kPrev];
  }
}

template <int NS, int DIR>
__global__ void __launch_bounds__(kV2TI *kV2TS) k_visc2(Zone z, Param p) {
  visc2_tile<NS, DIR, false>(z, p);
}

// Two temperatures: held to 128 registers (two CTAs per SM; 170-180 unbounded).
template <int NS, int DIR>
__global__ void __launch_bounds__(kV2TI *kV2TS, 2) k_visc2_2t(Zone z, Param p) {
  visc2_tile<NS, DIR, true>(z, p);
}

template <int NS, bool TT = false>
static int launch_visc2_ns(const Zone &z, const Param &p, cudaStream_t s, int &nl) {
  const int ndir = z.mz > 1 ? 3 : 2;
  for (int d = 0; d < ndir; ++d) {
    const int ext[3] = {z.mx, z.my, z.mz};
    const int tr = d == 0 ? z.my : z.mx;
    const int other = d == 2 ? z.my : z.mz;
    dim3 grid((tr + kV2TI - 1) / kV2TI, (ext[d] + kV2TS - 2) / (kV2TS - 1), other);
    static const char *names[3] = {"visc2_x", "visc2_y", "visc2_z"};
    ProfScope prof(names[d], s);
    if constexpr (TT) {
      if (d == 0) k_visc2_2t<NS, 0><<<grid, kV2TI * kV2TS, 0, s>>>(z, p);
      else if (d == 1) k_visc2_2t<NS, 1><<<grid, kV2TI * kV2TS, 0, s>>>(z, p);
      else k_visc2_2t<NS, 2><<<grid, kV2TI * kV2TS, 0, s>>>(z, p);
    } else {
      if (d == 0) k_visc2<NS, 0><<<grid, kV2TI * kV2TS, 0, s>>>(z, p);
      else if (d == 1) k_visc2<NS, 1><<<grid, kV2TI * kV2TS, 0, s>>>(z, p);
      else k_visc2<NS, 2><<<grid, kV2TI * kV2TS, 0, s>>>(z, p);
    }
    ++nl;
    CB2_TRY(check_launch());
  }
  return CB2_OK;
}

bool viscous_assigns_dq(const Param &p) { return p.viscous_order == 8 && p.n_spec == 0; }

int launch_viscous(const Zone &z, const Param &p, const FaceBC *faces, int n_faces, bool assign, cudaStream_t s,
                   int &nl, int phase) {
  if (p.viscous_order == 0) return CB2_OK;
  if (p.viscous_order == 8 && phase != 2) {
    const dim3 grid((z.mx + kVisTI - 1) / kVisTI, (z.my + kVisTJ - 1) / kVisTJ, z.mz), block(kVisTI, kVisTJ);
    {
      ProfScope prof("visc8_node_flux", s);
      if (p.n_spec == 0) {
        if (p.precision == CB2_PREC_MIXED) k_visc8_node_flux_air_f32<<<grid, block, 0, s>>>(z, p);
        else k_visc8_node_flux_air_f64<<<grid, block, 0, s>>>(z, p);
      } else {
        // mixtures: FP64 in both forms (their mixed form keeps the viscous terms in FP64)
        if (!z.kappa || !z.rhoD || (p.i_eve >= 0 && (!z.tve || !z.kappa_ve))) return CB2_ERR_INVALID;
        if (p.i_eve >= 0) {
          if (p.n_spec == 5) k_visc8_node_flux_mix<5, true><<<grid, block, 0, s>>>(z, p);
          else if (p.n_spec == 9) k_visc8_node_flux_mix<9, true><<<grid, block, 0, s>>>(z, p);
          else return CB2_ERR_UNSUPPORTED;
        } else if (p.n_spec == 5) {
          k_visc8_node_flux_mix<5, false><<<grid, block, 0, s>>>(z, p);
        } else if (p.n_spec == 9) {
          k_visc8_node_flux_mix<9, false><<<grid, block, 0, s>>>(z, p);
        } else {
          return CB2_ERR_UNSUPPORTED;
        }
      }
    }
    ++nl;
    CB2_TRY(check_launch());
    if (phase == 1) return CB2_OK;
  }
  if (p.viscous_order == 8) {
    CB2_TRY(launch_periodic_flux_exchange(z, p, faces, n_faces, s, nl));
    if (p.visc8_fused) return CB2_OK;  // the sweeps take the divergence
    {
      ProfScope prof("visc8_divergence", s);
      // the mixed form sums the FP32 node fluxes in FP32 and adds the result to the FP64 dq
      const dim3 grow((z.mx + kVisRow - 1) / kVisRow, z.my, z.mz);
      if (visc8_f32(p)) {
        if (assign) k_visc8_divergence_f32<true><<<grow, kVisRow, 0, s>>>(z, p);
        else k_visc8_divergence_f32<false><<<grow, kVisRow, 0, s>>>(z, p);
      } else if (assign) {
        k_visc8_divergence_f64<true><<<grow, kVisRow, 0, s>>>(z, p);
      } else {
        k_visc8_divergence_f64<false><<<grow, kVisRow, 0, s>>>(z, p);
      }
    }
    ++nl;
    return check_launch();
  }
  if (p.viscous_order == 2) {
    if (p.i_eve >= 0) {
      // two-temperature: the e_ve conduction and flux, T_ve in the diffusing enthalpy
      if (!z.tve || !z.kappa_ve) return CB2_ERR_INVALID;
      if (p.n_spec == 5) return launch_visc2_ns<5, true>(z, p, s, nl);
      if (p.n_spec == 9) return launch_visc2_ns<9, true>(z, p, s, nl);
      return CB2_ERR_UNSUPPORTED;
    }
    switch (p.n_spec) {
      case 0: return launch_visc2_ns<0>(z, p, s, nl);
      case 5: return launch_visc2_ns<5>(z, p, s, nl);
      case 9: return launch_visc2_ns<9>(z, p, s, nl);
      default: return CB2_ERR_UNSUPPORTED;
    }
  }
  return CB2_ERR_UNSUPPORTED;
}

}  // namespace cb2
