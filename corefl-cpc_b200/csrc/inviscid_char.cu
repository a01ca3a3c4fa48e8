// Characteristic WENO5/WENO7 inviscid flux with local Lax-Friedrichs splitting
// (inviscid_scheme 52/72; reference: compute_convective_term_weno_{x,y,z},
// src/WENO.cu:831-1559, 1561-2223, 2225-2886, air specialisation weno_ch_air_x/yz
// src/WENO.cu:10-244, 414-654) fused with the flux difference
// dq -= F_{i+1/2} - F_{i-1/2} (compute_derivative_{x,y,z}, src/WENO.cu:1532-1559).
//
// Per interface: Roe average of (u,v,w, Y) and of p/rho, mixture gamma/c at the Roe
// state, an orthonormal basis (k, n, q) from the face-averaged metric, one LLF lambda =
// max over the stencil of |U_k| + c|grad k|, projection of F and Q onto the left
// eigenvectors at every stencil node, WENO on the split characteristic fluxes, and the
// explicit back-projection.  The y/z face metric is averaged with the i+1 neighbour, as
// the reference does (src/WENO.cu:1615-1617, 2280-2282).  Two-temperature mixtures carry
// rho e_ve as one more scalar row, with the Roe-state thermo of the translational-rotational
// mode (TT).
#include "common.cuh"
#include "thermo.cuh"
#include "thermo_2t.cuh"
#include "weno.cuh"
#include "sweep.cuh"
#include "launch.h"

namespace cb2 {

// Node quantities kept in shared memory (index f of sF):
// 0 U_k = (rho u . grad k)/rho, 1-3 rho u_m U_k + p k_m, 4 p, 5 c |grad k|, 6 J.
constexpr int kNF = 7;

// The interface flux row v goes to out[v * os].  The scalar rows are written as soon as they are
// known, and out[v * os] (v >= 5) holds the row's energy coefficient until then, so that no
// per-scalar array stays in registers across the five characteristic fields.
template <int NS, int ORDER, bool TT = false>
__device__ __forceinline__ void char_flux(const double *__restrict__ sQ, const double *__restrict__ sF, int NN,
                                          int c, int st, double kx, double ky, double kz, double eps,
                                          bool shock, const Mech &mech, double *out, int os) {
  constexpr int NSC = NS + (TT ? 1 : 0);  // transported scalars: species (+ e_ve)
  constexpr int NV = 5 + NSC;
  constexpr int R = ORDER / 2 + 1;  // nodes on each side of the interface
  constexpr int NW = 2 * R - 1;     // values per WENO side
#define Qv(v, m) sQ[(v) * NN + c + (m) * st]
#define Fv(f, m) sF[(f) * NN + c + (m) * st]
  // reads inside the per-field loops: volatile, so that the stencil is not held in registers
  // across the fields
  const volatile double *vQ = sQ, *vF = sF;
#define QvL(v, m) vQ[(v) * NN + c + (m) * st]
#define FvL(f, m) vF[(f) * NN + c + (m) * st]
  // Roe average at the interface between node c (m = 0) and c + st (m = 1)
  const double rho_l = Qv(0, 0), rho_r = Qv(0, 1);
  double t1 = sqrt(rho_l * rho_r);
  const double rlc = 1 / (rho_l + t1), rrc = 1 / (t1 + rho_r);
  const double um = rlc * Qv(1, 0) + rrc * Qv(1, 1);
  const double vm = rlc * Qv(2, 0) + rrc * Qv(2, 1);
  const double wm = rlc * Qv(3, 0) + rrc * Qv(3, 1);
  double cm, gm1;
  // scalar-coupling sums sum_s alpha_s Q_s and sum_s alpha_s Q_s U_k at each stencil node
  double sbq[NS > 0 ? 2 * R : 1], sbf[NS > 0 ? 2 * R : 1];
  if constexpr (NS == 0) {
    const double t_roe = (rlc * Fv(4, 0) + rrc * Fv(4, 1)) / kRAir;
    cm = sqrt(kGammaAir * kRAir * t_roe);
    gm1 = kGammaAir - 1;
  } else {
    double svm[NSC], alpha[NSC], ecoef[NSC];
    double rmix = 0;
#pragma unroll
    for (int s = 0; s < NSC; ++s) svm[s] = rlc * Qv(5 + s, 0) + rrc * Qv(5 + s, 1);
#pragma unroll
    for (int s = 0; s < NS; ++s) rmix += svm[s] * __ldg(mech.gas_const + s);
    const double t_roe = (rlc * Fv(4, 0) + rrc * Fv(4, 1)) / fmax(rmix, 1e-12);
    double gamma;
    if constexpr (TT) characteristic_thermo_2t<NS>(t_roe, svm, mech, gamma, cm, alpha, ecoef);
    else characteristic_thermo<NS>(t_roe, svm, mech, gamma, cm, alpha, ecoef, nullptr);
    gm1 = gamma - 1;
#pragma unroll
    for (int s = 0; s < NSC; ++s) out[(5 + s) * os] = ecoef[s];
#pragma unroll
    for (int m = 0; m < 2 * R; ++m) {
      double sp = 0, sm = 0;
#pragma unroll
      for (int s = 0; s < NSC; ++s) {
        sp = fma(alpha[s], Qv(5 + s, m - R + 1), sp);
        sm = fma(alpha[s], Qv(5 + s, m - R + 1) * Fv(0, m - R + 1), sm);
      }
      sbq[m] = sp;
      sbf[m] = sm;
    }
  }
  // orthonormal basis (k, n, q)
  t1 = rnorm3d(kx, ky, kz);
  kx *= t1; ky *= t1; kz *= t1;
  const double Uk_bar = kx * um + ky * vm + kz * wm;
  double nx = 0, ny = 0, nz = 0;
  if (fabs(kx) > 0.8) { nx = -kz; nz = kx; }
  else { ny = kz; nz = -ky; }
  t1 = rnorm3d(nx, ny, nz);
  nx *= t1; ny *= t1; nz *= t1;
  double qx = ky * nz - kz * ny, qy = kz * nx - kx * nz, qz = kx * ny - ky * nx;
  t1 = rnorm3d(qx, qy, qz);
  qx *= t1; qy *= t1; qz *= t1;
  const double Un = nx * um + ny * vm + nz * wm;
  const double Uq = qx * um + qy * vm + qz * wm;
  const double ic2 = 1.0 / (cm * cm);
  const double alf = 0.5 * gm1 * (um * um + vm * vm + wm * wm);

  // LLF lambda over the stencil
  double lam = 0;
#pragma unroll
  for (int m = -R + 1; m <= R; ++m) {
    const double l = fabs(Fv(0, m)) + Fv(5, m);
    if (l > lam) lam = l;
  }
  double fch[5];
  // one characteristic field at a time: keeps the stencil projections of a single field live
#pragma unroll 1
  for (int l = 0; l < 5; ++l) {
    double L0, L1, L2, L3, L4, tc;
    if (l == 0 || l == 4) {
      const double sg = l == 0 ? 1.0 : -1.0;
      L0 = (alf + sg * Uk_bar * cm) * ic2 * 0.5;
      L1 = -(gm1 * um + sg * kx * cm) * ic2 * 0.5;
      L2 = -(gm1 * vm + sg * ky * cm) * ic2 * 0.5;
      L3 = -(gm1 * wm + sg * kz * cm) * ic2 * 0.5;
      L4 = gm1 * ic2 * 0.5;
      tc = 0.5;
    } else if (l == 1) {
      L0 = -Un; L1 = nx; L2 = ny; L3 = nz; L4 = 0; tc = 0;
    } else if (l == 2) {
      L0 = -Uq; L1 = qx; L2 = qy; L3 = qz; L4 = 0; tc = 0;
    } else {
      L0 = 1 - alf * ic2; L1 = gm1 * um * ic2; L2 = gm1 * vm * ic2; L3 = gm1 * wm * ic2; L4 = -gm1 * ic2;
      tc = -1;
    }
    double vp[NW], vmn[NW];
#pragma unroll
    for (int m = 0; m < 2 * R; ++m) {
      const int o = m - R + 1;
      const double uk = FvL(0, o);
      const double q0 = QvL(0, o), q4 = QvL(4, o);
      double LF = L0 * (q0 * uk) + L1 * FvL(1, o) + L2 * FvL(2, o) + L3 * FvL(3, o) + L4 * ((q4 + FvL(4, o)) * uk);
      double LQ = L0 * q0 + L1 * QvL(1, o) + L2 * QvL(2, o) + L3 * QvL(3, o) + L4 * q4;
      if constexpr (NS > 0) {
        LF += tc * sbf[m];
        LQ += tc * sbq[m];
      }
      const double hj = 0.5 * FvL(6, o);
      if (m < NW) vp[m] = hj * (LF + lam * LQ);
      if (m > 0) vmn[m - 1] = hj * (LF - lam * LQ);
    }
    fch[l] = weno_pm<ORDER>(vp, vmn, eps, shock);
  }
  // back-projection with the right eigenvectors
  const double f034 = fch[0] + fch[3] + fch[4];
  const double f04 = fch[0] - fch[4];
  double e = 0;
  if constexpr (NS > 0) {
#pragma unroll 1
    for (int s = 0; s < NSC; ++s) {
      const double svs = rlc * QvL(5 + s, 0) + rrc * QvL(5 + s, 1);
      double vp[NW], vmn[NW];
#pragma unroll
      for (int m = 0; m < 2 * R; ++m) {
        const int o = m - R + 1;
        const double LQ = QvL(5 + s, o) - svs * QvL(0, o);
        const double LF = FvL(0, o) * LQ;
        const double hj = 0.5 * FvL(6, o);
        if (m < NW) vp[m] = hj * (LF + lam * LQ);
        if (m > 0) vmn[m - 1] = hj * (LF - lam * LQ);
      }
      const double fs = weno_pm<ORDER>(vp, vmn, eps, shock);
      e += out[(5 + s) * os] * fs;
      out[(5 + s) * os] = svs * f034 + fs;
    }
  }
  out[0] = f034;
  out[os] = um * f034 - kx * cm * f04 + nx * fch[1] + qx * fch[2];
  out[2 * os] = vm * f034 - ky * cm * f04 + ny * fch[1] + qy * fch[2];
  out[3 * os] = wm * f034 - kz * cm * f04 + nz * fch[1] + qz * fch[2];
  const double h_roe = rlc * (Qv(4, 0) + Fv(4, 0)) + rrc * (Qv(4, 1) + Fv(4, 1));
  out[4 * os] = h_roe * f034 - Uk_bar * cm * f04 + Un * fch[1] + Uq * fch[2] - cm * cm / gm1 * fch[3] + e;
#undef Qv
#undef Fv
#undef QvL
#undef FvL
}

// Loads node data of one slot: conservative variables, U_k, momentum fluxes, p, c|grad k|, J.
template <int NS, int DIR, bool TT = false>
__device__ __forceinline__ void load_node(const Zone &z, idx_t g, double *sQ, double *sF, int NN, int slot) {
  constexpr int NV = 5 + NS + (TT ? 1 : 0);
  const idx_t sz = z.L.sz;
  const double q0 = z.cv[g], q1 = z.cv[g + sz], q2 = z.cv[g + 2 * sz], q3 = z.cv[g + 3 * sz], q4 = z.cv[g + 4 * sz];
  const double m0 = z.metric[g + (3 * DIR) * sz], m1 = z.metric[g + (3 * DIR + 1) * sz],
               m2 = z.metric[g + (3 * DIR + 2) * sz];
  const double pk = z.bv[g + 4 * sz];
  const double Uk = (q1 * m0 + q2 * m1 + q3 * m2) / q0;
  sQ[0 * NN + slot] = q0;
  sQ[1 * NN + slot] = q1;
  sQ[2 * NN + slot] = q2;
  sQ[3 * NN + slot] = q3;
  sQ[4 * NN + slot] = q4;
#pragma unroll
  for (int v = 5; v < NV; ++v) sQ[v * NN + slot] = z.cv[g + v * sz];
  sF[0 * NN + slot] = Uk;
  sF[1 * NN + slot] = fma(q1, Uk, pk * m0);
  sF[2 * NN + slot] = fma(q2, Uk, pk * m1);
  sF[3 * NN + slot] = fma(q3, Uk, pk * m2);
  sF[4 * NN + slot] = pk;
  double cg = norm3d(m0, m1, m2);
  if constexpr (NS == 0) cg *= sqrt(kGammaAir * kRAir * z.bv[g + 5 * sz]);
  else cg *= z.acoustic[g];
  sF[5 * NN + slot] = cg;
  sF[6 * NN + slot] = z.jac[g];
}

// Positivity limiter of the species rows of an interface flux (src/WENO.cu:1459-1528): with
// alpha = 1/3 (3-D) or 1/2, every species flux is blended with a first-order flux f1 by
// theta = min(theta_p, theta_m) so that the one-sided updates alpha J rhoY -+ dt f of the left
// and right nodes stay non-negative; NS counts every transported scalar (species and, in two
// temperatures, e_ve).  Slots cl / cr of the left / right node.
template <int NS>
__device__ __forceinline__ void positive_limit(const double *sQ, const double *sF, int NN, int cl, int cr,
                                               const Param &p, double *out, int os) {
#define fc(v) out[(v) * os]
  const double dt = step_dt(p, p.dt);
  const double alpha = p.dim == 3 ? 1.0 / 3.0 : 0.5;
  const double jl = sF[6 * NN + cl], jr = sF[6 * NN + cr];
  const double alphaL = 0.5 * alpha * jl, alphaR = 0.5 * alpha * jr;
  int start = -1;
  for (int s = 0; s < NS; ++s) {
    const double up = alphaL * sQ[(s + 5) * NN + cl] - dt * fc(s + 5);
    const double um = alphaR * sQ[(s + 5) * NN + cr] + dt * fc(s + 5);
    if (up < 0 || um < 0) {
      start = s;
      break;
    }
  }
  if (start < 0) return;
  const double Ul = sF[cl], Ur = sF[cr];
  const double U1 = Ul * jl, U2 = Ur * jr;
  for (int s = start; s < NS; ++s) {
    double f1 = 0, theta_p = 1, theta_m = 1;
    bool have_f1 = false;
    const double yl = sQ[(s + 5) * NN + cl], yr = sQ[(s + 5) * NN + cr];
    const double fp = 0.5 * jl * (Ul + sF[5 * NN + cl]) * yl;
    const double fm = 0.5 * jr * (Ur - sF[5 * NN + cr]) * yr;
    const double up = alphaL * yl - dt * fc(s + 5);
    if (up < 0) {
      f1 = 0.5 * (fp + U1 * yl) + 0.5 * (fm - U2 * yr);
      have_f1 = true;
      const double up_lf = alphaL * yl - dt * f1;
      if (fabs(up - up_lf) > 1e-20 * p.rho_ref) {
        theta_p = (0 - up_lf) / (up - up_lf);
        if (theta_p > 1) theta_p = 1.0;
        else if (theta_p < 0) theta_p = 0;
      }
    }
    const double um = alphaR * yr + dt * fc(s + 5);
    if (um < 0) {
      if (!have_f1) f1 = 0.5 * (fp + U1 * yl) + 0.5 * (fm - U2 * yr);
      const double um_lf = alphaR * yr + dt * f1;
      if (fabs(um - um_lf) > 1e-20 * p.rho_ref) {
        theta_m = (0 - um_lf) / (um - um_lf);
        if (theta_m > 1) theta_m = 1.0;
        else if (theta_m < 0) theta_m = 0;
      }
    }
    fc(s + 5) = fmin(theta_p, theta_m) * (fc(s + 5) - f1) + f1;
  }
#undef fc
}

template <int NS, int DIR, int ORDER, bool TT = false>
__global__ void __launch_bounds__(kSweepThreads, 2) k_weno_char(Zone z, Param p, idx_t run) {
  constexpr int NV = 5 + NS + (TT ? 1 : 0);
  constexpr int R = ORDER / 2 + 1;
  constexpr int NN = DIR == 0 ? (kSweepThreads + 2 * R - 1) : kTI * (kTS + 2 * R - 1);
  extern __shared__ double smem[];
  double *sQ = smem;
  double *sF = sQ + NV * NN;
  double *sFl = sF + kNF * NN;  // [NV][kSweepThreads]
  const int tid = threadIdx.x;
  const int g = z.ngg;
  const Layout &L = z.L;

  int i, j, k;          // node left of this thread's interface
  bool valid_if;        // this thread owns a real interface
  int c, st;            // shared slot of the left node and the sweep stride
  if constexpr (DIR == 0) {
    k = blockIdx.z;
    const idx_t q0 = (idx_t)blockIdx.x * (kSweepThreads - 1) - 1;  // run position of interface tid=0
    const idx_t base = (idx_t)k * L.disp1 + L.dispt - g;            // global index of run position 0
    // load nodes run positions [q0 - R + 1, q0 + kSweepThreads + R - 1]
    const idx_t qlo = q0 - R + 1;
    const idx_t qmin = -(idx_t)g * L.disp2, qmax = (idx_t)(L.my + g) * L.disp2;
    for (int s = tid; s < NN; s += kSweepThreads) {
      const idx_t q = qlo + s;
      if (q >= qmin && q < qmax) load_node<NS, 0, TT>(z, base + q, sQ, sF, NN, s);
    }
    const idx_t q = q0 + tid;
    const idx_t jj = q >= 0 ? q / L.disp2 : -1;
    i = (int)(q - jj * L.disp2) - g;
    j = (int)jj;
    valid_if = q >= 0 && q < run && i >= -1 && i <= L.mx - 1;
    c = tid + R - 1;
    st = 1;
  } else {
    const int ti = tid % kTI, ts = tid / kTI;
    i = blockIdx.x * kTI + ti;
    const int s0 = blockIdx.y * (kTS - 1);  // first node of the tile along the sweep
    const int ms = DIR == 1 ? L.my : L.mz;
    if (DIR == 1) k = blockIdx.z; else j = blockIdx.z;
    for (int s = ts; s < kTS + 2 * R - 1; s += kTS) {
      const int n = s0 - R + s;  // sweep index of this node slot
      if (i < L.mx && n < ms + g) {
        const idx_t gi = DIR == 1 ? L.at(i, n, k) : L.at(i, j, n);
        load_node<NS, DIR, TT>(z, gi, sQ, sF, NN, s * kTI + ti);
      }
    }
    const int n_if = s0 - 1 + ts;  // interface n_if + 1/2
    if (DIR == 1) j = n_if; else k = n_if;
    valid_if = i < L.mx && n_if <= ms - 1;
    c = (ts + R - 1) * kTI + ti;
    st = kTI;
  }
  __syncthreads();

  if (valid_if) {
    const idx_t sz = L.sz;
    const idx_t gl = L.at(i, j, k);
    // face metric: average with the next node along the sweep for x, with the i+1 node for y/z
    const idx_t gr = L.at(i + 1, j, k);
    const double *M = z.metric + (idx_t)(3 * DIR) * sz;
    const double kx = 0.5 * (M[gl] + M[gr]);
    const double ky = 0.5 * (M[gl + sz] + M[gr + sz]);
    const double kz = 0.5 * (M[gl + 2 * sz] + M[gr + 2 * sz]);
    bool shock = true;
    if (p.sensor_threshold > 1e-10) {
      shock = false;
      for (int d = -g + 1; d <= g; ++d) {
        const idx_t gs = DIR == 0 ? L.at(i + d, j, k) : (DIR == 1 ? L.at(i, j + d, k) : L.at(i, j, k + d));
        if (z.shock[gs] > p.sensor_threshold) { shock = true; break; }
      }
    }
    char_flux<NS, ORDER, TT>(sQ, sF, NN, c, st, kx, ky, kz, kWenoEps * p.weno_eps_scale, shock, p.mech,
                             sFl + tid, kSweepThreads);
    if constexpr (NS > 0) {
      if (p.positive_preserving)
        positive_limit<NS + (TT ? 1 : 0)>(sQ, sF, NN, c, c + st, p, sFl + tid, kSweepThreads);
    }
  }
  __syncthreads();

  // flux difference for the node right of interface tid-1 / left of interface tid
  int ni = i, nj = j, nk = k;
  bool valid_node;
  if constexpr (DIR == 0) {
    ni = i;  // node left of interface tid is node i; it uses interfaces tid-1 and tid
    valid_node = tid >= 1 && valid_if && i >= 0;
  } else {
    const int ts = tid / kTI;
    valid_node = ts >= 1 && valid_if && (DIR == 1 ? j >= 0 : k >= 0);
  }
  if (valid_node) {
    const int tprev = DIR == 0 ? tid - 1 : tid - kTI;
    const idx_t gd = z.L0.at(ni, nj, nk);
    const idx_t sz0 = z.L0.sz;
#pragma unroll
    for (int v = 0; v < NV; ++v)
      z.dq[gd + v * sz0] -= sFl[v * kSweepThreads + tid] - sFl[v * kSweepThreads + tprev];
  }
}

// ---- component-wise WENO (inviscid_scheme 51/71, src/WENO.cu:890-1089) ---------------------
// Each node is split with its own LLF speed lambda0 = |U_k| + c|grad k|:
//   F+- = 0.5 J ((U_k +- lambda0) Q + p (0, k_x, k_y, k_z, U_k)),
// and every conservative component is reconstructed on its own, with eps scaled by v_ref^2
// for momentum and v_ref^4 for energy.
template <int NS, int DIR>
__device__ __forceinline__ void load_node_split(const Zone &z, idx_t g, double *sP, double *sM, int NN, int slot) {
  constexpr int NV = 5 + NS;
  const idx_t sz = z.L.sz;
  const double q0 = z.cv[g], q1 = z.cv[g + sz], q2 = z.cv[g + 2 * sz], q3 = z.cv[g + 3 * sz], q4 = z.cv[g + 4 * sz];
  const double m0 = z.metric[g + (3 * DIR) * sz], m1 = z.metric[g + (3 * DIR + 1) * sz],
               m2 = z.metric[g + (3 * DIR + 2) * sz];
  double pk = z.bv[g + 4 * sz];
  const double Uk = (q1 * m0 + q2 * m1 + q3 * m2) / q0;
  double cg = norm3d(m0, m1, m2);
  if constexpr (NS == 0) cg *= sqrt(kGammaAir * kRAir * z.bv[g + 5 * sz]);
  else cg *= z.acoustic[g];
  const double lambda0 = fabs(Uk) + cg;
  const double hj = 0.5 * z.jac[g];
  const double sp = hj * (Uk + lambda0), sm = hj * (Uk - lambda0);
  pk *= hj;
  sP[0 * NN + slot] = sp * q0;
  sP[1 * NN + slot] = fma(sp, q1, pk * m0);
  sP[2 * NN + slot] = fma(sp, q2, pk * m1);
  sP[3 * NN + slot] = fma(sp, q3, pk * m2);
  sP[4 * NN + slot] = fma(sp, q4, pk * Uk);
  sM[0 * NN + slot] = sm * q0;
  sM[1 * NN + slot] = fma(sm, q1, pk * m0);
  sM[2 * NN + slot] = fma(sm, q2, pk * m1);
  sM[3 * NN + slot] = fma(sm, q3, pk * m2);
  sM[4 * NN + slot] = fma(sm, q4, pk * Uk);
#pragma unroll
  for (int v = 5; v < NV; ++v) {
    const double ql = z.cv[g + v * sz];
    sP[v * NN + slot] = sp * ql;
    sM[v * NN + slot] = sm * ql;
  }
}

template <int NS, int DIR, int ORDER>
__global__ void __launch_bounds__(kSweepThreads) k_weno_comp(Zone z, Param p, idx_t run) {
  constexpr int NV = 5 + NS;
  constexpr int R = ORDER / 2 + 1;
  constexpr int NW = 2 * R - 1;
  constexpr int NN = DIR == 0 ? (kSweepThreads + 2 * R - 1) : kTI * (kTS + 2 * R - 1);
  extern __shared__ double smem[];
  double *sP = smem;
  double *sM = sP + NV * NN;
  double *sFl = sM + NV * NN;
  const int tid = threadIdx.x;
  const int g = z.ngg;
  const Layout &L = z.L;
  int i, j, k;
  bool valid_if;
  int c, st;
  if constexpr (DIR == 0) {
    k = blockIdx.z;
    const idx_t q0 = (idx_t)blockIdx.x * (kSweepThreads - 1) - 1;
    const idx_t base = (idx_t)k * L.disp1 + L.dispt - g;
    const idx_t qlo = q0 - R + 1;
    const idx_t qmin = -(idx_t)g * L.disp2, qmax = (idx_t)(L.my + g) * L.disp2;
    for (int s = tid; s < NN; s += kSweepThreads) {
      const idx_t q = qlo + s;
      if (q >= qmin && q < qmax) load_node_split<NS, 0>(z, base + q, sP, sM, NN, s);
    }
    const idx_t q = q0 + tid;
    const idx_t jj = q >= 0 ? q / L.disp2 : -1;
    i = (int)(q - jj * L.disp2) - g;
    j = (int)jj;
    valid_if = q >= 0 && q < run && i >= -1 && i <= L.mx - 1;
    c = tid + R - 1;
    st = 1;
  } else {
    const int ti = tid % kTI, ts = tid / kTI;
    i = blockIdx.x * kTI + ti;
    const int s0 = blockIdx.y * (kTS - 1);
    const int ms = DIR == 1 ? L.my : L.mz;
    if (DIR == 1) k = blockIdx.z; else j = blockIdx.z;
    for (int s = ts; s < kTS + 2 * R - 1; s += kTS) {
      const int n = s0 - R + s;
      if (i < L.mx && n < ms + g) {
        const idx_t gi = DIR == 1 ? L.at(i, n, k) : L.at(i, j, n);
        load_node_split<NS, DIR>(z, gi, sP, sM, NN, s * kTI + ti);
      }
    }
    const int n_if = s0 - 1 + ts;
    if (DIR == 1) j = n_if; else k = n_if;
    valid_if = i < L.mx && n_if <= ms - 1;
    c = (ts + R - 1) * kTI + ti;
    st = kTI;
  }
  __syncthreads();
  if (valid_if) {
    bool shock = true;
    if (p.sensor_threshold > 1e-10) {
      shock = false;
      for (int d = -g + 1; d <= g; ++d) {
        const idx_t gs = DIR == 0 ? L.at(i + d, j, k) : (DIR == 1 ? L.at(i, j + d, k) : L.at(i, j, k + d));
        if (z.shock[gs] > p.sensor_threshold) { shock = true; break; }
      }
    }
    const double e0 = kWenoEps * p.weno_eps_scale;
    const double e1 = e0 * p.v_ref * p.v_ref, e2 = e1 * p.v_ref * p.v_ref;
#pragma unroll 1
    for (int l = 0; l < NV; ++l) {
      const double eps = (l >= 1 && l <= 3) ? e1 : (l == 4 ? e2 : e0);
      double vp[NW], vm[NW];
#pragma unroll
      for (int m = 0; m < NW; ++m) {
        vp[m] = sP[l * NN + c + (m - R + 1) * st];
        vm[m] = sM[l * NN + c + (m - R + 2) * st];
      }
      sFl[l * kSweepThreads + tid] = weno_pm<ORDER>(vp, vm, eps, shock);
    }
  }
  __syncthreads();
  bool valid_node;
  if constexpr (DIR == 0) valid_node = tid >= 1 && valid_if && i >= 0;
  else valid_node = (tid / kTI) >= 1 && valid_if && (DIR == 1 ? j >= 0 : k >= 0);
  if (valid_node) {
    const int tprev = DIR == 0 ? tid - 1 : tid - kTI;
    const idx_t gd = z.L0.at(i, j, k);
    const idx_t sz0 = z.L0.sz;
#pragma unroll
    for (int v = 0; v < NV; ++v) z.dq[gd + v * sz0] -= sFl[v * kSweepThreads + tid] - sFl[v * kSweepThreads + tprev];
  }
}

template <int NS, int ORDER>
static int launch_comp_dir(int dir, const Zone &z, const Param &p, cudaStream_t s) {
  constexpr int NV = 5 + NS;
  constexpr int R = ORDER / 2 + 1;
  SweepGeom geo;
  const dim3 grid = sweep_grid(dir, z.L, geo);
  const size_t smem = sizeof(double) * ((size_t)2 * NV * sweep_nodes(dir, R) + (size_t)NV * kSweepThreads);
  if (grid.x == 0 || grid.y == 0 || grid.z == 0) return CB2_OK;
  static const char *names[3] = {"weno_comp_x", "weno_comp_y", "weno_comp_z"};
  ProfScope prof(names[dir], s);
  if (dir == 0) {
    auto kern = k_weno_comp<NS, 0, ORDER>;
    CB2_TRY(prepare_smem(kern, smem));
    kern<<<grid, kSweepThreads, smem, s>>>(z, p, geo.run);
  } else if (dir == 1) {
    auto kern = k_weno_comp<NS, 1, ORDER>;
    CB2_TRY(prepare_smem(kern, smem));
    kern<<<grid, kSweepThreads, smem, s>>>(z, p, 0);
  } else {
    auto kern = k_weno_comp<NS, 2, ORDER>;
    CB2_TRY(prepare_smem(kern, smem));
    kern<<<grid, kSweepThreads, smem, s>>>(z, p, 0);
  }
  return check_launch();
}

template <int NS>
static int launch_comp_ns(const Zone &z, const Param &p, int order, cudaStream_t s, int &n_launch) {
  const int ndir = z.mz > 1 ? 3 : 2;
  for (int d = 0; d < ndir; ++d) {
    int rc = order == 5 ? launch_comp_dir<NS, 5>(d, z, p, s) : launch_comp_dir<NS, 7>(d, z, p, s);
    if (rc) return rc;
    ++n_launch;
  }
  return CB2_OK;
}

int launch_inviscid_comp(const Zone &z, const Param &p, cudaStream_t s, int &n_launch) {
  const int order = (p.inviscid_scheme == CB2_INV_WENO5_CP) ? 5 : 7;
  switch (p.n_spec) {
    case 0: return launch_comp_ns<0>(z, p, order, s, n_launch);
    case 5: return launch_comp_ns<5>(z, p, order, s, n_launch);
    case 9: return launch_comp_ns<9>(z, p, order, s, n_launch);
    default: return CB2_ERR_UNSUPPORTED;
  }
}

template <int NS, int ORDER, bool TT = false>
static int launch_dir(int dir, const Zone &z, const Param &p, cudaStream_t s) {
  constexpr int NV = 5 + NS + (TT ? 1 : 0);
  constexpr int R = ORDER / 2 + 1;
  SweepGeom geo;
  const dim3 grid = sweep_grid(dir, z.L, geo);
  const size_t smem = sizeof(double) * ((size_t)(NV + kNF) * sweep_nodes(dir, R) + (size_t)NV * kSweepThreads);
  if (grid.x == 0 || grid.y == 0 || grid.z == 0) return CB2_OK;
  static const char *names[3] = {"weno_char_x", "weno_char_y", "weno_char_z"};
  ProfScope prof(names[dir], s);
  if (dir == 0) {
    auto kern = k_weno_char<NS, 0, ORDER, TT>;
    CB2_TRY(prepare_smem(kern, smem));
    kern<<<grid, kSweepThreads, smem, s>>>(z, p, geo.run);
  } else if (dir == 1) {
    auto kern = k_weno_char<NS, 1, ORDER, TT>;
    CB2_TRY(prepare_smem(kern, smem));
    kern<<<grid, kSweepThreads, smem, s>>>(z, p, 0);
  } else {
    auto kern = k_weno_char<NS, 2, ORDER, TT>;
    CB2_TRY(prepare_smem(kern, smem));
    kern<<<grid, kSweepThreads, smem, s>>>(z, p, 0);
  }
  return check_launch();
}

template <int NS, bool TT = false>
static int launch_char_ns(const Zone &z, const Param &p, int order, cudaStream_t s, int &n_launch) {
  const int ndir = z.mz > 1 ? 3 : 2;
  for (int d = 0; d < ndir; ++d) {
    int rc = order == 5 ? launch_dir<NS, 5, TT>(d, z, p, s) : launch_dir<NS, 7, TT>(d, z, p, s);
    if (rc) return rc;
    ++n_launch;
  }
  return CB2_OK;
}

int launch_inviscid_char(const Zone &z, const Param &p, cudaStream_t s, int &n_launch) {
  const int order = (p.inviscid_scheme == CB2_INV_WENO5_CH) ? 5 : 7;
  if (p.i_eve >= 0) {
    if (p.n_spec == 5) return launch_char_ns<5, true>(z, p, order, s, n_launch);
    if (p.n_spec == 9) return launch_char_ns<9, true>(z, p, order, s, n_launch);
    return CB2_ERR_UNSUPPORTED;
  }
  switch (p.n_spec) {
    case 0: return launch_char_ns<0>(z, p, order, s, n_launch);
    case 5: return launch_char_ns<5>(z, p, order, s, n_launch);
    case 9: return launch_char_ns<9>(z, p, order, s, n_launch);
    default: return CB2_ERR_UNSUPPORTED;
  }
}

}  // namespace cb2
