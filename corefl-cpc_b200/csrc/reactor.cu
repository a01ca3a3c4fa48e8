// Batched 0-D constant-volume reactors: one warp per reactor, FP64 throughout.
//
// The integrator is the adaptive ROK4E Rosenbrock-Krylov scheme in its full-Jacobian form, as
// const_volume_reactor runs it with advance_scheme = 1, build_arnoldi = 0,
// adaptive_time_step = 1 (src/ConstVolumeReactor.cpp:385-700):
//   source       compute_src, generic mechanism (:925-951, rates :1692-1737) via chem_rates
//   Jacobian     compute_chem_src_jacobian (:1739-1758), d omega_m / d (rho Y)_n from the rates
//                of progress, in kg/(m^3 s) per kg/m^3
//   linear solve I - h gamma J factored by Crout-style LU with row pivoting and solved by
//                forward/back substitution (lu_decomp / lu_to_solution, :1802-1857)
//   temperature  update_t: Newton on the internal energy, |1 - T1/T| <= 1e-8, at most 100
//                iterations (:1456-1479)
//   step control error norm sqrt(mean((h sum e_i k_i / (RTol rhoY_new + ATol))^2)); accept if
//                <= 1; next step h * min(5, max(0.2, 0.8 err_last^0.1 err^-0.175)) after the
//                first accepted step, h * 0.2 on a rejected first step (:664-700)
// The Rosenbrock coefficients are the published ROK4E table (Tranquilli and Sandu), the same
// numbers src/Define.h:33-48 lists.  The Krylov instantiation replaces J by its Arnoldi
// projection (build_arnoldi = 1, Krylov limit n_spec).  k_reactor_fixed runs the fixed-step forms (explicit, EPI, DA,
// explicit RK3) of the same function.
#include <type_traits>

#include "chem.cuh"
#include "launch.h"
#include "cb200_serve.h"

namespace cb2 {

namespace rok4e {
constexpr double gamma = 0.572816062482135;
constexpr double a21 = 0.432364435748567;
constexpr double a31 = -0.51421131687617;
constexpr double a32 = 1.38227114461736;
constexpr double g21 = -0.602765307997356 / gamma;
constexpr double g31 = -1.389195789724843 / gamma;
constexpr double g32 = 1.072950969011413 / gamma;
constexpr double g41 = 0.992356412977094 / gamma;
constexpr double g42 = -1.390032613873701 / gamma;
constexpr double g43 = -0.440875890223325 / gamma;
constexpr double b1 = 0.194335256262729, b2 = 0.483167813989227, b4 = 0.322496929748044;
constexpr double e1 = -0.217819895945721 - b1, e2 = 1.03130847478467 - b2, e3 = 0.186511421161047, e4 = -b4;
}  // namespace rok4e

constexpr int kReactorThreads = 64;

// Forward and back substitution with the LU factors of warp_lu (row pivots in piv), as
// lu_to_solution does (src/ConstVolumeReactor.cpp:1835-1857).
__device__ __forceinline__ void lu_solve_n(const double *a, const int *piv, double *b, int N) {
  for (int r = 0; r < N; ++r) {
    const int t = piv[r];
    if (t != r) {
      const double x = b[t];
      b[t] = b[r];
      b[r] = x;
    }
  }
  for (int r = 1; r < N; ++r)
    for (int t = 0; t < r; ++t) b[r] -= a[r * N + t] * b[t];
  b[N - 1] /= a[N * N - 1];
  for (int r = N - 2; r >= 0; --r) {
    for (int t = r + 1; t < N; ++t) b[r] -= a[r * N + t] * b[t];
    b[r] /= a[r * N + r];
  }
}

template <int N>
__device__ __forceinline__ void lu_solve(const double *a, const int *piv, double *b) {
  lu_solve_n(a, piv, b, N);
}

template <int NS>
__global__ void __launch_bounds__(kReactorThreads) k_reactor_setup(cb2_reactor *R, int n, Mech m, const double *T0,
                                                                   const double *p0, const double *Y,
                                                                   const double *t_end, double h0) {
  const int id = blockIdx.x * kReactorThreads + threadIdx.x;
  if (id >= n) return;
  cb2_reactor st{};
  const double t = T0[id], p = p0[id];
  double y[NS], imw = 0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    y[s] = Y[(long long)id * NS + s];
    imw += y[s] / __ldg(m.mw + s);
  }
  const double rho = p / (t * kRu * imw);
  double h[NS];
  species_h<NS>(t, m, h);
  double E = 0;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    st.rhoY[s] = y[s] * rho;
    E += y[s] * h[s];
  }
  E -= p / rho;
  st.rho = rho;
  st.E = E;
  st.T = t;
  st.p = p;
  st.time = 0;
  st.t_end = t_end[id];
  st.h = h0;
  st.err_last = 0;
  R[id] = st;
}

// ---- one warp per reactor ----------------------------------------------------------------
// The lanes of a warp share one reactor: species-wise work on lanes 0..NS-1, one reaction per
// lane for the rates of progress, three Jacobian entries per lane, the rows of a column in the
// LU.  Every sum keeps the serial order: its terms are parked in shared memory and summed in
// index order by each lane, so every lane holds the same value.
constexpr int kReactorWarps = 4;  // reactors per CTA

template <int NS>
struct ReactorShared {
  double rhoY[NS], omega[NS], k1[NS], k2[NS], k3[NS], k4[NS], ys[NS], yk[NS], c[NS], gibbs[NS];
  double ta[NS], tb[NS];
  double q1[kMaxReac], q2[kMaxReac];
  double lhs[NS * NS];
  int piv[NS];
};

// Species s as a one-species mechanism (for the per-species thermo of one lane).
__device__ __forceinline__ Mech mech_species(const Mech &m, int s) {
  Mech o = m;
  o.t_low += s; o.t_mid += s; o.t_high += s;
  o.lo += 7 * s; o.hi += 7 * s;
  o.gas_const += s; o.imw += s; o.mw += s;
  if (m.nasa9) {
    o.n_range += s;
    o.t_cut += s * (m.max_range + 1);
    o.poly9 += s * m.max_range * 9;
  }
  return o;
}

// omega of the state y (partial densities) at temperature t; q1/q2 of every reaction.  Kept out
// of line: an attempt evaluates it three times, and three inlined copies overflowed the
// instruction cache (ncu: "no instruction" the largest stall); one copy cuts the attempt from
// 53 to 42 us at the cost of 3% of the saturated throughput.
template <int NS>
__device__ __noinline__ void warp_source(double t, const double *y, const Mech &m, bool gibbs_needed,
                                            ReactorShared<NS> &S, int lane) {
  if (lane < NS) {
    S.c[lane] = y[lane] / __ldg(m.mw + lane) * 1e-3;
    if (gibbs_needed) species_gibbs_rt<1>(t, mech_species(m, lane), &S.gibbs[lane]);
  }
  __syncwarp();
  constexpr double temp_p = kPatm / kRu * 1e-3;
  const double temp_t = temp_p / t;
  for (int r = lane; r < m.n_reac; r += 32) reaction_progress<NS>(r, t, t, S.c, S.gibbs, temp_t, m, S.q1[r], S.q2[r]);
  __syncwarp();
  if (lane < NS) {
    double cre = 0, des = 0;
    for (int r = 0; r < m.n_reac; ++r) {
      const double f = __ldg(m.stoi_f + r * NS + lane), b = __ldg(m.stoi_b + r * NS + lane);
      cre += S.q2[r] * f + S.q1[r] * b;
      des += S.q1[r] * f + S.q2[r] * b;
    }
    const double w = 1e+3 * __ldg(m.mw + lane);
    S.omega[lane] = cre * w - des * w;
  }
  __syncwarp();
}

// Newton T from E at the composition S.yk (mass fractions), mean 1/W imw, from t0.
template <int NS>
__device__ __forceinline__ double warp_temperature(double t0, double imw, double E, const Mech &m,
                                                   ReactorShared<NS> &S, int lane) {
  double t = t0;
  const double R = kRu * imw;
  double err = 1e+6;
  int iter = 0;
  while (err > 1e-8 && iter++ < 100) {
    if (lane < NS) {
      double h, cp;
      species_h_cp<1>(t, mech_species(m, lane), &h, &cp);
      S.ta[lane] = cp * S.yk[lane];
      S.tb[lane] = h * S.yk[lane];
    }
    __syncwarp();
    double cpt = 0, ht = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      cpt += S.ta[s];
      ht += S.tb[s];
    }
    __syncwarp();
    const double et = ht - R * t;
    const double cv = cpt - R;
    const double t1 = t - (et - E) / cv;
    err = fabs(1 - t1 / t);
    t = t1;
  }
  return t;
}

// sum over s of S.ta[s] in index order, after lanes 0..NS-1 wrote their terms
template <int NS>
__device__ __forceinline__ double warp_sum_ta(ReactorShared<NS> &S) {
  __syncwarp();
  double v = 0;
#pragma unroll
  for (int s = 0; s < NS; ++s) v += S.ta[s];
  __syncwarp();
  return v;
}

// LU of the n x n matrix S.lhs with row pivoting in the Crout ordering of lu_decomp
// (src/ConstVolumeReactor.cpp:1802-1833: column c of L, pivot, row c of U, scale), the rows or
// columns of each step on separate lanes; the pivot search keeps the serial rule (the first
// largest |.|).
template <typename SH>
__device__ __forceinline__ void warp_lu_n(SH &S, int N, int lane) {
  double *a = S.lhs;
  for (int n = 0; n < N; ++n) {
    if (lane >= n && lane < N) {
      double v = a[lane * N + n];
      for (int t = 0; t < n; ++t) v -= a[lane * N + t] * a[t * N + n];
      a[lane * N + n] = v;
    }
    __syncwarp();
    int ik = n;
    for (int r = n + 1; r < N; ++r)
      if (fabs(a[r * N + n]) > fabs(a[ik * N + n])) ik = r;
    if (lane == 0) S.piv[n] = ik;
    if (ik != n && lane < N) {
      const double x = a[ik * N + lane];
      a[ik * N + lane] = a[n * N + lane];
      a[n * N + lane] = x;
    }
    __syncwarp();
    if (lane > n && lane < N) {
      double v = a[n * N + lane];
      for (int t = 0; t < n; ++t) v -= a[n * N + t] * a[t * N + lane];
      a[n * N + lane] = v;
    }
    __syncwarp();
    const double d = a[n * N + n];
    if (lane > n && lane < N) a[lane * N + n] /= d;
    __syncwarp();
  }
}

template <int N, typename SH>
__device__ __forceinline__ void warp_lu(SH &S, int lane) {
  warp_lu_n(S, N, lane);
}

// Solves LU b = rhs in place on lane 0 (the substitutions are serial), then shares it.
template <int N, typename SH>
__device__ __forceinline__ void warp_solve(SH &S, double *b, int lane) {
  __syncwarp();
  if (lane == 0) lu_solve<N>(S.lhs, S.piv, b);
  __syncwarp();
}

// ---- the Krylov form (build_arnoldi = 1) ---------------------------------------------------
template <int NS>
struct KrylovShared : ReactorShared<NS> {
  double Q[NS * NS], H[NS * NS], f0[NS], w[NS], g[NS], sol[NS], f[NS];
};

// sum over s < NS of a[s] * b[s] in index order (gxl::vec_dot), the same value on every lane
template <int NS>
__device__ __forceinline__ double warp_dot(ReactorShared<NS> &S, const double *a, const double *b, int lane) {
  if (lane < NS) S.ta[lane] = a[lane] * b[lane];
  return warp_sum_ta<NS>(S);
}

// buildArnoldi (src/ConstVolumeReactor.cpp:1858-1930) with the Krylov limit NS and minimum 4, from
// f0 = S.f0 at (T, S.rhoY): q0 = f0 / |f0| (e_0 if |f0| < 1e-30); column c: w = (omega(T', rhoY +
// eps q_c) - f0) / eps, eps = 1e-6 (1 + |rhoY|), T' the Newton temperature of the perturbed state;
// modified Gram-Schmidt into H(0..c, c); H(c+1, c) = |w|.  Returns the Krylov dimension.
template <int NS>
__device__ int warp_arnoldi(double T, double rho, double E, const Mech &m, bool gibbs_needed, KrylovShared<NS> &S,
                            int lane) {
  for (int e = lane; e < NS * NS; e += 32) S.Q[e] = S.H[e] = 0.0;
  __syncwarp();
  const double eps = 1e-6 * (1 + sqrt(fmax(warp_dot<NS>(S, S.rhoY, S.rhoY, lane), 0.0)));
  const double nf = sqrt(fmax(warp_dot<NS>(S, S.f0, S.f0, lane), 0.0));
  if (lane < NS) S.Q[lane] = nf < 1e-30 ? (lane == 0 ? 1.0 : 0.0) : S.f0[lane] / nf;
  __syncwarp();
  int kd = 1;
  for (int col = 0; col < NS; ++col) {
    if (lane < NS) {
      S.ys[lane] = S.rhoY[lane] + eps * S.Q[col * NS + lane];
      S.yk[lane] = S.ys[lane] / rho;
      S.ta[lane] = S.yk[lane] / __ldg(m.mw + lane);
    }
    const double imw = warp_sum_ta<NS>(S);
    const double ts = warp_temperature<NS>(T, imw, E, m, S, lane);
    warp_source<NS>(ts, S.ys, m, gibbs_needed, S, lane);
    if (lane < NS) S.w[lane] = (S.omega[lane] - S.f0[lane]) / eps;
    __syncwarp();
    for (int row = 0; row <= col; ++row) {
      const double hij = warp_dot<NS>(S, S.Q + row * NS, S.w, lane);
      if (lane == 0) S.H[row * NS + col] = hij;
      if (lane < NS) S.w[lane] -= hij * S.Q[row * NS + lane];
      __syncwarp();
    }
    double hn = sqrt(fmax(warp_dot<NS>(S, S.w, S.w, lane), 0.0));
    if (col + 1 < NS && lane == 0) S.H[(col + 1) * NS + col] = hn;
    if (col + 1 < 4) {
      if (hn < 1e-30) hn = 1e-30;
      if (lane < NS) S.Q[(col + 1) * NS + lane] = S.w[lane] / hn;
      __syncwarp();
      kd = col + 2;
      continue;
    }
    if (hn > 1e-30 && col + 1 < NS) {
      if (lane < NS) S.Q[(col + 1) * NS + lane] = S.w[lane] / hn;
      __syncwarp();
      kd = col + 2;
    } else {
      kd = col + 1;
      break;
    }
  }
  __syncwarp();
  return kd;
}

// One stage on the Krylov basis: g = Q^T f, sol = (I - h gamma H)^-1 g (LU in S.lhs), d = g - sol
// (stages 1 and 2) or sol - g (stages 3 and 4, as the reference forms it), k = f - Q d.
template <int NS>
__device__ __forceinline__ void warp_krylov_stage(KrylovShared<NS> &S, int kd, bool flip, double *k, int lane) {
  for (int q = 0; q < kd; ++q) {
    const double d = warp_dot<NS>(S, S.Q + q * NS, S.f, lane);
    if (lane == 0) S.g[q] = S.sol[q] = d;
  }
  __syncwarp();
  if (lane == 0) {
    lu_solve_n(S.lhs, S.piv, S.sol, kd);
    for (int q = 0; q < kd; ++q) S.g[q] = flip ? S.sol[q] - S.g[q] : S.g[q] - S.sol[q];
  }
  __syncwarp();
  if (lane < NS) {
    double sum = 0;
    for (int q = 0; q < kd; ++q) sum += S.Q[q * NS + lane] * S.g[q];
    k[lane] = S.f[lane] - sum;
  }
  __syncwarp();
}

// d omega_r / d (rho Y)_c from the rates of progress in S.q1/S.q2 (compute_chem_src_jacobian,
// src/ConstVolumeReactor.cpp:1739-1758; its diagonal is compute_chem_src_jacobian_diagonal).
template <int NS>
__device__ __forceinline__ double jacobian_entry(int r, int c, const ReactorShared<NS> &S, const Mech &m) {
  double zz = 0;
  if (S.rhoY[c] > 1e-30) {
    for (int q = 0; q < m.n_reac; ++q) {
      const int fr = __ldg(m.stoi_f + q * NS + r), br = __ldg(m.stoi_b + q * NS + r);
      const int fc = __ldg(m.stoi_f + q * NS + c), bc = __ldg(m.stoi_b + q * NS + c);
      zz += (br - fr) * (fc * S.q1[q] - bc * S.q2[q]);
    }
    zz /= S.rhoY[c];
  }
  return zz * 1e+3 * __ldg(m.mw + r);
}

template <int NS, bool KRYLOV>
__global__ void __launch_bounds__(32 * kReactorWarps) k_reactor_advance(cb2_reactor *R, int n, Mech m,
                                                                        int max_attempts, double rtol, double atol) {
  using namespace rok4e;
  using SH = std::conditional_t<KRYLOV, KrylovShared<NS>, ReactorShared<NS>>;
  __shared__ SH smem[kReactorWarps];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int id = blockIdx.x * kReactorWarps + wid;
  if (id >= n) return;  // warp-uniform
  SH &S = smem[wid];
  double time = R[id].time, t_end = R[id].t_end, hh = R[id].h, err_last = R[id].err_last, T = R[id].T;
  double pr = R[id].p;
  int step = R[id].step, n_reject = R[id].n_reject, status = R[id].status;
  if (status || time >= t_end) return;
  const double rho = R[id].rho, E = R[id].E;
  if (lane < NS) S.rhoY[lane] = R[id].rhoY[lane];
  __syncwarp();
  const bool gibbs_needed = mech_needs_gibbs(m);
  for (int a = 0; a < max_attempts && time < t_end; ++a) {
    warp_source<NS>(T, S.rhoY, m, gibbs_needed, S, lane);
    const double h = fmin(hh, t_end - time);
    if (!(h > 0) || !isfinite(h)) {
      status |= CB2_REACTOR_NONPHYSICAL;
      break;
    }
    double imw = 0, ts = 0;
    if constexpr (KRYLOV) {
      // build_arnoldi = 1 (src/ConstVolumeReactor.cpp:446-594)
      if (lane < NS) S.f0[lane] = S.omega[lane];
      __syncwarp();
      const int kd = warp_arnoldi<NS>(T, rho, E, m, gibbs_needed, S, lane);
      for (int e = lane; e < kd * kd; e += 32) {
        const int i = e / kd, j = e % kd;
        const double hv = S.H[i * NS + j];
        S.lhs[e] = i == j ? 1.0 - h * gamma * hv : -h * gamma * hv;
      }
      __syncwarp();
      warp_lu_n(S, kd, lane);
      if (lane < NS) S.f[lane] = S.f0[lane];
      __syncwarp();
      warp_krylov_stage<NS>(S, kd, false, S.k1, lane);
      if (lane < NS) {
        S.ys[lane] = S.rhoY[lane] + h * a21 * S.k1[lane];
        S.yk[lane] = S.ys[lane] / rho;
        S.ta[lane] = S.yk[lane] / __ldg(m.mw + lane);
      }
      imw = warp_sum_ta<NS>(S);
      ts = warp_temperature<NS>(T, imw, E, m, S, lane);
      warp_source<NS>(ts, S.ys, m, gibbs_needed, S, lane);
      if (lane < NS) S.f[lane] = S.omega[lane] + g21 * S.k1[lane];
      __syncwarp();
      warp_krylov_stage<NS>(S, kd, false, S.k2, lane);
      if (lane < NS) S.k2[lane] = S.k2[lane] - g21 * S.k1[lane];
      __syncwarp();
      if (lane < NS) {
        S.ys[lane] = S.rhoY[lane] + h * (a31 * S.k1[lane] + a32 * S.k2[lane]);
        S.yk[lane] = S.ys[lane] / rho;
        S.ta[lane] = S.yk[lane] / __ldg(m.mw + lane);
      }
      imw = warp_sum_ta<NS>(S);
      ts = warp_temperature<NS>(ts, imw, E, m, S, lane);
      warp_source<NS>(ts, S.ys, m, gibbs_needed, S, lane);
      if (lane < NS) S.f[lane] = S.omega[lane] + g31 * S.k1[lane] + g32 * S.k2[lane];
      __syncwarp();
      warp_krylov_stage<NS>(S, kd, true, S.k3, lane);
      if (lane < NS) S.k3[lane] = S.k3[lane] - g31 * S.k1[lane] - g32 * S.k2[lane];
      __syncwarp();
      if (lane < NS) S.f[lane] = S.omega[lane] + g41 * S.k1[lane] + g42 * S.k2[lane] + g43 * S.k3[lane];
      __syncwarp();
      warp_krylov_stage<NS>(S, kd, true, S.k4, lane);
      if (lane < NS) S.k4[lane] = S.k4[lane] - g41 * S.k1[lane] - g42 * S.k2[lane] - g43 * S.k3[lane];
      __syncwarp();
    } else {
      // lhs = I - h gamma J
      for (int e = lane; e < NS * NS; e += 32) {
        const int r = e / NS, c = e % NS;
        const double j = jacobian_entry<NS>(r, c, S, m);
        S.lhs[e] = r == c ? 1.0 - h * gamma * j : -h * gamma * j;
      }
      __syncwarp();
      warp_lu<NS>(S, lane);
      // stage 1
      if (lane < NS) S.k1[lane] = S.omega[lane];
      warp_solve<NS>(S, S.k1, lane);
      // stage 2
      if (lane < NS) {
        S.ys[lane] = S.rhoY[lane] + h * a21 * S.k1[lane];
        S.yk[lane] = S.ys[lane] / rho;
        S.ta[lane] = S.yk[lane] / __ldg(m.mw + lane);
      }
      imw = warp_sum_ta<NS>(S);
      ts = warp_temperature<NS>(T, imw, E, m, S, lane);
      warp_source<NS>(ts, S.ys, m, gibbs_needed, S, lane);
      if (lane < NS) S.k2[lane] = S.omega[lane] + g21 * S.k1[lane];
      warp_solve<NS>(S, S.k2, lane);
      if (lane < NS) S.k2[lane] -= g21 * S.k1[lane];
      __syncwarp();
      // stage 3
      if (lane < NS) {
        S.ys[lane] = S.rhoY[lane] + h * (a31 * S.k1[lane] + a32 * S.k2[lane]);
        S.yk[lane] = S.ys[lane] / rho;
        S.ta[lane] = S.yk[lane] / __ldg(m.mw + lane);
      }
      imw = warp_sum_ta<NS>(S);
      ts = warp_temperature<NS>(ts, imw, E, m, S, lane);
      warp_source<NS>(ts, S.ys, m, gibbs_needed, S, lane);
      if (lane < NS) S.k3[lane] = S.omega[lane] + g31 * S.k1[lane] + g32 * S.k2[lane];
      warp_solve<NS>(S, S.k3, lane);
      if (lane < NS) S.k3[lane] -= g31 * S.k1[lane] + g32 * S.k2[lane];
      __syncwarp();
      // stage 4 (the source of stage 3 again)
      if (lane < NS) S.k4[lane] = S.omega[lane] + g41 * S.k1[lane] + g42 * S.k2[lane] + g43 * S.k3[lane];
      warp_solve<NS>(S, S.k4, lane);
      if (lane < NS) S.k4[lane] -= g41 * S.k1[lane] + g42 * S.k2[lane] + g43 * S.k3[lane];
      __syncwarp();
    }
    // embedded error estimate and step control
    if (lane < NS) {
      S.ys[lane] = S.rhoY[lane] + h * (b1 * S.k1[lane] + b2 * S.k2[lane] + b4 * S.k4[lane]);
      double dy = h * (e1 * S.k1[lane] + e2 * S.k2[lane] + e3 * S.k3[lane] + e4 * S.k4[lane]);
      dy /= rtol * S.ys[lane] + atol;
      S.ta[lane] = dy * dy;
    }
    double err = warp_sum_ta<NS>(S);
    err = sqrt(err / NS);
    double h_next = h;
    if (step > 0) h_next *= fmin(5.0, fmax(0.2, 0.8 * pow(err_last, 0.1) * pow(err + 1e-20, -0.175)));
    else if (err > 1) h_next *= 0.2;
    if (err <= 1) {
      if (lane < NS) {
        S.rhoY[lane] = S.ys[lane];
        S.yk[lane] = S.ys[lane] / rho;
        S.ta[lane] = S.yk[lane] / __ldg(m.mw + lane);
      }
      imw = warp_sum_ta<NS>(S);
      time += h;
      err_last = err;
      hh = h_next;
      T = warp_temperature<NS>(T, imw, E, m, S, lane);
      pr = rho * kRu * imw * T;
      ++step;
      if (!(T > 0) || !isfinite(T)) {
        status |= CB2_REACTOR_NONPHYSICAL;
        break;
      }
    } else {
      hh = h_next;
      ++n_reject;
    }
  }
  __syncwarp();
  if (lane < NS) R[id].rhoY[lane] = S.rhoY[lane];
  if (lane == 0) {
    if (time >= t_end) status |= CB2_REACTOR_DONE;
    R[id].time = time;
    R[id].h = hh;
    R[id].err_last = err_last;
    R[id].T = T;
    R[id].p = pr;
    R[id].step = step;
    R[id].n_reject = n_reject;
    R[id].status = status;
  }
}

// ---- fixed-step forms, one warp per reactor -------------------------------------------------
// const_volume_reactor with advance_scheme = 0 (src/ConstVolumeReactor.cpp:403-441: the source,
// then for implicit_method 1 (EPI, :1779-1793) omega <- (I - dt J)^-1 omega by the same LU, for
// implicit_method 2 (DA, :1795-1800) omega_l <- omega_l / (1 - dt J_ll); rhoY += omega dt clipped
// at 0, renormalised to rho when conserve_mass_corefl is set) or advance_scheme = 3 (:708-745, the
// explicit three-stage Runge-Kutta, two more source evaluations at the stage temperatures); then
// T by update_t, p, time += dt (:747-763).  dt is the reactor's h, left unchanged.
template <int NS>
__global__ void __launch_bounds__(32 * kReactorWarps) k_reactor_fixed(cb2_reactor *R, int n, Mech m, int max_steps,
                                                                      int scheme, bool conserve) {
  __shared__ ReactorShared<NS> smem[kReactorWarps];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int id = blockIdx.x * kReactorWarps + wid;
  if (id >= n) return;  // warp-uniform
  ReactorShared<NS> &S = smem[wid];
  double time = R[id].time, T = R[id].T, pr = R[id].p;
  const double t_end = R[id].t_end, dt = R[id].h;
  int step = R[id].step, status = R[id].status;
  if (status || time >= t_end) return;
  const double rho = R[id].rho, E = R[id].E;
  if (lane < NS) S.rhoY[lane] = R[id].rhoY[lane];
  __syncwarp();
  if (!(dt > 0) || !isfinite(dt)) {
    if (lane == 0) R[id].status = status | CB2_REACTOR_NONPHYSICAL;
    return;
  }
  const bool gibbs_needed = mech_needs_gibbs(m);
  for (int a = 0; a < max_steps && time < t_end; ++a) {
    warp_source<NS>(T, S.rhoY, m, gibbs_needed, S, lane);
    if (scheme <= CB2_REACTOR_DA) {
      if (scheme == CB2_REACTOR_EPI) {
        for (int e = lane; e < NS * NS; e += 32) {
          const int r = e / NS, c = e % NS;
          S.lhs[e] = (r == c ? 1.0 : 0.0) - dt * jacobian_entry<NS>(r, c, S, m);
        }
        __syncwarp();
        warp_lu<NS>(S, lane);
        warp_solve<NS>(S, S.omega, lane);
      } else if (scheme == CB2_REACTOR_DA) {
        if (lane < NS) S.omega[lane] /= 1 - dt * jacobian_entry<NS>(lane, lane, S, m);
        __syncwarp();
      }
      if (lane < NS) {
        const double v = S.rhoY[lane] + S.omega[lane] * dt;
        S.rhoY[lane] = v < 0 ? 0.0 : v;
        S.ta[lane] = S.rhoY[lane];
      }
      const double sum = warp_sum_ta<NS>(S);
      if (lane < NS) {
        S.yk[lane] = S.rhoY[lane] / (conserve ? sum : rho);
        if (conserve) S.rhoY[lane] = S.yk[lane] * rho;
      }
    } else {
      if (lane < NS) {
        S.ys[lane] = S.rhoY[lane] + S.omega[lane] * dt;
        S.yk[lane] = S.ys[lane] / rho;
        S.ta[lane] = S.yk[lane] / __ldg(m.mw + lane);
      }
      double imw = warp_sum_ta<NS>(S);
      double ts = warp_temperature<NS>(T, imw, E, m, S, lane);
      warp_source<NS>(ts, S.ys, m, gibbs_needed, S, lane);
      if (lane < NS) {
        S.ys[lane] = 0.75 * S.rhoY[lane] + 0.25 * (S.ys[lane] + S.omega[lane] * dt);
        S.yk[lane] = S.ys[lane] / rho;
        S.ta[lane] = S.yk[lane] / __ldg(m.mw + lane);
      }
      imw = warp_sum_ta<NS>(S);
      ts = warp_temperature<NS>(ts, imw, E, m, S, lane);
      warp_source<NS>(ts, S.ys, m, gibbs_needed, S, lane);
      if (lane < NS) {
        const double v = (S.rhoY[lane] + 2.0 * (S.ys[lane] + S.omega[lane] * dt)) / 3.0;
        S.rhoY[lane] = v < 0 ? 0.0 : v;
        S.yk[lane] = S.rhoY[lane] / rho;
      }
    }
    if (lane < NS) S.ta[lane] = S.yk[lane] / __ldg(m.mw + lane);
    const double imw = warp_sum_ta<NS>(S);
    T = warp_temperature<NS>(T, imw, E, m, S, lane);
    pr = rho * kRu * imw * T;
    time += dt;
    ++step;
    if (!(T > 0) || !isfinite(T)) {
      status |= CB2_REACTOR_NONPHYSICAL;
      break;
    }
  }
  __syncwarp();
  if (lane < NS) R[id].rhoY[lane] = S.rhoY[lane];
  if (lane == 0) {
    if (time >= t_end) status |= CB2_REACTOR_DONE;
    R[id].time = time;
    R[id].T = T;
    R[id].p = pr;
    R[id].step = step;
    R[id].status = status;
  }
}

int launch_reactor_fixed(const Param &p, cb2_reactor *r, int n, int max_steps, int scheme, cudaStream_t s) {
  const int form = scheme & 0xf;
  const bool conserve = (scheme & CB2_REACTOR_CONSERVE_MASS) != 0;
  if (form > CB2_REACTOR_RK3 || (scheme & ~(0xf | CB2_REACTOR_CONSERVE_MASS)) ||
      (conserve && form == CB2_REACTOR_RK3))
    return CB2_ERR_INVALID;
  const unsigned blocks = (unsigned)((n + kReactorWarps - 1) / kReactorWarps);
  ProfScope prof("reactor_fixed", s);
  switch (p.n_spec) {
    case 5: k_reactor_fixed<5><<<blocks, 32 * kReactorWarps, 0, s>>>(r, n, p.mech, max_steps, form, conserve); break;
    case 9: k_reactor_fixed<9><<<blocks, 32 * kReactorWarps, 0, s>>>(r, n, p.mech, max_steps, form, conserve); break;
    default: return CB2_ERR_UNSUPPORTED;
  }
  return check_launch();
}

int launch_reactor_setup(const Param &p, cb2_reactor *r, int n, const double *T0, const double *p0,
                         const double *Y, const double *t_end, double h0, cudaStream_t s) {
  const unsigned blocks = (unsigned)((n + kReactorThreads - 1) / kReactorThreads);
  ProfScope prof("reactor_setup", s);
  switch (p.n_spec) {
    case 5: k_reactor_setup<5><<<blocks, kReactorThreads, 0, s>>>(r, n, p.mech, T0, p0, Y, t_end, h0); break;
    case 9: k_reactor_setup<9><<<blocks, kReactorThreads, 0, s>>>(r, n, p.mech, T0, p0, Y, t_end, h0); break;
    default: return CB2_ERR_UNSUPPORTED;
  }
  return check_launch();
}

int launch_reactor_advance(const Param &p, cb2_reactor *r, int n, int max_attempts, double rtol, double atol,
                           cudaStream_t s, bool krylov) {
  const unsigned blocks = (unsigned)((n + kReactorWarps - 1) / kReactorWarps);
  ProfScope prof(krylov ? "reactor_advance_krylov" : "reactor_advance", s);
  const unsigned th = 32 * kReactorWarps;
  switch (p.n_spec * 2 + (krylov ? 1 : 0)) {
    case 10: k_reactor_advance<5, false><<<blocks, th, 0, s>>>(r, n, p.mech, max_attempts, rtol, atol); break;
    case 11: k_reactor_advance<5, true><<<blocks, th, 0, s>>>(r, n, p.mech, max_attempts, rtol, atol); break;
    case 18: k_reactor_advance<9, false><<<blocks, th, 0, s>>>(r, n, p.mech, max_attempts, rtol, atol); break;
    case 19: k_reactor_advance<9, true><<<blocks, th, 0, s>>>(r, n, p.mech, max_attempts, rtol, atol); break;
    default: return CB2_ERR_UNSUPPORTED;
  }
  return check_launch();
}

}  // namespace cb2
