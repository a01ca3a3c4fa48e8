// Batched 0-D constant-volume reactors: one thread per reactor, FP64 throughout.
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
// numbers src/Define.h:33-48 lists.
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

// omega [kg/(m^3 s)] of a state and the rates of progress q1/q2 of every reaction.
template <int NS>
__device__ __forceinline__ void reactor_source(double t, const double *rhoY, const Mech &m, double *omega,
                                               double *q1, double *q2) {
  double c[NS], cre[NS], des[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) c[s] = rhoY[s] / __ldg(m.mw + s) * 1e-3;
  chem_rates<NS>(t, c, m, cre, des, q1, q2);
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const double w = 1e+3 * __ldg(m.mw + s);
    omega[s] = cre[s] * w - des[s] * w;
  }
}

// T from the internal energy E at fixed composition (Newton from t0).
template <int NS>
__device__ __forceinline__ double reactor_temperature(double t0, double imw, const double *y, double E,
                                                      const Mech &m) {
  double t = t0;
  const double R = kRu * imw;
  double err = 1e+6;
  int iter = 0;
  double h[NS], cp[NS];
  while (err > 1e-8 && iter++ < 100) {
    nasa7_h_cp<NS>(t, m, h, cp);
    double cpt = 0, ht = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      cpt += cp[s] * y[s];
      ht += h[s] * y[s];
    }
    const double et = ht - R * t;
    const double cv = cpt - R;
    const double t1 = t - (et - E) / cv;
    err = fabs(1 - t1 / t);
    t = t1;
  }
  return t;
}

// In-place LU of the N x N row-major matrix a with row pivoting (Crout ordering: column n of L
// and then row n of U), piv[n] = the row swapped into n.
template <int N>
__device__ __forceinline__ void lu_factor(double *a, int *piv) {
  for (int n = 0; n < N; ++n) {
    int ik = n;
    for (int r = n; r < N; ++r) {
      double v = a[r * N + n];
      for (int t = 0; t < n; ++t) v -= a[r * N + t] * a[t * N + n];
      a[r * N + n] = v;
      if (fabs(v) > fabs(a[ik * N + n])) ik = r;
    }
    piv[n] = ik;
    if (ik != n) {
      for (int t = 0; t < N; ++t) {
        const double x = a[ik * N + t];
        a[ik * N + t] = a[n * N + t];
        a[n * N + t] = x;
      }
    }
    for (int c = n + 1; c < N; ++c) {
      double v = a[n * N + c];
      for (int t = 0; t < n; ++t) v -= a[n * N + t] * a[t * N + c];
      a[n * N + c] = v;
    }
    const double d = a[n * N + n];
    for (int r = n + 1; r < N; ++r) a[r * N + n] /= d;
  }
}

template <int N>
__device__ __forceinline__ void lu_solve(const double *a, const int *piv, double *b) {
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
  nasa7_h<NS>(t, m, h);
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

template <int NS>
__global__ void __launch_bounds__(kReactorThreads) k_reactor_advance(cb2_reactor *R, int n, Mech m, int max_attempts,
                                                                     double rtol, double atol) {
  using namespace rok4e;
  const int id = blockIdx.x * kReactorThreads + threadIdx.x;
  if (id >= n) return;
  cb2_reactor st = R[id];
  if (st.status || st.time >= st.t_end) return;
  double rhoY[NS], omega[NS], k1[NS], k2[NS], k3[NS], k4[NS], ys[NS], yk[NS];
  double q1[kMaxReac], q2[kMaxReac], lhs[NS * NS];
  int piv[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s) rhoY[s] = st.rhoY[s];
  const double rho = st.rho, E = st.E;
  for (int a = 0; a < max_attempts && st.time < st.t_end; ++a) {
    reactor_source<NS>(st.T, rhoY, m, omega, q1, q2);
    const double h = fmin(st.h, st.t_end - st.time);
    if (!(h > 0) || !isfinite(h)) {
      st.status |= CB2_REACTOR_NONPHYSICAL;
      break;
    }
    // lhs = I - h gamma J, J from the rates of progress of this state
    for (int r = 0; r < NS; ++r) {
      const double mwr = __ldg(m.mw + r);
      for (int c = 0; c < NS; ++c) {
        double zz = 0;
        if (rhoY[c] > 1e-30) {
          for (int q = 0; q < m.n_reac; ++q) {
            const int fr = __ldg(m.stoi_f + q * NS + r), br = __ldg(m.stoi_b + q * NS + r);
            const int fc = __ldg(m.stoi_f + q * NS + c), bc = __ldg(m.stoi_b + q * NS + c);
            zz += (br - fr) * (fc * q1[q] - bc * q2[q]);
          }
          zz /= rhoY[c];
        }
        const double j = zz * 1e+3 * mwr;
        lhs[r * NS + c] = r == c ? 1.0 - h * gamma * j : -h * gamma * j;
      }
    }
    lu_factor<NS>(lhs, piv);
    // stage 1
#pragma unroll
    for (int s = 0; s < NS; ++s) k1[s] = omega[s];
    lu_solve<NS>(lhs, piv, k1);
    // stage 2
    double imw = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      ys[s] = rhoY[s] + h * a21 * k1[s];
      yk[s] = ys[s] / rho;
      imw += yk[s] / __ldg(m.mw + s);
    }
    double ts = reactor_temperature<NS>(st.T, imw, yk, E, m);
    reactor_source<NS>(ts, ys, m, omega, q1, q2);
#pragma unroll
    for (int s = 0; s < NS; ++s) k2[s] = omega[s] + g21 * k1[s];
    lu_solve<NS>(lhs, piv, k2);
#pragma unroll
    for (int s = 0; s < NS; ++s) k2[s] -= g21 * k1[s];
    // stage 3
    imw = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      ys[s] = rhoY[s] + h * (a31 * k1[s] + a32 * k2[s]);
      yk[s] = ys[s] / rho;
      imw += yk[s] / __ldg(m.mw + s);
    }
    ts = reactor_temperature<NS>(ts, imw, yk, E, m);
    reactor_source<NS>(ts, ys, m, omega, q1, q2);
#pragma unroll
    for (int s = 0; s < NS; ++s) k3[s] = omega[s] + g31 * k1[s] + g32 * k2[s];
    lu_solve<NS>(lhs, piv, k3);
#pragma unroll
    for (int s = 0; s < NS; ++s) k3[s] -= g31 * k1[s] + g32 * k2[s];
    // stage 4 (the source of stage 3 again)
#pragma unroll
    for (int s = 0; s < NS; ++s) k4[s] = omega[s] + g41 * k1[s] + g42 * k2[s] + g43 * k3[s];
    lu_solve<NS>(lhs, piv, k4);
#pragma unroll
    for (int s = 0; s < NS; ++s) k4[s] -= g41 * k1[s] + g42 * k2[s] + g43 * k3[s];
    // embedded error estimate and step control
    double err = 0;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      ys[s] = rhoY[s] + h * (b1 * k1[s] + b2 * k2[s] + b4 * k4[s]);
      double dy = h * (e1 * k1[s] + e2 * k2[s] + e3 * k3[s] + e4 * k4[s]);
      dy /= rtol * ys[s] + atol;
      err += dy * dy;
    }
    err = sqrt(err / NS);
    double h_next = h;
    if (st.step > 0) h_next *= fmin(5.0, fmax(0.2, 0.8 * pow(st.err_last, 0.1) * pow(err + 1e-20, -0.175)));
    else if (err > 1) h_next *= 0.2;
    if (err <= 1) {
      imw = 0;
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        rhoY[s] = ys[s];
        yk[s] = ys[s] / rho;
        imw += yk[s] / __ldg(m.mw + s);
      }
      st.time += h;
      st.err_last = err;
      st.h = h_next;
      st.T = reactor_temperature<NS>(st.T, imw, yk, E, m);
      st.p = rho * kRu * imw * st.T;
      ++st.step;
      if (!(st.T > 0) || !isfinite(st.T)) {
        st.status |= CB2_REACTOR_NONPHYSICAL;
        break;
      }
    } else {
      st.h = h_next;
      ++st.n_reject;
    }
  }
#pragma unroll
  for (int s = 0; s < NS; ++s) st.rhoY[s] = rhoY[s];
  if (st.time >= st.t_end) st.status |= CB2_REACTOR_DONE;
  R[id] = st;
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
                           cudaStream_t s) {
  const unsigned blocks = (unsigned)((n + kReactorThreads - 1) / kReactorThreads);
  ProfScope prof("reactor_advance", s);
  switch (p.n_spec) {
    case 5: k_reactor_advance<5><<<blocks, kReactorThreads, 0, s>>>(r, n, p.mech, max_attempts, rtol, atol); break;
    case 9: k_reactor_advance<9><<<blocks, kReactorThreads, 0, s>>>(r, n, p.mech, max_attempts, rtol, atol); break;
    default: return CB2_ERR_UNSUPPORTED;
  }
  return check_launch();
}

}  // namespace cb2
