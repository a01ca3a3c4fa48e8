// FP64 host oracle of the 0-D constant-volume reactor (TEST INFRASTRUCTURE ONLY).
//
// Restates const_volume_reactor with advance_scheme = 1 (ROK4E), build_arnoldi = 0 and
// adaptive_time_step = 1 (src/ConstVolumeReactor.cpp:385-700) on the oracle's own chemistry:
//   source       compute_src (:925-951): c = rhoY / W * 1e-3, rates of progress, then
//                omega = (creation - destruction) * 1e3 W (chemical_source, :1720-1737)
//   Jacobian     compute_chem_src_jacobian (:1739-1758)
//   LU           lu_decomp / lu_to_solution (:1802-1857)
//   temperature  update_t (:1456-1479)
//   setup        rho = p / (T R_u imw), rhoY = rho Y, E = sum Y h(T) - p / rho (:61-66, :328-336)
// The ROK4E coefficients are the published table (src/Define.h:33-48 lists the same numbers).
// reactor_advance_fixed restates the fixed-step forms (explicit, EPI, DA, explicit RK3).
#include <algorithm>
#include <cmath>
#include <vector>
#include "oracle.hpp"

namespace oracle {

namespace {
constexpr double kGamma = 0.572816062482135;
constexpr double kA21 = 0.432364435748567, kA31 = -0.51421131687617, kA32 = 1.38227114461736;
constexpr double kG21 = -0.602765307997356 / kGamma, kG31 = -1.389195789724843 / kGamma,
                 kG32 = 1.072950969011413 / kGamma, kG41 = 0.992356412977094 / kGamma,
                 kG42 = -1.390032613873701 / kGamma, kG43 = -0.440875890223325 / kGamma;
constexpr double kB1 = 0.194335256262729, kB2 = 0.483167813989227, kB4 = 0.322496929748044;
constexpr double kE1 = -0.217819895945721 - kB1, kE2 = 1.03130847478467 - kB2, kE3 = 0.186511421161047,
                 kE4 = -kB4;

void source(const Mechanism &m, double t, const std::vector<double> &rhoY, std::vector<double> &q1,
            std::vector<double> &q2, std::vector<double> &omega) {
  const int ns = m.n_spec, nr = m.n_reac;
  double c[16];
  for (int l = 0; l < ns; ++l) c[l] = rhoY[l] / m.mw[l] * 1e-3;
  reaction_rates(m, t, c, q1.data(), q2.data());
  for (int i = 0; i < ns; ++i) {
    double creation = 0, destruction = 0;
    for (int j = 0; j < nr; ++j) {
      creation += q2[j] * m.stoi_f[j * ns + i] + q1[j] * m.stoi_b[j * ns + i];
      destruction += q1[j] * m.stoi_f[j * ns + i] + q2[j] * m.stoi_b[j * ns + i];
    }
    creation *= 1e+3 * m.mw[i];
    destruction *= 1e+3 * m.mw[i];
    omega[i] = creation - destruction;
  }
}

double temperature(const Mechanism &m, double t0, double imw, const std::vector<double> &y, double E) {
  const int ns = m.n_spec;
  double t = t0;
  const double R = R_u * imw;
  double err = 1e+6;
  int iter = 0;
  std::vector<double> h(ns), cp(ns);
  while (err > 1e-8 && iter++ < 100) {
    nasa7_h_cp(t, m, h.data(), cp.data());
    double cpt = 0, ht = 0;
    for (int l = 0; l < ns; ++l) {
      cpt += cp[l] * y[l];
      ht += h[l] * y[l];
    }
    const double et = ht - R * t;
    const double cv = cpt - R;
    const double t1 = t - (et - E) / cv;
    err = std::abs(1 - t1 / t);
    t = t1;
  }
  return t;
}

void lu(std::vector<double> &a, std::vector<int> &piv, int n) {
  for (int c = 0; c < n; ++c) {
    int ik = c;
    for (int r = c; r < n; ++r) {
      for (int t = 0; t < c; ++t) a[r * n + c] -= a[r * n + t] * a[t * n + c];
      if (std::abs(a[r * n + c]) > std::abs(a[ik * n + c])) ik = r;
    }
    piv[c] = ik;
    if (ik != c)
      for (int t = 0; t < n; ++t) std::swap(a[ik * n + t], a[c * n + t]);
    for (int q = c + 1; q < n; ++q)
      for (int t = 0; t < c; ++t) a[c * n + q] -= a[c * n + t] * a[t * n + q];
    for (int r = c + 1; r < n; ++r) a[r * n + c] /= a[c * n + c];
  }
}

void lu_solve(const std::vector<double> &a, const std::vector<int> &piv, std::vector<double> &b, int n) {
  for (int r = 0; r < n; ++r)
    if (piv[r] != r) std::swap(b[piv[r]], b[r]);
  for (int r = 1; r < n; ++r)
    for (int t = 0; t < r; ++t) b[r] -= a[r * n + t] * b[t];
  b[n - 1] /= a[n * n - 1];
  for (int r = n - 2; r >= 0; --r) {
    for (int t = r + 1; t < n; ++t) b[r] -= a[r * n + t] * b[t];
    b[r] /= a[r * n + r];
  }
}
// buildArnoldi (src/ConstVolumeReactor.cpp:1858-1930) with the Krylov limit n_spec and minimum
// 4: q0 = f0 / |f0| (e_0 when |f0| < 1e-30); column c: w = (omega(T', rhoY + eps q_c) - f0) / eps
// with eps = 1e-6 (1 + |rhoY|) and T' the Newton temperature of the perturbed state, modified
// Gram-Schmidt into H(0..c, c), H(c+1, c) = |w|; a new basis vector while c + 1 < 4 (|w| clamped
// at 1e-30) or |w| > 1e-30 and c + 1 < n_spec.  Q and H are n_spec x n_spec, row-major, H zeroed.
int arnoldi(const Mechanism &m, const std::vector<double> &rhoY, const std::vector<double> &f0, double T, double rho,
            double E, std::vector<double> &Q, std::vector<double> &H) {
  const int ns = m.n_spec, km = ns;
  auto dot = [&](const double *a, const double *b) {
    double s = 0;
    for (int l = 0; l < ns; ++l) s += a[l] * b[l];
    return s;
  };
  auto norm = [&](const double *a) { return std::sqrt(std::max(dot(a, a), 0.0)); };
  std::fill(Q.begin(), Q.end(), 0.0);
  std::fill(H.begin(), H.end(), 0.0);
  const double eps = 1e-6 * (1 + norm(rhoY.data()));
  const double nf = norm(f0.data());
  if (nf < 1e-30) Q[0] = 1.0;
  else
    for (int l = 0; l < ns; ++l) Q[l] = f0[l] / nf;
  int kd = 1;
  std::vector<double> ye(ns), yk(ns), q1(m.n_reac), q2(m.n_reac), fe(ns), w(ns);
  for (int col = 0; col < km; ++col) {
    double imw = 0;
    for (int l = 0; l < ns; ++l) {
      ye[l] = rhoY[l] + eps * Q[col * ns + l];
      yk[l] = ye[l] / rho;
      imw += yk[l] / m.mw[l];
    }
    const double ts = temperature(m, T, imw, yk, E);
    source(m, ts, ye, q1, q2, fe);
    for (int l = 0; l < ns; ++l) w[l] = (fe[l] - f0[l]) / eps;
    for (int row = 0; row <= col; ++row) {
      const double hij = dot(&Q[row * ns], w.data());
      H[row * km + col] = hij;
      for (int l = 0; l < ns; ++l) w[l] -= hij * Q[row * ns + l];
    }
    double hn = norm(w.data());
    if (col + 1 < km) H[(col + 1) * km + col] = hn;
    if (col + 1 < 4) {
      if (hn < 1e-30) hn = 1e-30;
      for (int l = 0; l < ns; ++l) Q[(col + 1) * ns + l] = w[l] / hn;
      kd = col + 2;
      continue;
    }
    if (hn > 1e-30 && col + 1 < km) {
      for (int l = 0; l < ns; ++l) Q[(col + 1) * ns + l] = w[l] / hn;
      kd = col + 2;
    } else {
      kd = col + 1;
      break;
    }
  }
  return kd;
}
}  // namespace

void reactor_setup(const Mechanism &m, double T0, double p0, const double *Y, double t_end, double h0,
                   ReactorState &st) {
  const int ns = m.n_spec;
  double imw = 0;
  for (int l = 0; l < ns; ++l) imw += Y[l] / m.mw[l];
  const double rho = p0 / (T0 * R_u * imw);
  std::vector<double> h(ns), cp(ns);
  nasa7_h_cp(T0, m, h.data(), cp.data());
  double E = 0;
  st.rhoY.assign(ns, 0.0);
  for (int l = 0; l < ns; ++l) {
    st.rhoY[l] = Y[l] * rho;
    E += Y[l] * h[l];
  }
  E -= p0 / rho;
  st.rho = rho;
  st.E = E;
  st.T = T0;
  st.p = p0;
  st.time = 0;
  st.t_end = t_end;
  st.h = h0;
  st.err_last = 0;
  st.step = st.n_reject = st.status = 0;
}

void reactor_advance(const Mechanism &m, ReactorState &st, int max_attempts, double rtol, double atol, bool krylov) {
  const int ns = m.n_spec, nr = m.n_reac;
  if (st.status || st.time >= st.t_end) return;
  std::vector<double> &rhoY = st.rhoY;
  std::vector<double> q1(nr), q2(nr), omega(ns), k1(ns), k2(ns), k3(ns), k4(ns), ys(ns), yk(ns), lhs(ns * ns);
  std::vector<int> piv(ns);
  std::vector<double> Q(ns * ns), H(ns * ns), f(ns);
  const double rho = st.rho, E = st.E;
  for (int a = 0; a < max_attempts && st.time < st.t_end; ++a) {
    source(m, st.T, rhoY, q1, q2, omega);
    const double h = std::min(st.h, st.t_end - st.time);
    if (!(h > 0) || !std::isfinite(h)) {
      st.status |= 2;
      break;
    }
    double imw = 0, ts = 0;
    if (krylov) {
      // build_arnoldi = 1 (:446-594): Arnoldi basis Q (Krylov dimension kd <= n_spec) of
      // finite-difference Jacobian products, LU of I - h gamma H, each stage projected, solved
      // and projected back; stages 3 and 4 take the correction as solve(g) - g, stages 1 and 2 as
      // g - solve(g), as the reference does
      const int kd = arnoldi(m, rhoY, omega, st.T, rho, E, Q, H);
      std::vector<double> L(kd * kd);
      std::vector<int> pk(kd);
      for (int i = 0; i < kd; ++i)
        for (int j = 0; j < kd; ++j)
          L[i * kd + j] = i == j ? 1.0 - h * kGamma * H[i * ns + j] : -h * kGamma * H[i * ns + j];
      lu(L, pk, kd);
      auto stage = [&](const std::vector<double> &f, bool flip, std::vector<double> &kk) {
        std::vector<double> g(kd), sol(kd);
        for (int q = 0; q < kd; ++q) {
          double d = 0;
          for (int l = 0; l < ns; ++l) d += Q[q * ns + l] * f[l];
          g[q] = sol[q] = d;
        }
        lu_solve(L, pk, sol, kd);
        for (int q = 0; q < kd; ++q) g[q] = flip ? sol[q] - g[q] : g[q] - sol[q];
        for (int l = 0; l < ns; ++l) {
          double sum = 0;
          for (int q = 0; q < kd; ++q) sum += Q[q * ns + l] * g[q];
          kk[l] = f[l] - sum;
        }
      };
      stage(omega, false, k1);
      imw = 0;
      for (int l = 0; l < ns; ++l) {
        ys[l] = rhoY[l] + h * kA21 * k1[l];
        yk[l] = ys[l] / rho;
        imw += yk[l] / m.mw[l];
      }
      ts = temperature(m, st.T, imw, yk, E);
      source(m, ts, ys, q1, q2, omega);
      for (int l = 0; l < ns; ++l) f[l] = omega[l] + kG21 * k1[l];
      stage(f, false, k2);
      for (int l = 0; l < ns; ++l) k2[l] = k2[l] - kG21 * k1[l];
      imw = 0;
      for (int l = 0; l < ns; ++l) {
        ys[l] = rhoY[l] + h * (kA31 * k1[l] + kA32 * k2[l]);
        yk[l] = ys[l] / rho;
        imw += yk[l] / m.mw[l];
      }
      ts = temperature(m, ts, imw, yk, E);
      source(m, ts, ys, q1, q2, omega);
      for (int l = 0; l < ns; ++l) f[l] = omega[l] + kG31 * k1[l] + kG32 * k2[l];
      stage(f, true, k3);
      for (int l = 0; l < ns; ++l) k3[l] = k3[l] - kG31 * k1[l] - kG32 * k2[l];
      for (int l = 0; l < ns; ++l) f[l] = omega[l] + kG41 * k1[l] + kG42 * k2[l] + kG43 * k3[l];
      stage(f, true, k4);
      for (int l = 0; l < ns; ++l) k4[l] = k4[l] - kG41 * k1[l] - kG42 * k2[l] - kG43 * k3[l];
    } else {
      for (int r = 0; r < ns; ++r)
        for (int c = 0; c < ns; ++c) {
          double zz = 0;
          if (rhoY[c] > 1e-30) {
            for (int q = 0; q < nr; ++q)
              zz += (m.stoi_b[q * ns + r] - m.stoi_f[q * ns + r]) *
                    (m.stoi_f[q * ns + c] * q1[q] - m.stoi_b[q * ns + c] * q2[q]);
            zz /= rhoY[c];
          }
          const double j = zz * 1e+3 * m.mw[r];
          lhs[r * ns + c] = r == c ? 1.0 - h * kGamma * j : -h * kGamma * j;
        }
      lu(lhs, piv, ns);
      k1 = omega;
      lu_solve(lhs, piv, k1, ns);
      imw = 0;
      for (int l = 0; l < ns; ++l) {
        ys[l] = rhoY[l] + h * kA21 * k1[l];
        yk[l] = ys[l] / rho;
        imw += yk[l] / m.mw[l];
      }
      ts = temperature(m, st.T, imw, yk, E);
      source(m, ts, ys, q1, q2, omega);
      for (int l = 0; l < ns; ++l) k2[l] = omega[l] + kG21 * k1[l];
      lu_solve(lhs, piv, k2, ns);
      for (int l = 0; l < ns; ++l) k2[l] -= kG21 * k1[l];
      imw = 0;
      for (int l = 0; l < ns; ++l) {
        ys[l] = rhoY[l] + h * (kA31 * k1[l] + kA32 * k2[l]);
        yk[l] = ys[l] / rho;
        imw += yk[l] / m.mw[l];
      }
      ts = temperature(m, ts, imw, yk, E);
      source(m, ts, ys, q1, q2, omega);
      for (int l = 0; l < ns; ++l) k3[l] = omega[l] + kG31 * k1[l] + kG32 * k2[l];
      lu_solve(lhs, piv, k3, ns);
      for (int l = 0; l < ns; ++l) k3[l] -= kG31 * k1[l] + kG32 * k2[l];
      for (int l = 0; l < ns; ++l) k4[l] = omega[l] + kG41 * k1[l] + kG42 * k2[l] + kG43 * k3[l];
      lu_solve(lhs, piv, k4, ns);
      for (int l = 0; l < ns; ++l) k4[l] -= kG41 * k1[l] + kG42 * k2[l] + kG43 * k3[l];
    }
    double err = 0;
    for (int l = 0; l < ns; ++l) {
      ys[l] = rhoY[l] + h * (kB1 * k1[l] + kB2 * k2[l] + kB4 * k4[l]);
      double dy = h * (kE1 * k1[l] + kE2 * k2[l] + kE3 * k3[l] + kE4 * k4[l]);
      dy /= rtol * ys[l] + atol;
      err += dy * dy;
    }
    err = std::sqrt(err / ns);
    double h_next = h;
    if (st.step > 0)
      h_next *= std::min(5.0, std::max(0.2, 0.8 * std::pow(st.err_last, 0.1) * std::pow(err + 1e-20, -0.175)));
    else if (err > 1)
      h_next *= 0.2;
    if (err <= 1) {
      imw = 0;
      for (int l = 0; l < ns; ++l) {
        rhoY[l] = ys[l];
        yk[l] = ys[l] / rho;
        imw += yk[l] / m.mw[l];
      }
      st.time += h;
      st.err_last = err;
      st.h = h_next;
      st.T = temperature(m, st.T, imw, yk, E);
      st.p = rho * R_u * imw * st.T;
      ++st.step;
      if (!(st.T > 0) || !std::isfinite(st.T)) {
        st.status |= 2;
        break;
      }
    } else {
      st.h = h_next;
      ++st.n_reject;
    }
  }
  if (st.time >= st.t_end) st.status |= 1;
}

// The fixed-step forms of const_volume_reactor with the step st.h: scheme 0 explicit, 1 EPI
// (omega <- (I - dt J)^-1 omega, src/ConstVolumeReactor.cpp:1779-1793), 2 DA (omega_l <- omega_l /
// (1 - dt J_ll), :1795-1800) -- advance_scheme = 0 with implicit_method = scheme, the update and
// the optional conserve_mass_corefl renormalisation of :403-441 -- and 3 the explicit
// three-stage Runge-Kutta of advance_scheme = 3 (:708-745); then T by update_t, p, time += dt
// (:747-763).
void reactor_advance_fixed(const Mechanism &m, ReactorState &st, int max_steps, int scheme, bool conserve) {
  const int ns = m.n_spec, nr = m.n_reac;
  if (st.status || st.time >= st.t_end) return;
  std::vector<double> &rhoY = st.rhoY;
  std::vector<double> q1(nr), q2(nr), omega(ns), yk(ns), yn(ns), lhs(ns * ns);
  std::vector<int> piv(ns);
  const double rho = st.rho, E = st.E, dt = st.h;
  if (!(dt > 0) || !std::isfinite(dt)) {
    st.status |= 2;
    return;
  }
  auto jac = [&](int r, int c) {
    double zz = 0;
    if (rhoY[c] > 1e-30) {
      for (int q = 0; q < nr; ++q)
        zz += (m.stoi_b[q * ns + r] - m.stoi_f[q * ns + r]) *
              (m.stoi_f[q * ns + c] * q1[q] - m.stoi_b[q * ns + c] * q2[q]);
      zz /= rhoY[c];
    }
    return zz * 1e+3 * m.mw[r];
  };
  for (int a = 0; a < max_steps && st.time < st.t_end; ++a) {
    source(m, st.T, rhoY, q1, q2, omega);
    double imw = 0;
    if (scheme <= 2) {
      if (scheme == 1) {
        for (int r = 0; r < ns; ++r)
          for (int c = 0; c < ns; ++c) lhs[r * ns + c] = (r == c ? 1.0 : 0.0) - dt * jac(r, c);
        lu(lhs, piv, ns);
        lu_solve(lhs, piv, omega, ns);
      } else if (scheme == 2) {
        for (int l = 0; l < ns; ++l) omega[l] /= 1 - dt * jac(l, l);
      }
      double sum = 0;
      for (int l = 0; l < ns; ++l) {
        rhoY[l] += omega[l] * dt;
        if (rhoY[l] < 0) rhoY[l] = 0;
        sum += rhoY[l];
      }
      for (int l = 0; l < ns; ++l) {
        yk[l] = rhoY[l] / (conserve ? sum : rho);
        if (conserve) rhoY[l] = yk[l] * rho;
      }
    } else {
      for (int l = 0; l < ns; ++l) {
        yn[l] = rhoY[l] + omega[l] * dt;
        yk[l] = yn[l] / rho;
        imw += yk[l] / m.mw[l];
      }
      double ts = temperature(m, st.T, imw, yk, E);
      source(m, ts, yn, q1, q2, omega);
      imw = 0;
      for (int l = 0; l < ns; ++l) {
        yn[l] = 0.75 * rhoY[l] + 0.25 * (yn[l] + omega[l] * dt);
        yk[l] = yn[l] / rho;
        imw += yk[l] / m.mw[l];
      }
      ts = temperature(m, ts, imw, yk, E);
      source(m, ts, yn, q1, q2, omega);
      for (int l = 0; l < ns; ++l) {
        rhoY[l] = (rhoY[l] + 2.0 * (yn[l] + omega[l] * dt)) / 3.0;
        if (rhoY[l] < 0) rhoY[l] = 0;
      }
      for (int l = 0; l < ns; ++l) yk[l] = rhoY[l] / rho;
    }
    imw = 0;
    for (int l = 0; l < ns; ++l) imw += yk[l] / m.mw[l];
    st.T = temperature(m, st.T, imw, yk, E);
    st.p = rho * R_u * imw * st.T;
    st.time += dt;
    ++st.step;
    if (!(st.T > 0) || !std::isfinite(st.T)) {
      st.status |= 2;
      break;
    }
  }
  if (st.time >= st.t_end) st.status |= 1;
}

}  // namespace oracle
