// Runs 0-D constant-volume reactors with the reference's own host functions and writes their
// states as JSON: cfd::compute_src, cfd::compute_chem_src_jacobian, cfd::lu_decomp,
// cfd::lu_to_solution and cfd::update_t of src/ConstVolumeReactor.cpp, and the ROK4E
// coefficients of src/Define.h, stepped with the adaptive ROK4E sequence of
// const_volume_reactor (advance_scheme = 1, build_arnoldi = 0, adaptive_time_step = 1,
// src/ConstVolumeReactor.cpp:385-700).
// TEST INFRASTRUCTURE ONLY: built into oracle/_ref/ by oracle/ref_build.py and run by
// tests/golden/make_mech.py to write tests/golden/h2_reactor_runs.json.
//
// Usage (from a directory holding ./input/<files>): dump_reactor <setup-file> <out.json> <n> [fixed]
// With "fixed", every case runs the fixed-step forms instead (advance_fixed below); with
// "krylov", the ROK4E sequence with build_arnoldi = 1.
// Case 0 is the reference's example (T0 = 1000 K, p0 = 202650 Pa, X = 0.295775 H2 /
// 0.147887 O2 / rest N2, 1.2 ms); cases 1..n-1 are seeded (T0, p0, phi) requests to 1 ms.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <string>
#include <vector>
#include "ChemData.h"
#include "Constants.h"
#include "ConstVolumeReactor.h"
#include "Define.h"
#include "Parameter.h"

struct Run {
  std::vector<real> rhoY;
  real rho, E, T, p, time, t_end, h, err_last;
  int step, n_reject;
};

static void advance(const cfd::Species &sp, const cfd::Reaction &re, Run &r, int max_attempts, real rtol,
                    real atol, bool krylov = false) {
  namespace k = cfd::rok4e;
  const int ns = sp.n_spec, nr = re.n_reac;
  std::vector<real> q1(nr), q2(nr), od(ns), om(ns), k1(ns), k2(ns), k3(ns), k4(ns), ys(ns), yk(ns);
  for (int a = 0; a < max_attempts && r.time < r.t_end; ++a) {
    cfd::compute_src(0, r.T, sp, re, r.rhoY, q1, q2, od, om);
    const real h = std::min(r.h, r.t_end - r.time);
    real imw = 0, ts = 0;
    if (krylov) {
      // build_arnoldi = 1 (src/ConstVolumeReactor.cpp:446-594): cfd::buildArnoldi, the LU of
      // I - h gamma H on the Krylov basis, each stage projected, solved and projected back; stages
      // 3 and 4 form the correction as solve(g) - g, stages 1 and 2 as g - solve(g), as there
      constexpr int KM = MAX_SPEC_NUMBER;
      real Q[KM * KM]{}, H[KM * KM]{}, g[KM]{}, b[KM]{}, L[KM * KM]{}, lu[KM * KM]{};
      const int kd = cfd::buildArnoldi(sp, r.rhoY, om.data(), Q, H, KM, 0, r.T, re, r.rho, r.E, 4);
      for (int i = 0; i < kd; ++i)
        for (int j = 0; j < kd; ++j)
          L[i * kd + j] = i == j ? 1.0 - h * k::gamma * H[i * KM + j] : -h * k::gamma * H[i * KM + j];
      auto piv = cfd::lu_decomp(L, kd);
      auto stage = [&](const std::vector<real> &f, bool flip, std::vector<real> &kk) {
        for (int q = 0; q < kd; ++q) {
          real d = 0;
          for (int l = 0; l < ns; ++l) d += Q[q * ns + l] * f[l];
          g[q] = d;
          b[q] = d;
        }
        for (int l = 0; l < kd * kd; ++l) lu[l] = L[l];
        cfd::lu_to_solution(lu, flip ? g : b, kd, piv);
        for (int q = 0; q < kd; ++q) g[q] -= b[q];
        for (int l = 0; l < ns; ++l) {
          real sum = 0;
          for (int q = 0; q < kd; ++q) sum += Q[q * ns + l] * g[q];
          kk[l] = f[l] - sum;
        }
      };
      stage(om, false, k1);
      imw = 0;
      for (int l = 0; l < ns; ++l) {
        ys[l] = r.rhoY[l] + h * k::alpha21 * k1[l];
        yk[l] = ys[l] / r.rho;
        imw += yk[l] / sp.mw[l];
      }
      ts = cfd::update_t(r.T, imw, sp, yk, r.E);
      cfd::compute_src(0, ts, sp, re, ys, q1, q2, od, om);
      std::vector<real> f(ns);
      for (int l = 0; l < ns; ++l) f[l] = om[l] + k::gamma21Gamma * k1[l];
      stage(f, false, k2);
      for (int l = 0; l < ns; ++l) k2[l] = k2[l] - k::gamma21Gamma * k1[l];
      imw = 0;
      for (int l = 0; l < ns; ++l) {
        ys[l] = r.rhoY[l] + h * (k::alpha31 * k1[l] + k::alpha32 * k2[l]);
        yk[l] = ys[l] / r.rho;
        imw += yk[l] / sp.mw[l];
      }
      ts = cfd::update_t(ts, imw, sp, yk, r.E);
      cfd::compute_src(0, ts, sp, re, ys, q1, q2, od, om);
      for (int l = 0; l < ns; ++l) f[l] = om[l] + k::gamma31Gamma * k1[l] + k::gamma32Gamma * k2[l];
      stage(f, true, k3);
      for (int l = 0; l < ns; ++l) k3[l] = k3[l] - k::gamma31Gamma * k1[l] - k::gamma32Gamma * k2[l];
      for (int l = 0; l < ns; ++l)
        f[l] = om[l] + k::gamma41Gamma * k1[l] + k::gamma42Gamma * k2[l] + k::gamma43Gamma * k3[l];
      stage(f, true, k4);
      for (int l = 0; l < ns; ++l)
        k4[l] = k4[l] - k::gamma41Gamma * k1[l] - k::gamma42Gamma * k2[l] - k::gamma43Gamma * k3[l];
    } else {
      auto jac = cfd::compute_chem_src_jacobian(r.rhoY, sp, re, q1, q2);
      std::vector<real> lhs(ns * ns);
      for (int m = 0; m < ns; ++m)
        for (int n = 0; n < ns; ++n)
          lhs[m * ns + n] = m == n ? 1.0 - h * k::gamma * jac[m * ns + n] : -h * k::gamma * jac[m * ns + n];
      auto piv = cfd::lu_decomp(lhs.data(), ns);
      auto solve = [&](std::vector<real> &b) {
        auto l = lhs;
        cfd::lu_to_solution(l.data(), b.data(), ns, piv);
      };
      k1 = om;
      solve(k1);
      imw = 0;
      for (int l = 0; l < ns; ++l) {
        ys[l] = r.rhoY[l] + h * k::alpha21 * k1[l];
        yk[l] = ys[l] / r.rho;
        imw += yk[l] / sp.mw[l];
      }
      ts = cfd::update_t(r.T, imw, sp, yk, r.E);
      cfd::compute_src(0, ts, sp, re, ys, q1, q2, od, om);
      for (int l = 0; l < ns; ++l) k2[l] = om[l] + k::gamma21Gamma * k1[l];
      solve(k2);
      for (int l = 0; l < ns; ++l) k2[l] -= k::gamma21Gamma * k1[l];
      imw = 0;
      for (int l = 0; l < ns; ++l) {
        ys[l] = r.rhoY[l] + h * (k::alpha31 * k1[l] + k::alpha32 * k2[l]);
        yk[l] = ys[l] / r.rho;
        imw += yk[l] / sp.mw[l];
      }
      ts = cfd::update_t(ts, imw, sp, yk, r.E);
      cfd::compute_src(0, ts, sp, re, ys, q1, q2, od, om);
      for (int l = 0; l < ns; ++l) k3[l] = om[l] + k::gamma31Gamma * k1[l] + k::gamma32Gamma * k2[l];
      solve(k3);
      for (int l = 0; l < ns; ++l) k3[l] -= k::gamma31Gamma * k1[l] + k::gamma32Gamma * k2[l];
      for (int l = 0; l < ns; ++l)
        k4[l] = om[l] + k::gamma41Gamma * k1[l] + k::gamma42Gamma * k2[l] + k::gamma43Gamma * k3[l];
      solve(k4);
      for (int l = 0; l < ns; ++l) k4[l] -= k::gamma41Gamma * k1[l] + k::gamma42Gamma * k2[l] + k::gamma43Gamma * k3[l];
    }
    real err = 0;
    std::vector<real> nw(ns);
    for (int l = 0; l < ns; ++l) {
      nw[l] = r.rhoY[l] + h * (k::b1 * k1[l] + k::b2 * k2[l] + k::b4 * k4[l]);
      real dy = h * (k::e1 * k1[l] + k::e2 * k2[l] + k::e3 * k3[l] + k::e4 * k4[l]);
      dy /= rtol * nw[l] + atol;
      err += dy * dy;
    }
    err = std::sqrt(err / ns);
    real hs = h;
    if (r.step > 0) hs *= std::min(5.0, std::max(0.2, 0.8 * std::pow(r.err_last, 0.1) * std::pow(err + 1e-20, -0.175)));
    else if (err > 1) hs *= 0.2;
    if (err <= 1) {
      imw = 0;
      for (int l = 0; l < ns; ++l) {
        r.rhoY[l] = nw[l];
        yk[l] = nw[l] / r.rho;
        imw += yk[l] / sp.mw[l];
      }
      r.time += h;
      r.err_last = err;
      r.h = hs;
      r.T = cfd::update_t(r.T, imw, sp, yk, r.E);
      r.p = r.rho * cfd::R_u * imw * r.T;
      ++r.step;
    } else {
      r.h = hs;
      ++r.n_reject;
    }
  }
}

// The fixed-step forms of const_volume_reactor (src/ConstVolumeReactor.cpp:403-441, 708-763), with
// the reference's own cfd::EPI / cfd::DA and Jacobians: scheme 0 explicit, 1 EPI (full Jacobian,
// LU), 2 DA (diagonal Jacobian) -- advance_scheme = 0 with implicit_method = scheme, optionally
// with conserve_mass_corefl -- and 3 the explicit three-stage Runge-Kutta (advance_scheme = 3).
static void advance_fixed(const cfd::Species &sp, const cfd::Reaction &re, Run &r, int max_steps, real dt, int scheme,
                          bool conserve) {
  const int ns = sp.n_spec, nr = re.n_reac;
  std::vector<real> q1(nr), q2(nr), od(ns), om(ns), yk(ns), yn(ns);
  for (int a = 0; a < max_steps && r.time < r.t_end; ++a) {
    cfd::compute_src(0, r.T, sp, re, r.rhoY, q1, q2, od, om);
    real imw = 0;
    if (scheme <= 2) {
      if (scheme == 1) cfd::EPI(cfd::compute_chem_src_jacobian(r.rhoY, sp, re, q1, q2), sp, dt, om);
      else if (scheme == 2) cfd::DA(cfd::compute_chem_src_jacobian_diagonal(r.rhoY, sp, re, q1, q2), sp, dt, om);
      real sum = 0;
      for (int l = 0; l < ns; ++l) {
        r.rhoY[l] += om[l] * dt;
        if (r.rhoY[l] < 0) r.rhoY[l] = 0;
        sum += r.rhoY[l];
      }
      for (int l = 0; l < ns; ++l) {
        yk[l] = r.rhoY[l] / (conserve ? sum : r.rho);
        if (conserve) r.rhoY[l] = yk[l] * r.rho;
      }
    } else {
      for (int l = 0; l < ns; ++l) {
        yn[l] = r.rhoY[l] + om[l] * dt;
        yk[l] = yn[l] / r.rho;
        imw += yk[l] / sp.mw[l];
      }
      real ts = cfd::update_t(r.T, imw, sp, yk, r.E);
      cfd::compute_src(0, ts, sp, re, yn, q1, q2, od, om);
      imw = 0;
      for (int l = 0; l < ns; ++l) {
        yn[l] = 0.75 * r.rhoY[l] + 0.25 * (yn[l] + om[l] * dt);
        yk[l] = yn[l] / r.rho;
        imw += yk[l] / sp.mw[l];
      }
      ts = cfd::update_t(ts, imw, sp, yk, r.E);
      cfd::compute_src(0, ts, sp, re, yn, q1, q2, od, om);
      for (int l = 0; l < ns; ++l) {
        r.rhoY[l] = (r.rhoY[l] + 2.0 * (yn[l] + om[l] * dt)) / 3.0;
        if (r.rhoY[l] < 0) r.rhoY[l] = 0;
      }
      for (int l = 0; l < ns; ++l) yk[l] = r.rhoY[l] / r.rho;
    }
    imw = 0;
    for (int l = 0; l < ns; ++l) imw += yk[l] / sp.mw[l];
    r.T = cfd::update_t(r.T, imw, sp, yk, r.E);
    r.p = r.rho * cfd::R_u * imw * r.T;
    r.time += dt;
    ++r.step;
  }
}

int main(int argc, char **argv) {
  if (argc < 4) return 2;
  const bool fixed = argc > 4 && std::string(argv[4]) == "fixed";
  const bool krylov = argc > 4 && std::string(argv[4]) == "krylov";
  cfd::Parameter parameter{std::string(argv[1])};
  cfd::Species sp(parameter);
  cfd::Reaction re(parameter, sp);
  const int ns = sp.n_spec;
  const int n = std::stoi(argv[3]);
  FILE *out = std::fopen(argv[2], "w");
  if (!out) return 3;
  std::mt19937_64 gen(20261204);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  const real rtol = 1e-6, atol = 1e-12, h0 = 1e-8;
  std::fprintf(out, "{\n\"n_spec\": %d, \"rtol\": %.17g, \"atol\": %.17g, \"h0\": %.17g,\n\"runs\": [\n", ns, rtol,
               atol, h0);
  for (int c = 0; c < n; ++c) {
    // mole fractions H2 : O2 : N2 (species order of the mechanism: H2 = 0, O2 = 2, N2 = last)
    real T0, p0, t_end, x[3];
    if (c == 0) {
      T0 = 1000;
      p0 = 202650;
      t_end = 1.2e-3;
      x[0] = 0.295775; x[1] = 0.147887; x[2] = 1 - x[0] - x[1];
    } else {
      T0 = 1000 + 500 * U(gen);
      p0 = 101325 * (1 + 9 * U(gen));
      const real phi = 0.5 + 1.5 * U(gen);
      const real s = 2 * phi + 1 + 3.76;
      x[0] = 2 * phi / s; x[1] = 1 / s; x[2] = 3.76 / s;
      t_end = 1e-3;
    }
    std::vector<real> y(ns, 0.0);
    y[0] = x[0] * sp.mw[0];
    y[2] = x[1] * sp.mw[2];
    y[ns - 1] = x[2] * sp.mw[ns - 1];
    const real mw = y[0] + y[2] + y[ns - 1];
    for (auto &v: y) v /= mw;
    Run r;
    real imw = 0;
    for (int l = 0; l < ns; ++l) imw += y[l] / sp.mw[l];
    r.rho = p0 / (T0 * cfd::R_u * imw);
    r.rhoY.resize(ns);
    std::vector<real> hk(ns), cpk(ns);
    sp.compute_enthalpy_and_cp(T0, hk.data(), cpk.data());
    r.E = 0;
    for (int l = 0; l < ns; ++l) {
      r.rhoY[l] = y[l] * r.rho;
      r.E += y[l] * hk[l];
    }
    r.E -= p0 / r.rho;
    r.T = T0; r.p = p0; r.time = 0; r.t_end = t_end; r.h = h0; r.err_last = 0; r.step = r.n_reject = 0;
    auto dump = [&](const char *tag, bool last) {
      std::fprintf(out, "\"%s\": {\"T\": %.17g, \"p\": %.17g, \"time\": %.17g, \"h\": %.17g, \"step\": %d, "
                        "\"n_reject\": %d, \"rhoY\": [", tag, r.T, r.p, r.time, r.h, r.step, r.n_reject);
      for (int l = 0; l < ns; ++l) std::fprintf(out, "%s%.17g", l ? ", " : "", r.rhoY[l]);
      std::fprintf(out, "]}%s", last ? "" : ",\n");
    };
    std::fprintf(out, "%s{\"T0\": %.17g, \"p0\": %.17g, \"t_end\": %.17g, \"Y\": [", c ? ",\n" : "", T0, p0, t_end);
    for (int l = 0; l < ns; ++l) std::fprintf(out, "%s%.17g", l ? ", " : "", y[l]);
    std::fprintf(out, "],\n");
    if (fixed) {
      // each form from the same initial state: (scheme, conserve_mass, dt, t_end)
      const Run r0 = r;
      const struct { int scheme, conserve; real dt, t_end; const char *tag; } forms[] = {
          {0, 0, 1e-9, 2e-5, "explicit"}, {0, 1, 1e-9, 2e-5, "explicit_conserve"}, {1, 0, 1e-7, 4e-4, "epi"},
          {1, 1, 1e-7, 4e-4, "epi_conserve"}, {2, 0, 1e-9, 5e-5, "da"}, {3, 0, 1e-9, 2e-5, "rk3"}};
      const int nf = sizeof(forms) / sizeof(forms[0]);
      for (int f = 0; f < nf; ++f) {
        r = r0;
        r.t_end = forms[f].t_end;
        r.h = forms[f].dt;
        std::fprintf(out, "\"%s\": {\"scheme\": %d, \"conserve_mass\": %d, \"dt\": %.17g, \"t_end\": %.17g,\n",
                     forms[f].tag, forms[f].scheme, forms[f].conserve, forms[f].dt, forms[f].t_end);
        advance_fixed(sp, re, r, 100, forms[f].dt, forms[f].scheme, forms[f].conserve);
        dump("after_100_steps", false);
        advance_fixed(sp, re, r, 100000000, forms[f].dt, forms[f].scheme, forms[f].conserve);
        dump("final", true);
        std::fprintf(out, "}%s", f + 1 < nf ? ",\n" : "");
      }
    } else {
      advance(sp, re, r, 8, rtol, atol, krylov);
      dump("after_8_attempts", false);
      // the Krylov form shrinks its steps until they stall short of t_end: 2000 attempts in all
      advance(sp, re, r, krylov ? 1992 : 1000000, rtol, atol, krylov);
      dump(krylov ? "after_2000_attempts" : "final", true);
    }
    std::fprintf(out, "}");
  }
  std::fprintf(out, "\n]\n}\n");
  std::fclose(out);
  return 0;
}
