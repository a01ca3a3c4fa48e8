// Evaluates the reference's own host chemistry source (cfd::compute_src of
// src/ConstVolumeReactor.cpp, the host twin of finite_rate_chemistry) and its host
// temperature Newton solver (cfd::update_t) on seeded states, and writes them as JSON.
// TEST INFRASTRUCTURE ONLY: built into oracle/_ref/ by oracle/ref_build.py and run by
// tests/golden/make_mech.py to write tests/golden/h2_chem_states.json.
//
// Usage (from a directory holding ./input/<files>): dump_chem <setup-file> <out.json> <n>
#include <cmath>
#include <cstdio>
#include <random>
#include <string>
#include <vector>
#include "ChemData.h"
#include "Constants.h"
#include "ConstVolumeReactor.h"
#include "Parameter.h"

int main(int argc, char **argv) {
  if (argc < 4) return 2;
  cfd::Parameter parameter{std::string(argv[1])};
  cfd::Species spec(parameter);
  cfd::Reaction reac(parameter, spec);
  const int ns = spec.n_spec;
  const int n = std::stoi(argv[3]);
  FILE *out = std::fopen(argv[2], "w");
  if (!out) return 3;
  std::mt19937_64 gen(20261203);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  std::fprintf(out, "{\n\"n_spec\": %d,\n\"states\": [\n", ns);
  for (int a = 0; a < n; ++a) {
    const double t = 700.0 + 2600.0 * U(gen);
    const double rho = 0.02 + 2.0 * U(gen);
    std::vector<double> y(ns), rhoY(ns), q1(reac.n_reac), q2(reac.n_reac), od(ns), om(ns);
    double sum = 0;
    for (int s = 0; s < ns; ++s) {
      // major species O(0.1), radicals down to 1e-8, one species exactly zero now and then
      const double e = -8.0 * U(gen);
      y[s] = (a % 7 == 3 && s == a % ns) ? 0.0 : std::pow(10.0, e);
      sum += y[s];
    }
    for (int s = 0; s < ns; ++s) {
      y[s] /= sum;
      rhoY[s] = rho * y[s];
    }
    cfd::compute_src(0, t, spec, reac, rhoY, q1, q2, od, om);
    // energy of this state at t, then the reference's Newton T from a guess 10% off
    std::vector<double> h(ns), cp(ns);
    spec.compute_enthalpy_and_cp(t, h.data(), cp.data());
    double imw = 0, e = 0;
    for (int s = 0; s < ns; ++s) {
      imw += y[s] / spec.mw[s];
      e += y[s] * h[s];
    }
    e -= cfd::R_u * imw * t;  // internal energy per unit mass
    const double t_newton = cfd::update_t(1.1 * t, imw, spec, y, e);
    std::fprintf(out, "%s{\"t\": %.17g, \"rho\": %.17g, \"e\": %.17g, \"t_guess\": %.17g, \"t_newton\": %.17g,\n",
                 a ? ",\n" : "", t, rho, e, 1.1 * t, t_newton);
    auto arr = [&](const char *nm, const std::vector<double> &v, bool last) {
      std::fprintf(out, "\"%s\": [", nm);
      for (int s = 0; s < ns; ++s) std::fprintf(out, "%s%.17g", s ? ", " : "", v[s]);
      std::fprintf(out, "]%s", last ? "}" : ", ");
    };
    arr("y", y, false);
    arr("h", h, false);
    arr("cp", cp, false);
    arr("omega", om, false);
    arr("omega_d", od, true);
  }
  std::fprintf(out, "\n],\n\"source\": \"cfd::compute_src, cfd::update_t and Species::compute_enthalpy_and_cp of the reference\"\n}\n");
  std::fclose(out);
  return 0;
}
