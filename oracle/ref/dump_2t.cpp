// Evaluates the reference's own host two-temperature functions and writes them as JSON: the
// tables cfd::Species::read_two_temperature parses (src/ChemData.cpp:130-233), the species
// vibrational-electronic energies and heat capacities of Species::compute_ve_energy /
// compute_ve_cv (:236-291), the mixture energy and T_ve inversion of
// Species::compute_mixture_ve_energy / invert_tve_from_eve (:293-322), and the VT relaxation
// source, equilibrium energy and effective relaxation time of cfd::compute_vt_relaxation_source
// (src/ConstVolumeReactor.cpp:953-998) on seeded states.
// TEST INFRASTRUCTURE ONLY: built into oracle/_ref/ by oracle/ref_build.py (with the reference's
// two-temperature switch on) and run by tests/golden/make_mech.py.
//
// Usage (from a directory holding ./input/<files>): dump_2t <setup-file> <out.json> <n>
#include <cmath>
#include <cstdio>
#include <random>
#include <string>
#include <vector>
#include "ChemData.h"
#include "ConstVolumeReactor.h"
#include "Parameter.h"

namespace {
FILE *g_out = nullptr;
void arr(const char *name, const std::vector<double> &v) {
  std::fprintf(g_out, "\"%s\": [", name);
  for (size_t i = 0; i < v.size(); ++i) std::fprintf(g_out, "%s%.17g", i ? ", " : "", v[i]);
  std::fprintf(g_out, "],\n");
}
}  // namespace

int main(int argc, char **argv) {
  if (argc < 4) return 2;
  cfd::Parameter parameter{std::string(argv[1])};
  cfd::Species sp(parameter);
  const int ns = sp.n_spec;
  const int n = std::stoi(argv[3]);
  g_out = std::fopen(argv[2], "w");
  if (!g_out) return 3;
  if (!sp.has_two_temperature_data) return 4;
  const int ml = std::max(1, sp.max_electronic_level);
  std::fprintf(g_out, "{\n\"n_spec\": %d,\n\"max_level\": %d,\n", ns, ml);
  std::fprintf(g_out, "\"n_level\": [");
  for (int s = 0; s < ns; ++s) std::fprintf(g_out, "%s%d", s ? ", " : "", sp.n_electronic_level[s]);
  std::fprintf(g_out, "],\n");
  arr("theta_v", sp.theta_v);
  arr("park_sigma", sp.park_sigma);
  std::vector<double> et, eg, la, lb;
  for (int s = 0; s < ns; ++s)
    for (int j = 0; j < ml; ++j) {
      et.push_back(sp.electronic_theta(s, j));
      eg.push_back(sp.electronic_g(s, j));
    }
  for (int s = 0; s < ns; ++s)
    for (int r = 0; r < ns; ++r) {
      la.push_back(sp.lt_a(s, r));
      lb.push_back(sp.lt_b(s, r));
    }
  arr("elec_theta", et);
  arr("elec_g", eg);
  arr("lt_a", la);
  arr("lt_b", lb);

  // per-species energies and heat capacities on a temperature ladder
  const std::vector<double> temps{0.5, 50.0, 300.0, 1000.0, 3000.0, 10000.0, 30000.0};
  arr("ladder_T", temps);
  std::vector<double> ev, cv;
  for (double t: temps)
    for (int s = 0; s < ns; ++s) {
      ev.push_back(sp.compute_ve_energy(s, t));
      cv.push_back(sp.compute_ve_cv(s, t));
    }
  arr("ladder_e_ve", ev);
  arr("ladder_cv_ve", cv);

  // seeded mixture states
  std::mt19937_64 gen(20261203);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  std::fprintf(g_out, "\"states\": [\n");
  for (int c = 0; c < n; ++c) {
    std::vector<double> y(ns);
    double sum = 0;
    for (int s = 0; s < ns; ++s) {
      // mostly a few major species, some exact zeros
      y[s] = U(gen) < 0.25 ? 0.0 : std::pow(U(gen), 3.0);
      sum += y[s];
    }
    if (sum <= 0) { y[ns - 1] = 1; sum = 1; }
    for (auto &v: y) v /= sum;
    const double rho = std::exp(std::log(1e-3) + U(gen) * std::log(2.0 / 1e-3));
    const double t = 300 + 9700 * U(gen);
    const double tve = 200 + 11800 * U(gen);
    double cv_t = 0, cv_tve = 0;
    const double eve_t = sp.compute_mixture_ve_energy(t, y, &cv_t);
    const double eve_tve = sp.compute_mixture_ve_energy(tve, y, &cv_tve);
    const double tve_inv = sp.invert_tve_from_eve(eve_tve, y, t);
    double eve_eq = 0, tau = 0;
    const double src = cfd::compute_vt_relaxation_source(rho, t, tve, y, sp, &eve_eq, &tau);
    std::fprintf(g_out, "%s{\"rho\": %.17g, \"T\": %.17g, \"Tve\": %.17g, \"Y\": [", c ? ",\n" : "", rho, t, tve);
    for (int s = 0; s < ns; ++s) std::fprintf(g_out, "%s%.17g", s ? ", " : "", y[s]);
    std::fprintf(g_out,
                 "], \"eve_T\": %.17g, \"cv_ve_T\": %.17g, \"eve_Tve\": %.17g, \"cv_ve_Tve\": %.17g, "
                 "\"tve_inverted\": %.17g, \"vt_source\": %.17g, \"eve_eq\": %.17g, \"tau_eff\": %.17g}",
                 eve_t, cv_t, eve_tve, cv_tve, tve_inv, src, eve_eq, tau);
  }
  std::fprintf(g_out, "\n]\n}\n");
  std::fclose(g_out);
  return 0;
}
