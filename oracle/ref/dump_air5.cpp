// Evaluates the reference's own host code for the two-temperature AIR5 case and writes it as
// JSON: the mechanism tables of cfd::Species / cfd::Reaction (src/ChemData.cpp) read with
// NASA9 multi-range thermo (read_therm_nasa9, :865-1034) and the AIR5 control-temperature
// model (:1247-1262), the vibrational-electronic tables of two_temperature.dat (:130-233);
// species h, cp (Species::compute_enthalpy_and_cp) and g/RT (compute_gibbs_div_rt,
// src/ConstVolumeReactor.cpp:1401-1454) on a temperature ladder; and on seeded states the
// chemical source of compute_src with (T, Tve) (:930-951), the e_ve chemical source
// (:1000-1006) and the two-temperature Newton temperature update_t_two_temperature
// (:1483-1551).
// TEST INFRASTRUCTURE ONLY: built into oracle/_ref/ by oracle/ref_build.py (two-temperature
// switch on) and run by tests/golden/make_mech.py.
//
// Usage (from a directory holding ./input/<files>): dump_air5 <setup-file> <out.json> <n>
#include <cmath>
#include <cstdio>
#include <random>
#include <string>
#include <vector>
#include "ChemData.h"
#include "Constants.h"
#include "ConstVolumeReactor.h"
#include "Parameter.h"

namespace {
FILE *g_out = nullptr;
void arr(const char *name, const std::vector<double> &v) {
  std::fprintf(g_out, "\"%s\": [", name);
  for (size_t i = 0; i < v.size(); ++i) std::fprintf(g_out, "%s%.17g", i ? ", " : "", v[i]);
  std::fprintf(g_out, "],\n");
}
void iarr(const char *name, const std::vector<int> &v) {
  std::fprintf(g_out, "\"%s\": [", name);
  for (size_t i = 0; i < v.size(); ++i) std::fprintf(g_out, "%s%d", i ? ", " : "", v[i]);
  std::fprintf(g_out, "],\n");
}
template <typename M>
std::vector<double> mat(const M &m, int r, int c) {
  std::vector<double> v;
  for (int i = 0; i < r; ++i)
    for (int j = 0; j < c; ++j) v.push_back(m(i, j));
  return v;
}
template <typename M>
std::vector<int> imat(const M &m, int r, int c) {
  std::vector<int> v;
  for (int i = 0; i < r; ++i)
    for (int j = 0; j < c; ++j) v.push_back(m(i, j));
  return v;
}
}  // namespace

int main(int argc, char **argv) {
  if (argc < 4) return 2;
  cfd::Parameter parameter{std::string(argv[1])};
  cfd::Species sp(parameter);
  cfd::Reaction reac(parameter, sp);
  const int ns = sp.n_spec, nr = reac.n_reac;
  const int n = std::stoi(argv[3]);
  g_out = std::fopen(argv[2], "w");
  if (!g_out) return 3;
  if (!sp.has_two_temperature_data || sp.nasa_7_or_9 != 9) return 4;
  std::fprintf(g_out, "{\n\"n_spec\": %d,\n\"n_reac\": %d,\n\"nasa_7_or_9\": %d,\n", ns, nr, sp.nasa_7_or_9);
  std::fprintf(g_out, "\"species\": [");
  for (int s = 0; s < ns; ++s) std::fprintf(g_out, "%s\"%s\"", s ? ", " : "", sp.spec_name[s].c_str());
  std::fprintf(g_out, "],\n");
  arr("mw", sp.mw);
  // NASA9 multi-range tables: cuts [ns][max_range+1], coefficients [ns][max_range][9]
  int max_range = 0;
  for (int s = 0; s < ns; ++s) max_range = std::max(max_range, sp.n_temperature_range[s]);
  std::fprintf(g_out, "\"max_range\": %d,\n", max_range);
  iarr("n_temperature_range", std::vector<int>(sp.n_temperature_range.begin(), sp.n_temperature_range.begin() + ns));
  std::vector<double> cuts, poly;
  for (int s = 0; s < ns; ++s) {
    for (int j = 0; j <= max_range; ++j) cuts.push_back(j <= sp.n_temperature_range[s] ? sp.temperature_range(s, j) : 0.0);
    for (int j = 0; j < max_range; ++j)
      for (int c = 0; c < 9; ++c) poly.push_back(sp.therm_poly_coeff(c, j, s));
  }
  arr("temperature_range", cuts);
  arr("therm_poly_coeff", poly);
  arr("geometry", sp.geometry);
  arr("LJ_potent_inv", sp.LJ_potent_inv);
  arr("vis_coeff", sp.vis_coeff);
  arr("WjDivWi_to_One4th", mat(sp.WjDivWi_to_One4th, ns, ns));
  arr("sqrt_WiDivWjPl1Mul8", mat(sp.sqrt_WiDivWjPl1Mul8, ns, ns));
  arr("binary_diffusivity_coeff", mat(sp.binary_diffusivity_coeff, ns, ns));
  arr("kb_over_eps_jk", mat(sp.kb_over_eps_jk, ns, ns));
  arr("ZRotF298", sp.ZRotF298);
  std::vector<int> lab(reac.label.begin(), reac.label.begin() + nr);
  std::vector<int> rev(reac.rev_type.begin(), reac.rev_type.begin() + nr);
  std::vector<int> ord(reac.order.begin(), reac.order.begin() + nr);
  iarr("reac_type", lab);
  iarr("rev_type", rev);
  iarr("reac_order", ord);
  iarr("stoi_f", imat(reac.stoi_f, nr, ns));
  iarr("stoi_b", imat(reac.stoi_b, nr, ns));
  auto head = [&](const std::vector<double> &v) { return std::vector<double>(v.begin(), v.begin() + nr); };
  arr("A", head(reac.A));
  arr("b", head(reac.b));
  arr("Ea", head(reac.Ea));
  arr("A2", head(reac.A2));
  arr("b2", head(reac.b2));
  arr("Ea2", head(reac.Ea2));
  arr("third_body_coeff", mat(reac.third_body_coeff, nr, ns));
  arr("troe_alpha", head(reac.troe_alpha));
  arr("troe_t3", head(reac.troe_t3));
  arr("troe_t1", head(reac.troe_t1));
  arr("troe_t2", head(reac.troe_t2));
  std::fprintf(g_out, "\"two_temperature_reaction_temperature\": %d,\n",
               reac.two_temperature_reaction_temperature ? 1 : 0);
  arr("tcf_a", head(reac.tcf_a));
  arr("tcf_b", head(reac.tcf_b));
  arr("tcb_a", head(reac.tcb_a));
  arr("tcb_b", head(reac.tcb_b));

  // two-temperature tables
  const int ml = std::max(1, sp.max_electronic_level);
  std::fprintf(g_out, "\"max_level\": %d,\n", ml);
  iarr("n_level", std::vector<int>(sp.n_electronic_level.begin(), sp.n_electronic_level.begin() + ns));
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

  // thermo on a ladder that crosses every range boundary and both extrapolated ends
  const std::vector<double> temps{100.0, 199.9, 200.0, 250.0, 300.0, 999.9, 1000.0, 1000.1, 2500.0,
                                  5999.0, 6000.0, 6001.0, 12000.0, 19999.0, 20000.0, 20001.0, 30000.0};
  arr("ladder_T", temps);
  std::vector<double> lh, lcp, lg, lev, lcv;
  std::vector<double> h(ns), cp(ns);
  std::vector<double> g(ns);
  for (double t: temps) {
    sp.compute_enthalpy_and_cp(t, h.data(), cp.data());
    cfd::compute_gibbs_div_rt(t, sp, g);
    for (int s = 0; s < ns; ++s) {
      lh.push_back(h[s]);
      lcp.push_back(cp[s]);
      lg.push_back(g[s]);
      lev.push_back(sp.compute_ve_energy(s, t));
      lcv.push_back(sp.compute_ve_cv(s, t));
    }
  }
  arr("ladder_h", lh);
  arr("ladder_cp", lcp);
  arr("ladder_gibbs_rt", lg);
  arr("ladder_e_ve", lev);
  arr("ladder_cv_ve", lcv);

  // seeded states: chemistry with (T, Tve) and the two-temperature Newton temperature
  std::mt19937_64 gen(20261204);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  std::fprintf(g_out, "\"states\": [\n");
  std::vector<double> q1(nr), q2(nr), omega_d(ns), omega(ns);
  for (int c = 0; c < n; ++c) {
    std::vector<double> y(ns);
    double sum = 0;
    for (int s = 0; s < ns; ++s) {
      y[s] = U(gen) < 0.2 ? 0.0 : std::pow(U(gen), 2.0);
      sum += y[s];
    }
    if (sum <= 0) { y[0] = 1; sum = 1; }
    for (auto &v: y) v /= sum;
    const double rho = std::exp(std::log(1e-3) + U(gen) * std::log(0.5 / 1e-3));
    const double t = 300 + 14700 * U(gen);
    const double tve = 250 + 11750 * U(gen);
    std::vector<double> rhoY(ns);
    for (int s = 0; s < ns; ++s) rhoY[s] = rho * y[s];
    cfd::compute_src(0, t, tve, sp, reac, rhoY, q1, q2, omega_d, omega);
    const double eve_src = cfd::compute_two_temperature_chemical_source(tve, sp, omega);
    // internal energy of the state (trans-rot at t + ve at tve) and the Newton temperature from
    // a guess 15% off
    sp.compute_enthalpy_and_cp(t, h.data(), cp.data());
    double e_eq = 0;
    for (int s = 0; s < ns; ++s) e_eq += y[s] * (h[s] - cfd::R_u / sp.mw[s] * t);
    const double eve_t = sp.compute_mixture_ve_energy(t, y);
    const double eve = sp.compute_mixture_ve_energy(tve, y);
    const double E = e_eq - eve_t + eve;
    const double t_newton = cfd::update_t_two_temperature(0.85 * t, sp, y, E, eve);
    std::fprintf(g_out, "%s{\"rho\": %.17g, \"T\": %.17g, \"Tve\": %.17g, \"Y\": [", c ? ",\n" : "", rho, t, tve);
    for (int s = 0; s < ns; ++s) std::fprintf(g_out, "%s%.17g", s ? ", " : "", y[s]);
    std::fprintf(g_out, "], \"omega\": [");
    for (int s = 0; s < ns; ++s) std::fprintf(g_out, "%s%.17g", s ? ", " : "", omega[s]);
    std::fprintf(g_out, "], \"omega_d\": [");
    for (int s = 0; s < ns; ++s) std::fprintf(g_out, "%s%.17g", s ? ", " : "", omega_d[s]);
    std::fprintf(g_out, "], \"eve_source\": %.17g, \"E\": %.17g, \"eve\": %.17g, \"T_newton\": %.17g}", eve_src, E,
                 eve, t_newton);
  }
  std::fprintf(g_out, "\n],\n\"source\": \"cfd::Species/cfd::Reaction of src/ChemData.cpp, host chemistry of "
                      "src/ConstVolumeReactor.cpp\"\n}\n");
  std::fclose(g_out);
  return 0;
}
