// Runs the reference's own mechanism/thermo/transport parser (cfd::Species and
// cfd::Reaction, src/ChemData.cpp) on a setup file and prints every table the hot path
// reads from DParameter as JSON, so the library and the oracle get the exact tables the
// reference computes.
// TEST INFRASTRUCTURE ONLY: built into oracle/_ref/ by oracle/ref_build.py and run by
// tests/golden/make_mech.py to write the committed mechanism fixtures.
//
// Usage (from a directory holding ./input/<files>):  dump_mech <setup-file> <out.json>
#include <cstdio>
#include <string>
#include <vector>
#include "ChemData.h"
#include "Parameter.h"

namespace {
FILE *g_out = nullptr;
void arr(const char *name, const std::vector<double> &v, bool comma = true) {
  std::fprintf(g_out, "\"%s\": [", name);
  for (size_t i = 0; i < v.size(); ++i) std::fprintf(g_out, "%s%.17g", i ? ", " : "", v[i]);
  std::fprintf(g_out, "]%s\n", comma ? "," : "");
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
  if (argc < 2) {
    std::fprintf(stderr, "usage: dump_mech <setup-file>\n");
    return 2;
  }
  cfd::Parameter parameter{std::string(argv[1])};
  cfd::Species spec(parameter);
  cfd::Reaction reac(parameter, spec);
  const int ns = spec.n_spec, nr = reac.n_reac;
  g_out = std::fopen(argc > 2 ? argv[2] : "mech.json", "w");
  if (!g_out) return 3;
  std::fprintf(g_out, "{\n\"n_spec\": %d,\n\"n_reac\": %d,\n\"nasa_7_or_9\": %d,\n", ns, nr, spec.nasa_7_or_9);
  std::fprintf(g_out, "\"species\": [");
  for (int s = 0; s < ns; ++s) std::fprintf(g_out, "%s\"%s\"", s ? ", " : "", spec.spec_name[s].c_str());
  std::fprintf(g_out, "],\n");
  arr("mw", spec.mw);
  if (spec.nasa_7_or_9 == 7) {
    arr("low_temp_coeff", mat(spec.low_temp_coeff, ns, 7));
    arr("high_temp_coeff", mat(spec.high_temp_coeff, ns, 7));
    arr("t_low", spec.t_low);
    arr("t_mid", spec.t_mid);
    arr("t_high", spec.t_high);
  }
  arr("geometry", spec.geometry);
  arr("LJ_potent_inv", spec.LJ_potent_inv);
  arr("vis_coeff", spec.vis_coeff);
  arr("WjDivWi_to_One4th", mat(spec.WjDivWi_to_One4th, ns, ns));
  arr("sqrt_WiDivWjPl1Mul8", mat(spec.sqrt_WiDivWjPl1Mul8, ns, ns));
  arr("binary_diffusivity_coeff", mat(spec.binary_diffusivity_coeff, ns, ns));
  arr("kb_over_eps_jk", mat(spec.kb_over_eps_jk, ns, ns));
  arr("ZRotF298", spec.ZRotF298);
  if (nr > 0) {
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
  }
  std::fprintf(g_out, "\"source\": \"cfd::Species/cfd::Reaction of src/ChemData.cpp\"\n}\n");
  std::fclose(g_out);
  return 0;
}
