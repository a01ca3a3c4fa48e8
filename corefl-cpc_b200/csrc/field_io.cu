// Flowfield files: the bound blocks' state in the Tecplot binary format (version 112, ordered
// zones, double data at the nodes), as the reference writes output/flowfield.plt
// (FieldIO::initialize / print_field, src/FieldIO.h:77-470) and reads it back to restart
// (read_flowfield, src/Initialize.cu:167-411).  Host code: the fields come to the host over the
// caller's stream, the file is written with stdio.
//
// Layout (the published V112 format, with the choices the reference makes):
//   header : "#!TDV112", int32 1 (byte order), int32 0 (full file), title "Solution file",
//            int32 n_var, the variable names; per zone: float 299, its name "zone <b>", int32 -1
//            (parent), -2 (strand), float64 solution time, int32 -1 (colour), 0 (ordered), 0 (node
//            data), 0 (no raw face neighbours), 0 (no connections), IMax, JMax, KMax (the block's
//            nodes plus 2 ngg_out), 0 (no auxiliary data); float 357 (end of header).
//   data   : per zone: float 299, int32 2 (double) per variable, 0 (no passive), 0 (no sharing),
//            -1 (no shared connectivity), the (min, max) pair of every variable over the written
//            nodes, then the variables, i fastest.
//   Strings are int32 characters closed by a zero.
// Variables: x, y, z, density, u, v, w, pressure, temperature, the species, Eve (two
// temperatures), mach, Tve (two temperatures): the reference's default output list with no
// turbulence, passive scalars or user-defined auxiliaries (Parameter::setup_default_settings,
// src/Parameter.cpp:837-953; add_other_variable_name, src/UDIO.cu:11-38).
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "launch.h"

namespace cb2 {
const Param *ctx_param(const cb2_ctx *ctx);
int ctx_zones(const cb2_ctx *ctx, std::vector<Zone> &zones);
}  // namespace cb2

using namespace cb2;

namespace {

struct Out {
  std::FILE *f = nullptr;
  bool ok = true;
  void raw(const void *p, size_t n) {
    if (ok && std::fwrite(p, 1, n, f) != n) ok = false;
  }
  void i32(int32_t v) { raw(&v, 4); }
  void f32(float v) { raw(&v, 4); }
  void f64(double v) { raw(&v, 8); }
  void str(const std::string &s) {
    for (unsigned char c : s) i32(static_cast<int32_t>(c));
    i32(0);
  }
};

struct In {
  std::FILE *f = nullptr;
  bool ok = true;
  void raw(void *p, size_t n) {
    if (ok && std::fread(p, 1, n, f) != n) ok = false;
  }
  void skip(long n) {
    if (ok && std::fseek(f, n, SEEK_CUR) != 0) ok = false;
  }
  int32_t i32() {
    int32_t v = 0;
    raw(&v, 4);
    return v;
  }
  float f32() {
    float v = 0;
    raw(&v, 4);
    return v;
  }
  double f64() {
    double v = 0;
    raw(&v, 8);
    return v;
  }
  std::string str() {
    std::string s;
    for (int n = 0; ok && n < 4096; ++n) {
      const int32_t c = i32();
      if (c == 0) return s;
      s += static_cast<char>(c);
    }
    ok = false;
    return s;
  }
};

std::string upper(std::string s) {
  for (char &c : s)
    if (c >= 'a' && c <= 'z') c = static_cast<char>(c - 'a' + 'A');
  return s;
}

// A device array of one padded block (ghost g) brought to the host.
int fetch(std::vector<double> &h, const double *d, size_t n, cudaStream_t s) {
  h.resize(n);
  return check_cuda(cudaMemcpyAsync(h.data(), d, n * sizeof(double), cudaMemcpyDeviceToHost, s));
}

}  // namespace

extern "C" int cb2_write_flowfield(cb2_ctx *ctx, const char *path, const double *const *xyz,
                                   const char *const *species_names, int ngg_out, double solution_time,
                                   void *stream) {
  std::vector<Zone> zones;
  CB2_TRY(ctx_zones(ctx, zones));
  const Param &p = *ctx_param(ctx);
  if (!path || !xyz || ngg_out < 0 || (p.n_spec > 0 && !species_names)) return CB2_ERR_INVALID;
  const bool two_t = p.i_eve >= 0;
  for (size_t b = 0; b < zones.size(); ++b) {
    const Zone &z = zones[b];
    if (ngg_out > z.ngg || !z.mach || (two_t && !z.tve) || !xyz[3 * b] || !xyz[3 * b + 1] || !xyz[3 * b + 2])
      return CB2_ERR_INVALID;
  }
  for (int l = 0; l < p.n_spec; ++l)
    if (!species_names[l]) return CB2_ERR_INVALID;
  std::vector<std::string> names{"x", "y", "z", "density", "u", "v", "w", "pressure", "temperature"};
  for (int l = 0; l < p.n_spec; ++l) names.emplace_back(species_names[l]);
  if (two_t) names.emplace_back("Eve");
  names.emplace_back("mach");
  if (two_t) names.emplace_back("Tve");
  const int n_var = static_cast<int>(names.size());
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  // the blocks' fields on the host: bv, sv, mach, T_ve per block
  const size_t nb = zones.size();
  std::vector<std::vector<double>> bv(nb), sv(nb), mach(nb), tve(nb);
  for (size_t b = 0; b < nb; ++b) {
    const Zone &z = zones[b];
    const size_t sz = static_cast<size_t>(z.L.sz);
    CB2_TRY(fetch(bv[b], z.bv, 6 * sz, s));
    if (p.n_scalar > 0) CB2_TRY(fetch(sv[b], z.sv, p.n_scalar * sz, s));
    CB2_TRY(fetch(mach[b], z.mach, sz, s));
    if (two_t) CB2_TRY(fetch(tve[b], z.tve, sz, s));
  }
  CB2_TRY(check_cuda(cudaStreamSynchronize(s)));

  Out o;
  o.f = std::fopen(path, "wb");
  if (!o.f) return CB2_ERR_INVALID;
  // header
  o.raw("#!TDV112", 8);
  o.i32(1);
  o.i32(0);
  o.str("Solution file");
  o.i32(n_var);
  for (const auto &n : names) o.str(n);
  for (size_t b = 0; b < nb; ++b) {
    const Zone &z = zones[b];
    o.f32(299.0f);
    o.str("zone " + std::to_string(b));
    o.i32(-1);
    o.i32(-2);
    o.f64(solution_time);
    o.i32(-1);
    o.i32(0);
    o.i32(0);
    o.i32(0);
    o.i32(0);
    o.i32(z.mx + 2 * ngg_out);
    o.i32(z.my + 2 * ngg_out);
    o.i32(z.mz + 2 * ngg_out);
    o.i32(0);
  }
  o.f32(357.0f);
  // data
  for (size_t b = 0; b < nb; ++b) {
    const Zone &z = zones[b];
    const Layout &L = z.L;
    const int n = ngg_out;
    const size_t sz = static_cast<size_t>(L.sz);
    // the padded arrays of the written variables, in the file's order
    std::vector<const double *> src;
    for (int c = 0; c < 3; ++c) src.push_back(xyz[3 * b + c]);
    for (int l = 0; l < 6; ++l) src.push_back(bv[b].data() + l * sz);
    for (int l = 0; l < p.n_scalar; ++l) src.push_back(sv[b].data() + l * sz);
    src.push_back(mach[b].data());
    if (two_t) src.push_back(tve[b].data());
    o.f32(299.0f);
    for (int l = 0; l < n_var; ++l) o.i32(2);
    o.i32(0);
    o.i32(0);
    o.i32(-1);
    // (min, max) of each variable over the written nodes, from the first node on, as std::min/max
    for (const double *a : src) {
      double lo = a[L.at(-n, -n, -n)], hi = lo;
      for (int k = -n; k < z.mz + n; ++k)
        for (int j = -n; j < z.my + n; ++j)
          for (int i = -n; i < z.mx + n; ++i) {
            const double v = a[L.at(i, j, k)];
            if (v < lo) lo = v;
            if (hi < v) hi = v;
          }
      o.f64(lo);
      o.f64(hi);
    }
    const int ni = z.mx + 2 * n;
    for (const double *a : src)
      for (int k = -n; k < z.mz + n; ++k)
        for (int j = -n; j < z.my + n; ++j) o.raw(a + L.at(-n, j, k), ni * sizeof(double));
  }
  const bool ok = o.ok;
  if (std::fclose(o.f) != 0 || !ok) return CB2_ERR_INVALID;
  return CB2_OK;
}

extern "C" int cb2_read_flowfield(cb2_ctx *ctx, const char *path, const char *const *species_names,
                                  double *solution_time, void *stream) {
  std::vector<Zone> zones;
  CB2_TRY(ctx_zones(ctx, zones));
  const Param &p = *ctx_param(ctx);
  if (!path || (p.n_spec > 0 && !species_names)) return CB2_ERR_INVALID;
  const bool two_t = p.i_eve >= 0;
  In in;
  in.f = std::fopen(path, "rb");
  if (!in.f) return CB2_ERR_INVALID;
  struct Closer {
    std::FILE *f;
    ~Closer() { std::fclose(f); }
  } closer{in.f};
  char magic[8];
  in.raw(magic, 8);
  if (!in.ok || std::memcmp(magic, "#!TDV", 5) != 0) return CB2_ERR_INVALID;
  in.skip(8);  // byte order, file type
  in.str();    // title
  const int n_var = in.i32();
  if (!in.ok || n_var < 3 || n_var > 4096) return CB2_ERR_INVALID;
  // where each variable goes (identify_variable_labels, src/Initialize.cu:412-487):
  // 0..5 bv, 6 + l sv (species, then Eve at i_eve), -2 T_ve, -1 ignored
  std::vector<int> dest(n_var, -1);
  bool tve_read = false;
  for (int l = 0; l < n_var; ++l) {
    const std::string n = upper(in.str());
    int d = -1;
    if (n == "DENSITY" || n == "ROE" || n == "RHO") d = 0;
    else if (n == "U") d = 1;
    else if (n == "V") d = 2;
    else if (n == "W") d = 3;
    else if (n == "P" || n == "PRESSURE") d = 4;
    else if (n == "T" || n == "TEMPERATURE") d = 5;
    else {
      for (int s = 0; s < p.n_spec; ++s)
        if (n == upper(species_names[s] ? species_names[s] : "")) d = 6 + s;
      if (two_t && n == "EVE") d = 6 + p.i_eve;
      if (two_t && n == "TVE") {
        d = -2;
        tve_read = true;
      }
    }
    dest[l] = d;
  }
  // zones: their sizes must be the bound blocks' plus the same 2 g on every side
  std::vector<int> dims;
  double t_sol = 0;
  for (float marker = in.f32(); in.ok && marker > 298.999f && marker < 299.001f; marker = in.f32()) {
    in.str();
    in.skip(8);
    t_sol = in.f64();
    in.skip(20);
    for (int a = 0; a < 3; ++a) dims.push_back(in.i32());
    in.skip(4);
  }
  if (!in.ok || dims.size() != 3 * zones.size()) return CB2_ERR_INVALID;
  std::vector<int> gfile(zones.size());
  for (size_t b = 0; b < zones.size(); ++b) {
    const Zone &z = zones[b];
    const int g = (dims[3 * b] - z.mx) / 2;
    if (g < 0 || g > z.ngg || dims[3 * b] != z.mx + 2 * g || dims[3 * b + 1] != z.my + 2 * g ||
        dims[3 * b + 2] != z.mz + 2 * g)
      return CB2_ERR_INVALID;
    gfile[b] = g;
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  std::vector<double> line;
  for (size_t b = 0; b < zones.size(); ++b) {
    const Zone &z = zones[b];
    const Layout &L = z.L;
    const int g = gfile[b];
    const size_t sz = static_cast<size_t>(L.sz);
    in.skip(4 + 4L * n_var + 12 + 16L * n_var);  // marker, formats, flags, min/max pairs
    // the block's arrays on the host, overwritten where the file has them, then sent back
    std::vector<double> bv, sv, tve;
    CB2_TRY(fetch(bv, z.bv, 6 * sz, s));
    if (p.n_scalar > 0) CB2_TRY(fetch(sv, z.sv, p.n_scalar * sz, s));
    if (two_t) tve.assign(sz, 0.0);  // a file without Tve leaves T_ve to be found from e_ve
    CB2_TRY(check_cuda(cudaStreamSynchronize(s)));
    const int ni = z.mx + 2 * g;
    line.resize(ni);
    for (int l = 0; l < n_var; ++l) {
      double *dst = nullptr;
      if (dest[l] >= 0 && dest[l] < 6) dst = bv.data() + dest[l] * sz;
      else if (dest[l] >= 6) dst = sv.data() + (dest[l] - 6) * sz;
      else if (dest[l] == -2) dst = tve.data();
      for (int k = -g; k < z.mz + g; ++k)
        for (int j = -g; j < z.my + g; ++j) {
          in.raw(line.data(), ni * sizeof(double));
          if (dst) std::memcpy(dst + L.at(-g, j, k), line.data(), ni * sizeof(double));
        }
    }
    if (!in.ok) return CB2_ERR_INVALID;
    CB2_TRY(check_cuda(cudaMemcpyAsync(z.bv, bv.data(), 6 * sz * sizeof(double), cudaMemcpyHostToDevice, s)));
    if (p.n_scalar > 0)
      CB2_TRY(check_cuda(cudaMemcpyAsync(z.sv, sv.data(), p.n_scalar * sz * sizeof(double), cudaMemcpyHostToDevice, s)));
    if (two_t && z.tve) {
      if (tve_read) {
        CB2_TRY(check_cuda(cudaMemcpyAsync(z.tve, tve.data(), sz * sizeof(double), cudaMemcpyHostToDevice, s)));
      } else {
        CB2_TRY(check_cuda(cudaMemsetAsync(z.tve, 0, sz * sizeof(double), s)));
      }
    }
    CB2_TRY(check_cuda(cudaStreamSynchronize(s)));
  }
  if (solution_time) *solution_time = t_sol;
  return CB2_OK;
}
