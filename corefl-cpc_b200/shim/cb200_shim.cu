// Reference-side shim: what a COREFL maintainer adds to the reference's own build so that its
// RK3 loop calls libcb200 (include/cb200.h).  It reads the reference's Parameter, Species,
// Reaction, Mesh and Field objects and fills the library's plain-pointer views; nothing here
// copies field data (every array stays the reference's device array).
//
// Build: add this file and include/ to the reference's src/CMakeLists.txt and link
// corefl-cpc_b200/libcb200.so.  tests/test_shim_cpu.py compiles it against the reference's
// headers (both the one- and two-temperature builds) to check that every name used here exists
// there.
//
// Use from src/RK.cuh (RK3<mix>):
//   cb200::Shim shim;
//   if (shim.attach(parameter, species, reaction, mesh, field) != CB2_OK) MpiParallel::exit();
//   ...
//   real dt_io = dt;                                         // the whole step body, RK.cuh:119-237
//   if (cb2_rk3_step(shim.ctx, &dt_io, fixed_time_step ? 1 : 0, nullptr) != CB2_OK) MpiParallel::exit();
#include <map>
#include <string>
#include <variant>
#include <vector>

#include "cb200.h"

#include "BoundCond.h"
#include "ChemData.h"
#include "Field.h"
#include "Mesh.h"
#include "Parameter.h"

namespace cb200 {

// The library's views of one block's DZone arrays (src/Field.h:14-95).  `h` is the host copy of
// the zone (Field::h_ptr), whose arrays are device memory.
inline cb2_zone_view zone_view(cfd::DZone &h, const cfd::Block &blk, bool two_temperature) {
  cb2_zone_view v{};
  v.mx = blk.mx;
  v.my = blk.my;
  v.mz = blk.mz;
  v.ngg = blk.ngg;
  v.cv = h.cv.data();
  v.bv = h.bv.data();
  v.sv = h.sv.data();
  v.qn = h.qn.data();
  v.dq = h.dq.data();
  v.metric = h.metric.data();
  v.jac = h.jac.data();
  v.mul = h.mul.data();
  v.thermal_conductivity = h.thermal_conductivity.data();
  v.rho_D = h.rho_D.data();
  v.acoustic_speed = h.acoustic_speed.data();
  v.gamma = h.gamma.data();
  v.mach = h.mach.data();
  v.fFlux = h.fFlux.data();
  v.gFlux = h.gFlux.data();
  v.hFlux = h.hFlux.data();
  v.vis_flux = h.vis_flux.data();
  v.shock_sensor = h.shock_sensor.data();
  v.dt_local = h.dt_local.data();
  v.reaction_timeScale = h.reaction_timeScale.data();
  v.entropy_fix_delta = h.entropy_fix_delta.data();
  if (two_temperature) {
    v.temperature_ve = h.temperature_ve.data();
    v.thermal_conductivity_ve = h.thermal_conductivity_ve.data();
  }
  return v;
}

// Flattened copies of the species and reaction tables (row-major, as cb2_mechanism reads them);
// they must outlive cb2_init, which copies them to the device.
struct MechTables {
  std::vector<double> low, high, wj, sq, bdc, kbe, tb, t_cut, poly9, elec_theta, elec_g, lt_a, lt_b;
  std::vector<int> stoi_f, stoi_b, n_range, n_level;
  cb2_mechanism mech{};
  cb2_two_temperature two_t{};
};

template <typename M>
std::vector<double> rows(const M &m, int r, int c) {
  std::vector<double> v;
  v.reserve((size_t)r * c);
  for (int i = 0; i < r; ++i)
    for (int j = 0; j < c; ++j) v.push_back(m(i, j));
  return v;
}
template <typename M>
std::vector<int> irows(const M &m, int r, int c) {
  std::vector<int> v;
  v.reserve((size_t)r * c);
  for (int i = 0; i < r; ++i)
    for (int j = 0; j < c; ++j) v.push_back(m(i, j));
  return v;
}

// The mechanism (src/ChemData.h, cfd::Species and cfd::Reaction) as cb2_mechanism, and with
// the two-temperature tables when the species carry them.
inline void fill_mechanism(const cfd::Species &sp, const cfd::Reaction &re, bool vt_relaxation, MechTables &t) {
  const int ns = sp.n_spec, nr = re.n_reac;
  cb2_mechanism &m = t.mech;
  m.n_spec = ns;
  m.n_reac = nr;
  m.mw = sp.mw.data();
  if (sp.nasa_7_or_9 == 9) {
    int mr = 0;
    for (int s = 0; s < ns; ++s) mr = std::max(mr, sp.n_temperature_range[s]);
    t.n_range.assign(sp.n_temperature_range.begin(), sp.n_temperature_range.begin() + ns);
    for (int s = 0; s < ns; ++s) {
      for (int j = 0; j <= mr; ++j) t.t_cut.push_back(j <= sp.n_temperature_range[s] ? sp.temperature_range(s, j) : 0.0);
      for (int j = 0; j < mr; ++j)
        for (int c = 0; c < 9; ++c) t.poly9.push_back(sp.therm_poly_coeff(c, j, s));
    }
    m.therm_nasa_7_9 = 9;
    m.max_range = mr;
    m.n_temperature_range = t.n_range.data();
    m.temperature_range = t.t_cut.data();
    m.therm_poly_coeff = t.poly9.data();
  } else {
    t.low = rows(sp.low_temp_coeff, ns, 7);
    t.high = rows(sp.high_temp_coeff, ns, 7);
    m.therm_nasa_7_9 = 7;
    m.low_temp_coeff = t.low.data();
    m.high_temp_coeff = t.high.data();
    m.t_low = sp.t_low.data();
    m.t_mid = sp.t_mid.data();
    m.t_high = sp.t_high.data();
  }
  m.geometry = sp.geometry.data();
  m.LJ_potent_inv = sp.LJ_potent_inv.data();
  m.vis_coeff = sp.vis_coeff.data();
  t.wj = rows(sp.WjDivWi_to_One4th, ns, ns);
  t.sq = rows(sp.sqrt_WiDivWjPl1Mul8, ns, ns);
  t.bdc = rows(sp.binary_diffusivity_coeff, ns, ns);
  t.kbe = rows(sp.kb_over_eps_jk, ns, ns);
  m.WjDivWi_to_One4th = t.wj.data();
  m.sqrt_WiDivWjPl1Mul8 = t.sq.data();
  m.binary_diffusivity_coeff = t.bdc.data();
  m.kb_over_eps_jk = t.kbe.data();
  m.ZRotF298 = sp.ZRotF298.data();
  if (nr > 0) {
    t.stoi_f = irows(re.stoi_f, nr, ns);
    t.stoi_b = irows(re.stoi_b, nr, ns);
    t.tb = rows(re.third_body_coeff, nr, ns);
    m.reac_type = re.label.data();
    m.rev_type = re.rev_type.data();
    m.stoi_f = t.stoi_f.data();
    m.stoi_b = t.stoi_b.data();
    m.reac_order = re.order.data();
    m.A = re.A.data();
    m.b = re.b.data();
    m.Ea = re.Ea.data();
    m.A2 = re.A2.data();
    m.b2 = re.b2.data();
    m.Ea2 = re.Ea2.data();
    m.third_body_coeff = t.tb.data();
    m.troe_alpha = re.troe_alpha.data();
    m.troe_t3 = re.troe_t3.data();
    m.troe_t1 = re.troe_t1.data();
    m.troe_t2 = re.troe_t2.data();
    if (re.two_temperature_reaction_temperature) {
      m.two_temperature_reaction_temperature = 1;
      m.tcf_a = re.tcf_a.data();
      m.tcf_b = re.tcf_b.data();
      m.tcb_a = re.tcb_a.data();
      m.tcb_b = re.tcb_b.data();
    }
  }
  if (sp.has_two_temperature_data) {
    const int ml = std::max(1, sp.max_electronic_level);
    t.n_level.assign(sp.n_electronic_level.begin(), sp.n_electronic_level.begin() + ns);
    for (int s = 0; s < ns; ++s)
      for (int j = 0; j < ml; ++j) {
        t.elec_theta.push_back(j < sp.n_electronic_level[s] ? sp.electronic_theta(s, j) : 0.0);
        t.elec_g.push_back(j < sp.n_electronic_level[s] ? sp.electronic_g(s, j) : 0.0);
      }
    t.lt_a = rows(sp.lt_a, ns, ns);
    t.lt_b = rows(sp.lt_b, ns, ns);
    cb2_two_temperature &d = t.two_t;
    d.n_spec = ns;
    d.max_level = ml;
    d.theta_v = sp.theta_v.data();
    d.n_level = t.n_level.data();
    d.elec_theta = t.elec_theta.data();
    d.elec_g = t.elec_g.data();
    d.lt_a = t.lt_a.data();
    d.lt_b = t.lt_b.data();
    d.park_sigma = sp.park_sigma.data();
    d.enable_vt_relaxation = vt_relaxation ? 1 : 0;
  }
}

// The face conditions the library applies, by label: the setup's boundary_conditions structs
// (src/BoundCond.cu:80-200 reads the same ones).  An outflow with if_backPressure is the library's
// back-pressure outflow, one with nonReflecting its non-reflecting outflow.  Other types (subsonic inflow, the separate back_pressure type, ...) are
// left to the reference: their label maps to -1.
struct FaceKinds {
  std::map<int, int> type;          // label -> CB2_BC_*
  std::map<int, std::string> name;  // label -> struct name (inflow and wall data)
};

inline FaceKinds face_kinds(const cfd::Parameter &par) {
  FaceKinds k;
  for (const auto &bc : par.get_string_array("boundary_conditions")) {
    const auto &info = par.get_struct(bc);
    const std::string type = std::get<std::string>(info.at("type"));
    const int label = std::get<int>(info.at("label"));
    int t = -1;
    if (type == "wall") t = CB2_BC_WALL;
    else if (type == "symmetry") t = CB2_BC_SYMMETRY;
    else if (type == "inflow") t = CB2_BC_INFLOW;
    else if (type == "outflow") t = CB2_BC_OUTFLOW;
    else if (type == "periodic") t = CB2_BC_PERIODIC;
    else if (type == "farfield") t = CB2_BC_FARFIELD;
    k.type[label] = t;
    k.name[label] = bc;
  }
  return k;
}

// One registered cfd::Boundary as the library takes it: the ranges as read from the boundary
// file (the library repeats register_boundary's ngg extension itself, src/Mesh.cpp:14-32).
inline cb2_face_bc face(const cfd::Boundary &b, int dim, int ngg, bool extended) {
  cb2_face_bc c{};
  c.face = b.face;
  c.direction = b.direction;
  for (int a = 0; a < 3; ++a) {
    c.range_start[a] = b.range_start[a];
    c.range_end[a] = b.range_end[a];
  }
  if (extended) {
    for (int a = 0; a < dim; ++a) {
      if (a == b.face) continue;
      c.range_start[a] += ngg;
      c.range_end[a] -= ngg;
    }
  }
  if (dim == 2) c.range_start[2] = c.range_end[2] = 0;
  return c;
}

struct Shim {
  cb2_ctx *ctx = nullptr;
  MechTables tables;
  std::vector<cfd::Inflow> inflows;      // keep every inflow's and farfield's sv alive until bind
  std::vector<cfd::FarField> farfields;  // has copied it
  std::vector<cfd::Wall> walls;          // and every catalytic wall's yk

  ~Shim() {
    if (ctx) cb2_destroy(ctx);
  }

  // Replaces the DParameter the hot path reads (src/DParameter.cu:6-436) and binds every block:
  // its DZone arrays, its face conditions and its inner faces.
  int attach(cfd::Parameter &par, const cfd::Species &sp, const cfd::Reaction &re, cfd::Mesh &mesh,
             std::vector<cfd::Field> &field) {
    const int i_eve = par.get_int("i_eve");
    const bool two_t = i_eve >= 0;
    cb2_param_view pv{};
    pv.abi_version = CB2_ABI_VERSION;
    pv.dim = mesh.dimension;
    pv.n_var = par.get_int("n_var");
    pv.n_spec = sp.n_spec;
    pv.n_scalar = par.get_int("n_scalar");
    pv.n_scalar_transported = par.get_int("n_scalar_transported");
    pv.inviscid_scheme = par.get_int("inviscid_scheme");
    pv.reconstruction = par.get_int("reconstruction");
    pv.limiter = par.get_int("limiter");
    pv.viscous_order = par.get_int("viscous_order");
    pv.positive_preserving = par.get_bool("positive_preserving") ? 1 : 0;
    pv.gradP_in_diffusion_flux = par.get_bool("gradPInDiffusionFlux") ? 1 : 0;
    pv.reaction = par.get_int("reaction");
    pv.shock_sensor = par.get_int("shock_sensor");
    pv.sensor_eps = par.get_real("shockSensor_epsilon");
    pv.sensor_threshold = par.get_real("shockSensor_threshold");
    pv.entropy_fix_factor = par.get_real("entropy_fix_factor");
    pv.Pr = par.get_real("prandtl_number");
    pv.cfl = par.get_real("cfl");
    pv.rho_ref = par.get_real("rho_inf");
    pv.v_ref = par.get_real("v_inf");
    pv.p_ref = par.get_real("p_inf");
    pv.c_ref = par.get_real("speed_of_sound");
    pv.limit_flow = par.get_bool("limit_flow") ? 1 : 0;
    pv.dt = par.get_real("dt");
    pv.precision = CB2_PREC_FP64;
    if (sp.n_spec > 0) {
      fill_mechanism(sp, re, two_t && par.get_bool("enable_vt_relaxation"), tables);
      pv.mech = &tables.mech;
      if (two_t) pv.two_t = &tables.two_t;
    }
    int rc = cb2_init(&pv, &ctx);
    if (rc != CB2_OK) return rc;

    const FaceKinds kinds = face_kinds(par);
    const bool extended = pv.viscous_order == 2;  // need_extend_boundary, src/Mesh.cpp:637
    for (int b = 0; b < mesh.n_block; ++b) {
      cfd::Block &blk = mesh[b];
      std::vector<cb2_face_bc> faces;
      for (const cfd::Boundary &bd : blk.boundary) {
        const auto it = kinds.type.find(bd.type_label);
        if (it == kinds.type.end() || it->second < 0) return CB2_ERR_UNSUPPORTED;
        cb2_face_bc c = face(bd, pv.dim, blk.ngg, extended);
        c.type = it->second;
        const std::string &name = kinds.name.at(bd.type_label);
        if (c.type == CB2_BC_INFLOW) {
          inflows.emplace_back(name, sp, par);
          const cfd::Inflow &in = inflows.back();
          c.rho = in.density;
          c.u = in.u;
          c.v = in.v;
          c.w = in.w;
          c.p = in.pressure;
          c.T = in.temperature;
          c.sv = in.sv;
        } else if (c.type == CB2_BC_FARFIELD) {
          farfields.emplace_back(name, const_cast<cfd::Species &>(sp), par);
          const cfd::FarField &ff = farfields.back();
          c.rho = ff.density;
          c.u = ff.u;
          c.v = ff.v;
          c.w = ff.w;
          c.p = ff.pressure;
          c.T = ff.temperature;
          c.wall_temperature_ve = ff.temperature_ve > 0 ? ff.temperature_ve : 0.0;
          c.sv = ff.sv;
        } else if (c.type == CB2_BC_OUTFLOW) {
          cfd::Outflow out(name, par);  // back pressure (if_backPressure) as p > 0
          if (out.if_backPressure == 1) c.p = out.backPressure;
          if (out.nonReflecting > 0) c.type |= CB2_BC_NONREFLECTING;  // nonReflectingBoundary's faces
        } else if (c.type == CB2_BC_WALL) {
          walls.emplace_back(par.get_struct(name), par, sp);
          const cfd::Wall &wall = walls.back();
          c.wall_temperature = wall.thermal_type == cfd::Wall::ThermalType::isothermal ? wall.temperature : 0.0;
          c.wall_temperature_ve = wall.temperature_ve > 0 ? wall.temperature_ve : 0.0;
          if (wall.if_blow_shock_wave) {  // blowing wall: its window and the freestream velocity
            c.blow_shock_wave = 1;
            c.blow_coefficient = wall.blow_shock_wave_coefficient;
            c.blow_start_step = wall.blow_shock_wave_start_step;
            c.blow_end_step = wall.blow_shock_wave_end_step;
            c.u = par.get_real("ux_inf");
            c.v = par.get_real("uy_inf");
            c.w = par.get_real("uz_inf");
          }
          if (wall.catalytic_type == 1) c.sv = wall.yk;  // fully catalytic: the wall mass fractions
        }
        faces.push_back(c);
      }
      cb2_zone_view v = zone_view(*field[b].h_ptr, blk, two_t);
      rc = cb2_bind_block(ctx, b, &v, faces.data(), (int)faces.size());
      if (rc != CB2_OK) return rc;
    }
    for (int b = 0; b < mesh.n_block; ++b) {
      std::vector<cb2_inner_face> in;
      for (const cfd::InnerFace &f : mesh[b].inner_face) {
        cb2_inner_face c{};
        for (int a = 0; a < 3; ++a) {
          c.range_start[a] = f.range_start[a];
          c.range_end[a] = f.range_end[a];
          c.target_start[a] = f.target_start[a];
          c.target_end[a] = f.target_end[a];
          c.src_tar[a] = f.src_tar[a];
          c.loop_dir[a] = f.loop_dir[a];
          c.target_loop_dir[a] = f.target_loop_dir[a];
          c.n_point[a] = f.n_point[a];
        }
        c.face = f.face;
        c.direction = f.direction;
        c.target_block = f.target_block;
        c.target_face = f.target_face;
        c.target_direction = f.target_direction;
        in.push_back(c);
      }
      if (!in.empty()) {
        rc = cb2_bind_inner_faces(ctx, b, in.data(), (int)in.size());
        if (rc != CB2_OK) return rc;
      }
    }
    return CB2_OK;
  }
};

}  // namespace cb200
