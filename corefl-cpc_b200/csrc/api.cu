// extern "C" entry points of libcb200 (declared in include/cb200.h) and the RK3 step
// orchestration (the stage body of RK3<mix>, src/RK.cuh:107-237).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include "common.cuh"
#include "launch.h"
#include "sweep.cuh"
#include "block_batch.h"
#include "cb200_serve.h"

namespace cb2 {

static thread_local std::string g_cuda_error;

void set_cuda_error(cudaError_t e) { g_cuda_error = cudaGetErrorString(e); }

// ---- per-launch profiler ------------------------------------------------------------------
struct Profiler {
  struct Rec {
    std::string name;
    cudaEvent_t a, b;
  };
  std::vector<Rec> open;                      // recorded, not yet resolved
  std::vector<cudaEvent_t> pool;              // reusable events
  std::vector<std::string> names;             // aggregated results
  std::vector<unsigned long long> counts;
  std::vector<double> total_ms;
  cudaEvent_t take() {
    if (!pool.empty()) {
      cudaEvent_t e = pool.back();
      pool.pop_back();
      return e;
    }
    cudaEvent_t e;
    cudaEventCreate(&e);
    return e;
  }
  void resolve() {
    for (auto &r : open) {
      cudaEventSynchronize(r.b);
      float ms = 0;
      cudaEventElapsedTime(&ms, r.a, r.b);
      size_t k = 0;
      while (k < names.size() && names[k] != r.name) ++k;
      if (k == names.size()) {
        names.push_back(r.name);
        counts.push_back(0);
        total_ms.push_back(0);
      }
      counts[k] += 1;
      total_ms[k] += ms;
      pool.push_back(r.a);
      pool.push_back(r.b);
    }
    open.clear();
  }
  ~Profiler() {
    for (auto &r : open) { cudaEventDestroy(r.a); cudaEventDestroy(r.b); }
    for (auto e : pool) cudaEventDestroy(e);
  }
};

thread_local Profiler *g_prof = nullptr;

void prof_begin(Profiler *p, const char *name, cudaStream_t s) {
  Profiler::Rec r{name, p->take(), p->take()};
  cudaEventRecord(r.a, s);
  p->open.push_back(r);
}

void prof_end(Profiler *p, cudaStream_t s) {
  if (!p->open.empty()) cudaEventRecord(p->open.back().b, s);
}

struct Block {
  bool bound = false;
  cb2_zone_view v{};
  Zone z{};
  std::vector<FaceBC> faces;
  std::vector<cb2_inner_face> inner;  // inner faces of a multi-block grid (cb2_bind_inner_faces)
  int *d_btype = nullptr;     // six face flag arrays, one allocation
  float *d_f32 = nullptr;     // mixed form: bv32 and met32, one allocation
  double *d_face_sv = nullptr;  // inflow faces' scalars, one allocation
};

}  // namespace cb2

using namespace cb2;

struct cb2_ctx {
  Param p{};
  cb2_param_view view{};
  void *d_tables = nullptr;  // mechanism tables (one allocation)
  unsigned *d_status = nullptr;
  double *d_dtmin = nullptr;     // running min of the CFL dt
  double *d_partial = nullptr;   // per-CTA partial minima of the reduction
  int n_partial = 0;
  std::vector<Block> blocks;
  unsigned long long n_launch = 0;
  Profiler *prof = nullptr;  // non-null while profiling is enabled
  unsigned long long bind_gen = 0;  // bumped by every cb2_bind_block (invalidates the step graph)
  // device-driven step loop of cb2_rk3_run: one CUDA graph whose WHILE node replays one step
  struct StepGraph {
    cudaStream_t capture = nullptr;  // capture stream (non-blocking, created on first use)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    unsigned long long gen = ~0ull;  // bind_gen the graph was captured at
    int fixed_dt = -1;               // the dt mode it was captured in
    unsigned long long launches = 0; // kernels per step inside the graph
  } sg;
  RunState *d_run = nullptr;  // time, t_end, dt, step counter of the graph loop
  // batched closed blocks (cb2_block_batch_*)
  BlockCase *d_batch = nullptr;
  int n_batch = 0;            // capacity of d_batch
  int *d_queue = nullptr;     // work counter of the persistent batch grid
  int batch_ni = kNI;         // y/z tile width of the batch kernel (cb2_block_batch_autotune)
  int batch_cs = 8;           // CTAs per thread-block cluster sharing one batched block
  // multi-block steps: the per-block work of a stage runs on these streams concurrently, forked
  // from the caller's stream and joined back before anything that reads another block
  std::vector<cudaStream_t> branch;
  cudaEvent_t ev_fork = nullptr;
  std::vector<cudaEvent_t> ev_join;
};

namespace cb2 {
const Param *ctx_param(const cb2_ctx *ctx) { return ctx ? &ctx->p : nullptr; }
// The zones of the context's blocks 0 .. n-1, all of which must be bound.
int ctx_zones(const cb2_ctx *ctx, std::vector<Zone> &zones) {
  zones.clear();
  if (!ctx || ctx->blocks.empty()) return CB2_ERR_INVALID;
  for (const Block &B : ctx->blocks) {
    if (!B.bound) return CB2_ERR_INVALID;
    zones.push_back(B.z);
  }
  return CB2_OK;
}
}  // namespace cb2

namespace {
// Makes the context's profiler current for this thread while an entry point runs.
struct ProfGuard {
  Profiler *prev;
  explicit ProfGuard(cb2_ctx *ctx) : prev(g_prof) { g_prof = ctx ? ctx->prof : nullptr; }
  ~ProfGuard() { g_prof = prev; }
};
}  // namespace

namespace {

int fail_cuda(cudaError_t e) {
  set_cuda_error(e);
  return CB2_ERR_CUDA;
}

// Copies the mechanism into one device allocation and fills the device pointers of Mech.
int upload_mechanism(const cb2_mechanism &m, const cb2_two_temperature *tt, cb2_ctx *ctx) {
  const int ns = m.n_spec, nr = m.n_reac;
  std::vector<double> buf;
  std::vector<int> ibuf;
  struct DSlot { const double **dst; size_t off; };
  struct ISlot { const int **dst; size_t off; };
  std::vector<DSlot> ds;
  std::vector<ISlot> is;
  Mech &d = ctx->p.mech;
  auto addd = [&](const double **dst, const double *src, size_t n) {
    ds.push_back({dst, buf.size()});
    for (size_t a = 0; a < n; ++a) buf.push_back(src ? src[a] : 0.0);
  };
  auto addi = [&](const int **dst, const int *src, size_t n) {
    is.push_back({dst, ibuf.size()});
    for (size_t a = 0; a < n; ++a) ibuf.push_back(src ? src[a] : 0);
  };
  // 1/mw, R_u/mw and 1/(1/mw) exactly as DParameter and the transport kernel derive them
  std::vector<double> imw(ns), rg(ns), mw2(ns);
  for (int s = 0; s < ns; ++s) {
    imw[s] = 1.0 / m.mw[s];
    rg[s] = kRu / m.mw[s];
    mw2[s] = 1.0 / imw[s];
  }
  addd(&d.imw, imw.data(), ns);
  addd(&d.gas_const, rg.data(), ns);
  addd(&d.mw, mw2.data(), ns);
  addd(&d.lo, m.low_temp_coeff, (size_t)ns * 7);
  addd(&d.hi, m.high_temp_coeff, (size_t)ns * 7);
  addd(&d.t_low, m.t_low, ns);
  addd(&d.t_mid, m.t_mid, ns);
  addd(&d.t_high, m.t_high, ns);
  addd(&d.geometry, m.geometry, ns);
  addd(&d.lj_inv, m.LJ_potent_inv, ns);
  addd(&d.vis_coeff, m.vis_coeff, ns);
  addd(&d.wjwi14, m.WjDivWi_to_One4th, (size_t)ns * ns);
  addd(&d.sqwiwj8, m.sqrt_WiDivWjPl1Mul8, (size_t)ns * ns);
  addd(&d.bdc, m.binary_diffusivity_coeff, (size_t)ns * ns);
  addd(&d.kbe, m.kb_over_eps_jk, (size_t)ns * ns);
  addd(&d.zrot, m.ZRotF298, ns);
  // natural logs of the reduced-temperature factors: the transport kernel forms the powers
  // (T k)^a as exp(a (ln T + ln k)) with one ln T per node (usable when every factor is > 0)
  {
    std::vector<double> lk((size_t)ns * ns, 0.0), ll(ns, 0.0);
    bool ok = m.kb_over_eps_jk && m.LJ_potent_inv;
    for (size_t a = 0; ok && a < (size_t)ns * ns; ++a) ok = m.kb_over_eps_jk[a] > 0;
    for (int a = 0; ok && a < ns; ++a) ok = m.LJ_potent_inv[a] > 0;
    if (ok) {
      for (size_t a = 0; a < (size_t)ns * ns; ++a) lk[a] = std::log(m.kb_over_eps_jk[a]);
      for (int a = 0; a < ns; ++a) ll[a] = std::log(m.LJ_potent_inv[a]);
    }
    addd(&d.ln_kbe, lk.data(), (size_t)ns * ns);
    addd(&d.ln_lj_inv, ll.data(), ns);
    d.transport_ln = ok ? 1 : 0;
  }
  d.ln_temp_p = std::log(kPatm / kRu * 1e-3);
  addd(&d.A, m.A, nr);
  addd(&d.b, m.b, nr);
  addd(&d.Ea, m.Ea, nr);
  addd(&d.A2, m.A2, nr);
  addd(&d.b2, m.b2, nr);
  addd(&d.Ea2, m.Ea2, nr);
  addd(&d.tbc, m.third_body_coeff, (size_t)nr * ns);
  addd(&d.troe_alpha, m.troe_alpha, nr);
  addd(&d.troe_t3, m.troe_t3, nr);
  addd(&d.troe_t1, m.troe_t1, nr);
  addd(&d.troe_t2, m.troe_t2, nr);
  addi(&d.reac_type, m.reac_type, nr);
  addi(&d.rev_type, m.rev_type, nr);
  addi(&d.stoi_f, m.stoi_f, (size_t)nr * ns);
  addi(&d.stoi_b, m.stoi_b, (size_t)nr * ns);
  addi(&d.reac_order, m.reac_order, nr);
  const bool nasa9 = m.therm_nasa_7_9 == 9;
  if (nasa9) {
    const size_t mr = (size_t)m.max_range;
    addd(&d.t_cut, m.temperature_range, ns * (mr + 1));
    addd(&d.poly9, m.therm_poly_coeff, ns * mr * 9);
    addi(&d.n_range, m.n_temperature_range, ns);
  }
  const bool park = m.two_temperature_reaction_temperature != 0 && nr > 0;
  if (park) {
    addd(&d.tcf_a, m.tcf_a, nr);
    addd(&d.tcf_b, m.tcf_b, nr);
    addd(&d.tcb_a, m.tcb_a, nr);
    addd(&d.tcb_b, m.tcb_b, nr);
  }
  if (tt) {
    const size_t ml = (size_t)tt->max_level;
    addd(&d.theta_v, tt->theta_v, ns);
    addd(&d.elec_theta, tt->elec_theta, ns * ml);
    addd(&d.elec_g, tt->elec_g, ns * ml);
    addd(&d.lt_a, tt->lt_a, (size_t)ns * ns);
    addd(&d.lt_b, tt->lt_b, (size_t)ns * ns);
    addd(&d.park_sigma, tt->park_sigma, ns);
    addi(&d.n_level, tt->n_level, ns);
    // Electronic levels past which the partition sums stop changing (see ve_energy): for
    // ascending level temperatures theta_1 < theta_2 < ..., a level l >= 2 with
    // theta_l - theta_1 > A T contributes g_l theta_l^k exp(-theta_l / T) (k = 0, 1, 2) below
    // 2^-54 of the first excited level's term, i.e. below half an ulp of every running sum, when
    // A = ln(max_l (g_l / g_1) max(1, (theta_l / theta_1)^2)) + 54 ln 2 (+ 1 of margin).
    // Unsorted or degenerate level tables get A = inf (every level is summed).
    std::vector<double> cut((size_t)ns, INFINITY);
    for (int sp = 0; sp < ns; ++sp) {
      const int nl = tt->n_level[sp];
      const double *th = tt->elec_theta + (size_t)sp * ml, *gg = tt->elec_g + (size_t)sp * ml;
      if (nl < 3 || !(th[1] > 0) || !(gg[1] > 0) || th[0] > th[1]) continue;
      bool ok = true;
      double worst = 1.0;
      for (int l = 2; l < nl && ok; ++l) {
        if (!(th[l] >= th[l - 1]) || gg[l] < 0) ok = false;
        const double r = th[l] / th[1];
        worst = std::max(worst, gg[l] / gg[1] * std::max(1.0, r * r));
      }
      if (ok) cut[(size_t)sp] = std::log(worst) + 54.0 * std::log(2.0) + 1.0;
    }
    addd(&d.elec_cut, cut.data(), ns);
  }
  const size_t bd = buf.size() * sizeof(double), bi = ibuf.size() * sizeof(int);
  char *dev = nullptr;
  cudaError_t e = cudaMalloc(&dev, bd + bi + 16);
  if (e != cudaSuccess) return fail_cuda(e);
  ctx->d_tables = dev;
  if (bd) { e = cudaMemcpy(dev, buf.data(), bd, cudaMemcpyHostToDevice); if (e) return fail_cuda(e); }
  if (bi) { e = cudaMemcpy(dev + bd, ibuf.data(), bi, cudaMemcpyHostToDevice); if (e) return fail_cuda(e); }
  for (auto &s : ds) *s.dst = reinterpret_cast<const double *>(dev) + s.off;
  for (auto &s : is) *s.dst = reinterpret_cast<const int *>(dev + bd) + s.off;
  d.n_spec = ns;
  d.n_reac = nr;
  d.nasa9 = nasa9 ? 1 : 0;
  d.max_range = nasa9 ? m.max_range : 0;
  d.park = park ? 1 : 0;
  d.max_level = tt ? tt->max_level : 0;
  d.enable_vt = tt && tt->enable_vt_relaxation ? 1 : 0;
  return CB2_OK;
}

// register_boundary (src/Mesh.cpp:14-32): the face is the first dimension whose start and
// end coincide, the low face points to -1; with `extend` the tangential ranges grow by ngg,
// and for 2-D blocks the k range becomes [-ngg, ngg] (or [0, 0] without extension).
FaceBC register_face(const cb2_face_bc &f, int dim, int ngg, bool extend) {
  FaceBC b{};
  b.type = f.type & ~CB2_BC_NONREFLECTING;
  b.nonreflecting = (f.type & CB2_BC_NONREFLECTING) != 0;
  for (int a = 0; a < 3; ++a) { b.start[a] = f.range_start[a]; b.end[a] = f.range_end[a]; }
  b.face = f.face;
  b.direction = f.direction;
  const int gx = extend ? ngg : 0;
  for (int a = 0; a < dim; ++a) {
    if (a == b.face) continue;
    if (b.end[a] < b.start[a]) { int t = b.end[a]; b.end[a] = b.start[a]; b.start[a] = t; }
    b.start[a] -= gx;
    b.end[a] += gx;
  }
  if (dim == 2) { b.start[2] = -gx; b.end[2] = gx; }
  b.rho = f.rho; b.u = f.u; b.v = f.v; b.w = f.w; b.p = f.p; b.T = f.T; b.wall_T = f.wall_temperature;
  b.wall_Tve = f.wall_temperature_ve;
  b.sv = nullptr;  // set at bind to the device copy of f.sv
  b.blow = b.type == CB2_BC_WALL && f.blow_shock_wave != 0;
  b.blow_start = f.blow_start_step;
  b.blow_end = f.blow_end_step;
  b.blow_coef = f.blow_coefficient;
  return b;
}

Zone make_zone(const cb2_zone_view &v) {
  Zone z{};
  z.mx = v.mx; z.my = v.my; z.mz = v.mz; z.ngg = v.ngg;
  z.L = make_layout(v.mx, v.my, v.mz, v.ngg);
  z.L0 = make_layout(v.mx, v.my, v.mz, 0);
  z.L1 = make_layout(v.mx, v.my, v.mz, 1);
  z.cv = v.cv; z.bv = v.bv; z.sv = v.sv; z.qn = v.qn; z.dq = v.dq; z.metric = v.metric; z.jac = v.jac;
  z.mul = v.mul; z.kappa = v.thermal_conductivity; z.rhoD = v.rho_D; z.acoustic = v.acoustic_speed;
  z.gamma = v.gamma; z.mach = v.mach; z.fF = v.fFlux; z.gF = v.gFlux; z.hF = v.hFlux; z.visf = v.vis_flux;
  z.shock = v.shock_sensor; z.dtl = v.dt_local; z.rts = v.reaction_timeScale; z.efd = v.entropy_fix_delta;
  z.tve = v.temperature_ve;
  z.kappa_ve = v.thermal_conductivity_ve;
  return z;
}

Block *get_block(cb2_ctx *ctx, int blk) {
  if (!ctx || blk < 0 || blk >= (int)ctx->blocks.size() || !ctx->blocks[blk].bound) return nullptr;
  return &ctx->blocks[blk];
}

// The two-temperature model is built for the pointwise stage operations (stage update with
// the VT relaxation, cv from bv); its flux terms are not, so the other entry points refuse it.
bool two_temperature(const cb2_ctx *ctx) { return ctx && ctx->p.i_eve >= 0; }

unsigned two_temperature_rhs_terms(const cb2_ctx *ctx);

// Faces whose ghost fill is built for two temperatures: all of them.  Periodic, outflow and
// symmetry copy bv, every scalar (e_ve included) and T_ve, inflow sets the given scalars, the wall
// sets T_ve and e_ve, and each rebuilds cv with the T_ve sync, as the reference's apply_* kernels
// do (src/BoundCond.cu:2130-3440).
bool two_temperature_faces(const Block &B) {
  for (const FaceBC &f : B.faces)
    if (f.type != CB2_BC_PERIODIC && f.type != CB2_BC_OUTFLOW && f.type != CB2_BC_WALL &&
        f.type != CB2_BC_SYMMETRY && f.type != CB2_BC_INFLOW && f.type != CB2_BC_FARFIELD)
      return false;
  return true;
}

// Whether the whole two-temperature step is built for this context: every residual term the
// settings ask for and the ghost fill of every bound block.
bool two_temperature_step(const cb2_ctx *ctx) {
  unsigned need = CB2_RHS_INVISCID;
  if (ctx->p.viscous_order > 0) need |= CB2_RHS_VISCOUS;
  if (ctx->p.reaction) need |= CB2_RHS_CHEMISTRY;
  if ((need & ~two_temperature_rhs_terms(ctx)) != 0) return false;
  for (const Block &B : ctx->blocks)
    if (B.bound && !two_temperature_faces(B)) return false;
  return true;
}

// The residual terms built for two-temperature contexts: the chemistry source with the control
// temperatures and the e_ve source, the 2nd- and 8th-order viscous fluxes with the e_ve terms,
// and the characteristic WENO fluxes with rho e_ve as a scalar row.
// An inviscid context has no viscous term to build, so asking for it (CB2_RHS_ALL) is no refusal.
unsigned two_temperature_rhs_terms(const cb2_ctx *ctx) {
  unsigned m = CB2_RHS_CHEMISTRY;
  if (ctx->p.viscous_order == 2 || ctx->p.viscous_order == 8 || ctx->p.viscous_order == 0) m |= CB2_RHS_VISCOUS;
  if (ctx->p.inviscid_scheme == CB2_INV_WENO5_CH || ctx->p.inviscid_scheme == CB2_INV_WENO7_CH ||
      ctx->p.inviscid_scheme == CB2_INV_AUSMP || ctx->p.inviscid_scheme == CB2_INV_HLLC)
    m |= CB2_RHS_INVISCID;
  return m;
}

int count(cb2_ctx *ctx, int n) {
  ctx->n_launch += (unsigned long long)n;
  return CB2_OK;
}

}  // namespace

extern "C" {

const char *cb2_strerror(int code) {
  switch (code) {
    case CB2_OK: return "ok";
    case CB2_ERR_CUDA: return "CUDA runtime error";
    case CB2_ERR_INVALID: return "invalid argument";
    case CB2_ERR_NONPHYSICAL: return "non-physical state";
    case CB2_ERR_TIMEOUT: return "device wait timed out";
    case CB2_ERR_UNSUPPORTED: return "unsupported scheme/model combination";
    case CB2_ERR_NOMEM: return "out of device memory";
    default: return "unknown error";
  }
}

const char *cb2_last_cuda_error(void) { return g_cuda_error.c_str(); }

unsigned long long cb2_launch_count(const cb2_ctx *ctx) { return ctx ? ctx->n_launch : 0ull; }

int cb2_init(const cb2_param_view *pv, cb2_ctx **out) {
  if (!pv || !out) return CB2_ERR_INVALID;
  *out = nullptr;
  if (pv->abi_version != CB2_ABI_VERSION) return CB2_ERR_INVALID;
  const int ns = pv->mech ? pv->mech->n_spec : 0;
  if (pv->n_spec != ns) return CB2_ERR_INVALID;
  if (ns != 0 && ns != 5 && ns != 9) return CB2_ERR_UNSUPPORTED;
  if (ns > 0) {
    const cb2_mechanism &m = *pv->mech;
    if (m.therm_nasa_7_9 == 9) {
      // NASA9 multi-range tables: every species has 1..max_range ranges with rising boundaries
      if (m.max_range < 1 || m.max_range > 4 || !m.n_temperature_range || !m.temperature_range ||
          !m.therm_poly_coeff)
        return CB2_ERR_INVALID;
      for (int s = 0; s < ns; ++s) {
        const int n = m.n_temperature_range[s];
        if (n < 1 || n > m.max_range) return CB2_ERR_INVALID;
        const double *cut = m.temperature_range + s * (m.max_range + 1);
        for (int r = 0; r < n; ++r)
          if (!(cut[r] > 0 && cut[r] < cut[r + 1])) return CB2_ERR_INVALID;
      }
    } else if (m.therm_nasa_7_9 != 0 && m.therm_nasa_7_9 != 7) {
      return CB2_ERR_INVALID;
    } else if (!m.low_temp_coeff || !m.high_temp_coeff || !m.t_low || !m.t_mid || !m.t_high) {
      return CB2_ERR_INVALID;
    }
    if (m.two_temperature_reaction_temperature && m.n_reac > 0 &&
        (!m.tcf_a || !m.tcf_b || !m.tcb_a || !m.tcb_b))
      return CB2_ERR_INVALID;
  }
  // two-temperature: e_ve is the scalar after the species (i_eve = n_spec)
  const cb2_two_temperature *tt = pv->two_t;
  if (tt) {
    if (ns == 0 || tt->n_spec != ns || tt->max_level < 1 || !tt->theta_v || !tt->n_level || !tt->elec_theta ||
        !tt->elec_g || !tt->lt_a || !tt->lt_b || !tt->park_sigma)
      return CB2_ERR_INVALID;
    for (int s = 0; s < ns; ++s)
      if (tt->n_level[s] < 0 || tt->n_level[s] > tt->max_level) return CB2_ERR_INVALID;
    if (pv->n_var != 6 + ns || pv->n_scalar != ns + 1 || pv->n_scalar_transported != ns + 1)
      return CB2_ERR_INVALID;
    if (pv->precision != CB2_PREC_FP64) return CB2_ERR_UNSUPPORTED;
  } else if (pv->n_var != 5 + ns || pv->n_scalar != ns) {
    return CB2_ERR_UNSUPPORTED;
  }
  const int sch = pv->inviscid_scheme;
  const bool weno_ch = sch == CB2_INV_WENO5_CH || sch == CB2_INV_WENO7_CH || sch == CB2_INV_WENO5_CP ||
                       sch == CB2_INV_WENO7_CP;
  const bool pvpath = sch == CB2_INV_AUSMP || sch == CB2_INV_HLLC || sch == CB2_INV_ROE || (sch == 1 && ns == 0);
  if (!weno_ch && !pvpath) return CB2_ERR_UNSUPPORTED;
  // two temperatures: AUSM+ and HLLC are the primitive-variable fluxes of the reference's
  // two-temperature build
  if (tt && pvpath && sch != CB2_INV_AUSMP && sch != CB2_INV_HLLC) return CB2_ERR_UNSUPPORTED;
  if (pvpath) {
    const int r = pv->reconstruction;
    if (!(r == 1 || r == 2 || r == 3 || r == 5 || r == 7)) return CB2_ERR_INVALID;
  }
  if (pv->viscous_order != 0 && pv->viscous_order != 2 && pv->viscous_order != 8) return CB2_ERR_INVALID;
  // the positivity limiter acts on the species rows of the characteristic-WENO fluxes
  if (pv->positive_preserving && (ns == 0 || !(sch == CB2_INV_WENO5_CH || sch == CB2_INV_WENO7_CH)))
    return CB2_ERR_UNSUPPORTED;
  if (pv->reaction && ns == 0) return CB2_ERR_INVALID;
  if (pv->limit_flow && !(pv->rho_ref > 0 && pv->p_ref > 0)) return CB2_ERR_INVALID;
  if (pv->precision != CB2_PREC_FP64 && pv->precision != CB2_PREC_MIXED) return CB2_ERR_INVALID;
  // mixed form: FP32 sweeps for WENO5/7 primitive reconstruction with AUSM+/HLLC/Roe
  if (pv->precision == CB2_PREC_MIXED &&
      (!pvpath || sch == 1 || (pv->reconstruction != CB2_REC_WENO5 && pv->reconstruction != CB2_REC_WENO7)))
    return CB2_ERR_UNSUPPORTED;
  cb2_ctx *ctx = new cb2_ctx;
  ctx->view = *pv;
  Param &p = ctx->p;
  p.dim = pv->dim;
  p.n_var = pv->n_var;
  p.n_spec = ns;
  p.n_scalar = pv->n_scalar;
  p.n_scalar_transported = pv->n_scalar_transported;
  p.n_reac = pv->mech ? pv->mech->n_reac : 0;
  p.inviscid_scheme = sch;
  p.reconstruction = pv->reconstruction;
  p.limiter = pv->limiter;
  p.viscous_order = pv->viscous_order;
  p.positive_preserving = pv->positive_preserving;
  p.gradP = pv->gradP_in_diffusion_flux;
  p.reaction = pv->reaction;
  p.shock_sensor = pv->shock_sensor;
  p.sensor_eps = pv->sensor_eps;
  p.sensor_threshold = pv->sensor_threshold;
  p.entropy_fix_factor = pv->entropy_fix_factor;
  p.Pr = pv->Pr;
  p.cfl = pv->cfl;
  p.rho_ref = pv->rho_ref;
  p.v_ref = pv->v_ref;
  // weno_eps_scale = (rho_inf v_inf)^2 (src/DParameter.cu:29-32)
  p.weno_eps_scale = pv->rho_ref * pv->v_ref * pv->rho_ref * pv->v_ref;
  p.mu_constant = pv->mu_constant;
  p.precision = pv->precision;
  p.dt = pv->dt;
  p.limit_flow = pv->limit_flow;
  if (p.limit_flow) {
    // bounds of src/DParameter.cu:371-387
    p.lf_ll[0] = 1e-6 * pv->rho_ref;
    p.lf_ul[0] = 1e+3 * pv->rho_ref;
    const double vref = fabs(pv->v_ref) < 1 ? pv->c_ref : pv->v_ref;
    for (int l = 1; l < 4; ++l) {
      p.lf_ll[l] = -1000 * vref;
      p.lf_ul[l] = 1000 * vref;
    }
    p.lf_ll[4] = 1e-6 * pv->p_ref;
    p.lf_ul[4] = 1e+3 * pv->p_ref;
  }
  int rc = CB2_OK;
  p.i_eve = tt ? ns : -1;
  if (pv->mech) rc = upload_mechanism(*pv->mech, tt, ctx);
  if (rc == CB2_OK) {
    cudaError_t e = cudaMalloc(&ctx->d_status, sizeof(unsigned) + 2 * sizeof(double));
    if (e != cudaSuccess) rc = fail_cuda(e);
    else {
      e = cudaMemset(ctx->d_status, 0, sizeof(unsigned));
      if (e != cudaSuccess) rc = fail_cuda(e);
      ctx->d_dtmin = reinterpret_cast<double *>(reinterpret_cast<char *>(ctx->d_status) + sizeof(double));
      p.status = ctx->d_status;
    }
  }
  if (rc != CB2_OK) {
    cb2_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return CB2_OK;
}

void cb2_destroy(cb2_ctx *ctx) {
  if (!ctx) return;
  for (cudaStream_t b : ctx->branch) cudaStreamDestroy(b);
  for (cudaEvent_t e : ctx->ev_join) cudaEventDestroy(e);
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->sg.exec) cudaGraphExecDestroy(ctx->sg.exec);
  if (ctx->sg.graph) cudaGraphDestroy(ctx->sg.graph);
  if (ctx->sg.capture) cudaStreamDestroy(ctx->sg.capture);
  cudaFree(ctx->d_run);
  cudaFree(ctx->d_batch);
  cudaFree(ctx->d_queue);
  for (auto &b : ctx->blocks) {
    cudaFree(b.d_btype);
    cudaFree(b.d_f32);
    cudaFree(b.d_face_sv);
  }
  cudaFree(ctx->d_tables);
  cudaFree(ctx->d_status);
  cudaFree(ctx->d_partial);
  delete ctx->prof;
  delete ctx;
}

int cb2_profile_enable(cb2_ctx *ctx, int on) {
  if (!ctx) return CB2_ERR_INVALID;
  if (on && !ctx->prof) ctx->prof = new Profiler;
  if (!on && ctx->prof) {
    ctx->prof->resolve();
    delete ctx->prof;
    ctx->prof = nullptr;
  }
  return CB2_OK;
}

int cb2_profile_count(cb2_ctx *ctx) {
  if (!ctx || !ctx->prof) return 0;
  ctx->prof->resolve();
  return (int)ctx->prof->names.size();
}

int cb2_profile_entry(cb2_ctx *ctx, int idx, char *name, int name_len, unsigned long long *count,
                      double *total_ms) {
  if (!ctx || !ctx->prof || !name || name_len < 1 || !count || !total_ms) return CB2_ERR_INVALID;
  Profiler &p = *ctx->prof;
  p.resolve();
  if (idx < 0 || idx >= (int)p.names.size()) return CB2_ERR_INVALID;
  std::snprintf(name, (size_t)name_len, "%s", p.names[idx].c_str());
  *count = p.counts[idx];
  *total_ms = p.total_ms[idx];
  return CB2_OK;
}

int cb2_profile_reset(cb2_ctx *ctx) {
  if (!ctx || !ctx->prof) return CB2_ERR_INVALID;
  ctx->prof->resolve();
  ctx->prof->names.clear();
  ctx->prof->counts.clear();
  ctx->prof->total_ms.clear();
  return CB2_OK;
}

int cb2_bind_block(cb2_ctx *ctx, int blk, const cb2_zone_view *v, const cb2_face_bc *faces, int n_faces) {
  if (!ctx || !v || blk < 0 || n_faces < 0 || (n_faces > 0 && !faces)) return CB2_ERR_INVALID;
  if (v->mx < 1 || v->my < 1 || v->mz < 1 || v->ngg < 1) return CB2_ERR_INVALID;
  const Param &p = ctx->p;
  const int sch = p.inviscid_scheme;
  const bool pvpath = !(sch == CB2_INV_WENO5_CH || sch == CB2_INV_WENO7_CH || sch == CB2_INV_WENO5_CP ||
                        sch == CB2_INV_WENO7_CP);
  const int need_g = (sch == CB2_INV_WENO7_CH || sch == CB2_INV_WENO7_CP ||
                      (pvpath && p.reconstruction == CB2_REC_WENO7) || p.viscous_order == 8) ? 4
                     : (sch == CB2_INV_WENO5_CH || sch == CB2_INV_WENO5_CP ||
                        (pvpath && p.reconstruction == CB2_REC_WENO5)) ? 3 : 2;
  if (v->ngg < need_g) return CB2_ERR_INVALID;
  // the sweeps index one padded k plane with 32-bit positions
  if ((long long)(v->mx + 2 * v->ngg) * (v->my + 2 * v->ngg) >= (1LL << 31)) return CB2_ERR_UNSUPPORTED;
  if (!v->cv || !v->bv || !v->dq || !v->metric || !v->jac || !v->qn) return CB2_ERR_INVALID;
  if (p.n_spec > 0 && (!v->sv || !v->acoustic_speed || !v->gamma || !v->mul || !v->thermal_conductivity ||
                       !v->rho_D))
    return CB2_ERR_INVALID;
  if (p.i_eve >= 0 && (!v->sv || !v->temperature_ve)) return CB2_ERR_INVALID;
  if (p.viscous_order > 0 && !v->mul) return CB2_ERR_INVALID;
  if (p.viscous_order == 8 && (!v->fFlux || !v->gFlux || !v->hFlux)) return CB2_ERR_INVALID;
  if (p.inviscid_scheme == CB2_INV_ROE && !v->entropy_fix_delta) return CB2_ERR_INVALID;
  if (p.sensor_threshold > 1e-10 && !v->shock_sensor) return CB2_ERR_INVALID;
  for (int f = 0; f < n_faces; ++f) {
    const auto &b = faces[f];
    if (b.face < 0 || b.face > 2 || (b.direction != 1 && b.direction != -1)) return CB2_ERR_INVALID;
    const int t = b.type & ~CB2_BC_NONREFLECTING;
    if (t != CB2_BC_OUTFLOW && t != CB2_BC_PERIODIC && t != CB2_BC_WALL && t != CB2_BC_SYMMETRY &&
        t != CB2_BC_INFLOW && t != CB2_BC_FARFIELD)
      return CB2_ERR_INVALID;
    // only an outflow face can be non-reflecting (Outflow::nonReflecting)
    if ((b.type & CB2_BC_NONREFLECTING) && t != CB2_BC_OUTFLOW) return CB2_ERR_INVALID;
    // an inflow or farfield state of a mixture carries its scalars (Y_k, e_ve)
    if ((b.type == CB2_BC_INFLOW || b.type == CB2_BC_FARFIELD) && p.n_scalar > 0 && !b.sv) return CB2_ERR_INVALID;
    if (b.type == CB2_BC_FARFIELD && !(b.rho > 0 && b.p > 0 && b.T > 0)) return CB2_ERR_INVALID;
  }
  if ((int)ctx->blocks.size() <= blk) ctx->blocks.resize(blk + 1);
  Block &B = ctx->blocks[blk];
  cudaFree(B.d_btype);
  B.d_btype = nullptr;
  cudaFree(B.d_f32);
  B.d_f32 = nullptr;
  cudaFree(B.d_face_sv);
  B.d_face_sv = nullptr;
  B.v = *v;
  B.z = make_zone(*v);
  B.faces.clear();
  const bool extend = p.viscous_order == 2;
  for (int f = 0; f < n_faces; ++f) B.faces.push_back(register_face(faces[f], p.dim, v->ngg, extend));
  {
    // the inflow faces' scalars go to the device with the face (Inflow::sv lives in device memory)
    std::vector<double> all_sv;
    std::vector<int> at(n_faces, -1);
    const int nsc = std::max(p.n_scalar, 1);
    for (int f = 0; f < n_faces; ++f) {
      const bool wall = faces[f].type == CB2_BC_WALL;
      if (!(faces[f].type == CB2_BC_INFLOW || faces[f].type == CB2_BC_FARFIELD || (wall && faces[f].sv))) continue;
      // a catalytic wall's sv holds the n_spec wall mass fractions (Wall::yk)
      const int nin = wall ? p.n_spec : p.n_scalar;
      at[f] = (int)all_sv.size();
      for (int l = 0; l < nsc; ++l) all_sv.push_back(faces[f].sv && l < nin ? faces[f].sv[l] : 0.0);
    }
    if (!all_sv.empty()) {
      cudaError_t e = cudaMalloc(&B.d_face_sv, all_sv.size() * sizeof(double));
      if (e != cudaSuccess) return fail_cuda(e);
      e = cudaMemcpy(B.d_face_sv, all_sv.data(), all_sv.size() * sizeof(double), cudaMemcpyHostToDevice);
      if (e != cudaSuccess) return fail_cuda(e);
      for (int f = 0; f < n_faces; ++f)
        if (at[f] >= 0) B.faces[f].sv = B.d_face_sv + at[f];
    }
  }
  // physical-boundary flags per face node, from the raw (unextended) ranges (src/Mesh.cpp:855-900)
  const int mx = v->mx, my = v->my, mz = v->mz;
  std::vector<int> il(my * mz, 0), ir(my * mz, 0), jl(mx * mz, 0), jr(mx * mz, 0), kl(mx * my, 0), kr(mx * my, 0);
  for (int f = 0; f < n_faces; ++f) {
    const auto &b = faces[f];
    if (b.type == CB2_BC_PERIODIC) continue;
    int lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = b.range_start[a] < b.range_end[a] ? b.range_start[a] : b.range_end[a];
      hi[a] = b.range_start[a] < b.range_end[a] ? b.range_end[a] : b.range_start[a];
    }
    for (int a = 0; a < 3; ++a) { if (lo[a] < 0) lo[a] = 0; }
    if (hi[0] >= mx) hi[0] = mx - 1;
    if (hi[1] >= my) hi[1] = my - 1;
    if (hi[2] >= mz) hi[2] = mz - 1;
    for (int k = lo[2]; k <= hi[2]; ++k)
      for (int j = lo[1]; j <= hi[1]; ++j)
        for (int i = lo[0]; i <= hi[0]; ++i) {
          const int t = b.type & ~CB2_BC_NONREFLECTING;
          if (b.face == 0) (b.direction < 0 ? il : ir)[j + k * my] = t;
          else if (b.face == 1) (b.direction < 0 ? jl : jr)[i + k * mx] = t;
          else (b.direction < 0 ? kl : kr)[i + j * mx] = t;
        }
  }
  const size_t n_all = il.size() + ir.size() + jl.size() + jr.size() + kl.size() + kr.size();
  cudaError_t e = cudaMalloc(&B.d_btype, n_all * sizeof(int));
  if (e != cudaSuccess) return fail_cuda(e);
  std::vector<int> all;
  all.reserve(n_all);
  for (auto *vv : {&il, &ir, &jl, &jr, &kl, &kr}) all.insert(all.end(), vv->begin(), vv->end());
  e = cudaMemcpy(B.d_btype, all.data(), n_all * sizeof(int), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return fail_cuda(e);
  size_t off = 0;
  const int *base = B.d_btype;
  B.z.bt.il = base + off; off += il.size();
  B.z.bt.ir = base + off; off += ir.size();
  B.z.bt.jl = base + off; off += jl.size();
  B.z.bt.jr = base + off; off += jr.size();
  B.z.bt.kl = base + off; off += kl.size();
  B.z.bt.kr = base + off;
  // reduction scratch sized for the largest bound block
  const int np = min_reduce_partials((long long)mx * my * mz);
  if (np > ctx->n_partial) {
    cudaFree(ctx->d_partial);
    ctx->d_partial = nullptr;
    e = cudaMalloc(&ctx->d_partial, np * sizeof(double));
    if (e != cudaSuccess) { ctx->n_partial = 0; return fail_cuda(e); }
    ctx->n_partial = np;
  }
  if (p.precision == CB2_PREC_MIXED) {
    // FP32 copies: bv (refreshed per residual) and metric + J (snapshot of the bound block)
    const size_t sz = (size_t)B.z.L.sz;
    auto up = [](size_t n) { return (n + 63) / 64 * 64; };  // each copy starts on a 256-byte boundary
    const size_t off = up(6 * sz), offf = off + up(10 * sz);
    const size_t nflux = p.viscous_order == 8 && visc8_f32(p) ? up((size_t)p.n_var * sz) : 0;
    e = cudaMalloc(&B.d_f32, (offf + 3 * nflux) * sizeof(float));
    if (e != cudaSuccess) return fail_cuda(e);
    B.z.bv32 = B.d_f32;
    B.z.met32 = B.d_f32 + off;
    if (nflux) {
      B.z.fF32 = B.d_f32 + offf;
      B.z.gF32 = B.z.fF32 + nflux;
      B.z.hF32 = B.z.gF32 + nflux;
    }
    int nl = 0;
    CB2_TRY(launch_to_f32(v->metric, B.z.met32, 9 * sz, nullptr, nl));
    CB2_TRY(launch_to_f32(v->jac, B.z.met32 + 9 * sz, sz, nullptr, nl));
    CB2_TRY(check_cuda(cudaDeviceSynchronize()));
  }
  B.bound = true;
  ++ctx->bind_gen;
  return CB2_OK;
}

int cb2_store_qn(cb2_ctx *ctx, int blk, void *stream) {
  Block *B = get_block(ctx, blk);
  if (!B) return CB2_ERR_INVALID;
  ProfGuard pg(ctx);
  cudaStream_t s = (cudaStream_t)stream;
  ProfScope prof("store_qn", s);
  const size_t bytes = (size_t)B->z.L.sz * ctx->p.n_var * sizeof(double);
  return check_cuda(cudaMemcpyAsync(B->z.qn, B->z.cv, bytes, cudaMemcpyDeviceToDevice, s));
}

int cb2_rhs(cb2_ctx *ctx, int blk, unsigned mask, void *stream) {
  Block *B = get_block(ctx, blk);
  if (!B) return CB2_ERR_INVALID;
  if (two_temperature(ctx) && (mask & CB2_RHS_ALL & ~two_temperature_rhs_terms(ctx))) return CB2_ERR_UNSUPPORTED;
  // the 8th-order node fluxes of a multi-block grid are exchanged across the inner faces between
  // all blocks' node fluxes and any block's divergence: cb2_viscous does that for every block
  if ((mask & CB2_RHS_VISCOUS) && ctx->p.viscous_order == 8 && !B->inner.empty()) return CB2_ERR_UNSUPPORTED;
  const bool accumulate = (mask & CB2_RHS_ACCUMULATE) != 0;
  ProfGuard pg(ctx);
  cudaStream_t s = (cudaStream_t)stream;
  const Param &p = ctx->p;
  int nl = 0;
  if (p.precision == CB2_PREC_MIXED) {
    ProfScope prof("bv_to_f32", s);
    CB2_TRY(launch_to_f32(B->z.bv, B->z.bv32, 6 * (size_t)B->z.L.sz, s, nl));
  }
  const bool visc = (mask & CB2_RHS_VISCOUS) && p.viscous_order > 0;
  const bool pv = p.inviscid_scheme != CB2_INV_WENO5_CH && p.inviscid_scheme != CB2_INV_WENO7_CH &&
                  p.inviscid_scheme != CB2_INV_WENO5_CP && p.inviscid_scheme != CB2_INV_WENO7_CP;
  // mixed form of air with 8th-order viscous terms and WENO7 primitive sweeps over all three
  // directions: the sweeps take the viscous divergence along their direction (the tile already
  // holds the +-4 stencil), and the x sweep, the first term of the residual, assigns dq.  The FP64
  // form keeps the separate divergence kernel: its tile with the node fluxes (55 KB, more
  // registers) runs fewer CTAs per SM, which cost more than the divergence pass it saves.
  Param pf = p;
  pf.visc8_fused = visc && p.viscous_order == 8 && p.n_spec == 0 && (mask & CB2_RHS_INVISCID) && pv &&
                           p.reconstruction == CB2_REC_WENO7 && !B->z.sweep_mask && p.precision == CB2_PREC_MIXED &&
                           !accumulate
                       ? 2
                       : 0;
  // no zeroing of dq when the first term assigns it, or when the caller's dq is added to
  const bool assign = !accumulate && (pf.visc8_fused || (visc && viscous_assigns_dq(p)));
  if (!assign && !accumulate) {
    ProfScope prof("zero_dq", s);
    CB2_TRY(check_cuda(cudaMemsetAsync(B->z.dq, 0, (size_t)B->z.L0.sz * p.n_var * sizeof(double), s)));
  }
  if (visc) CB2_TRY(launch_viscous(B->z, pf, B->faces.data(), (int)B->faces.size(), assign, s, nl));
  if ((mask & CB2_RHS_CHEMISTRY) && p.reaction) CB2_TRY(launch_chemistry(B->z, p, s, nl));
  if (mask & CB2_RHS_INVISCID) {
    if (p.inviscid_scheme == CB2_INV_WENO5_CH || p.inviscid_scheme == CB2_INV_WENO7_CH)
      CB2_TRY(launch_inviscid_char(B->z, p, s, nl));
    else if (p.inviscid_scheme == CB2_INV_WENO5_CP || p.inviscid_scheme == CB2_INV_WENO7_CP)
      CB2_TRY(launch_inviscid_comp(B->z, p, s, nl));
    else
      CB2_TRY(launch_inviscid_pv(B->z, pf, s, nl));
    // the non-reflecting outflow faces correct dq after the inviscid flux (src/RK.cuh:190-193)
    CB2_TRY(launch_nonreflecting(B->z, p, B->faces.data(), (int)B->faces.size(), s, nl));
  }
  return count(ctx, nl);
}

static bool inner_face_in_range(const Zone &z, const Zone &zt, const cb2_inner_face &f);

int cb2_viscous(cb2_ctx *ctx, void *stream) {
  if (!ctx || ctx->blocks.empty()) return CB2_ERR_INVALID;
  if (two_temperature(ctx) && !(two_temperature_rhs_terms(ctx) & CB2_RHS_VISCOUS)) return CB2_ERR_UNSUPPORTED;
  ProfGuard pg(ctx);
  cudaStream_t s = (cudaStream_t)stream;
  const Param &p = ctx->p;
  Param pf = p;
  pf.visc8_fused = 0;
  const bool assign = p.viscous_order > 0 && viscous_assigns_dq(p);
  const int nb = (int)ctx->blocks.size();
  int nl = 0;
  // every block's dq and (order 8) node fluxes
  for (int b = 0; b < nb; ++b) {
    Block &B = ctx->blocks[b];
    if (!B.bound) continue;
    if (p.precision == CB2_PREC_MIXED) {
      ProfScope prof("bv_to_f32", s);
      CB2_TRY(launch_to_f32(B.z.bv, B.z.bv32, 6 * (size_t)B.z.L.sz, s, nl));
    }
    if (!assign) {
      ProfScope prof("zero_dq", s);
      CB2_TRY(check_cuda(cudaMemsetAsync(B.z.dq, 0, (size_t)B.z.L0.sz * p.n_var * sizeof(double), s)));
    }
    if (p.viscous_order > 0)
      CB2_TRY(launch_viscous(B.z, pf, B.faces.data(), (int)B.faces.size(), assign, s, nl, p.viscous_order == 8 ? 1 : 0));
  }
  if (p.viscous_order == 8) {
    // the node fluxes across the inner faces, then each block's periodic exchange and divergence
    // (exchange_value: inner faces before periodic ones, src/DataCommunication.cu:437-485)
    for (int b = 0; b < nb; ++b) {
      Block &B = ctx->blocks[b];
      if (!B.bound) continue;
      for (const cb2_inner_face &f : B.inner) {
        Block *T = get_block(ctx, f.target_block);
        if (!T || !inner_face_in_range(B.z, T->z, f)) return CB2_ERR_INVALID;
        CB2_TRY(launch_inner_flux_exchange(B.z, T->z, p, f, s, nl));
      }
    }
    for (int b = 0; b < nb; ++b) {
      Block &B = ctx->blocks[b];
      if (B.bound) CB2_TRY(launch_viscous(B.z, pf, B.faces.data(), (int)B.faces.size(), assign, s, nl, 2));
    }
  }
  return count(ctx, nl);
}

int cb2_shock_sensor(cb2_ctx *ctx, int blk, void *stream) {
  Block *B = get_block(ctx, blk);
  if (!B || !B->z.shock) return CB2_ERR_INVALID;
  if (two_temperature(ctx)) return CB2_ERR_UNSUPPORTED;
  ProfGuard pg(ctx);
  int nl = 0;
  CB2_TRY(launch_shock_sensor(B->z, ctx->p, (cudaStream_t)stream, nl));
  return count(ctx, nl);
}

int cb2_stage_update(cb2_ctx *ctx, int blk, double dt, int rk, void *stream) {
  Block *B = get_block(ctx, blk);
  if (!B || rk < 0 || rk > 2) return CB2_ERR_INVALID;
  ProfGuard pg(ctx);
  int nl = 0;
  CB2_TRY(launch_stage_update(B->z, ctx->p, dt, rk, (cudaStream_t)stream, nl));
  return count(ctx, nl);
}

int cb2_autotune(cb2_ctx *ctx, int blk, int *tile_ni_out, void *stream) {
  Block *B = get_block(ctx, blk);
  if (!B) return CB2_ERR_INVALID;
  if (two_temperature(ctx)) return CB2_ERR_UNSUPPORTED;
  const Param &p = ctx->p;
  Zone &z = B->z;
  cudaStream_t s = (cudaStream_t)stream;
  const int sch = p.inviscid_scheme;
  const bool tunable = (sch == CB2_INV_AUSMP || sch == CB2_INV_HLLC || sch == CB2_INV_ROE) && p.n_spec == 0 &&
                       (p.reconstruction == CB2_REC_WENO5 || p.reconstruction == CB2_REC_WENO7);
  const int ndir = z.mz > 1 ? 3 : 2;
  if (tunable) {
    // candidates run on a scratch residual, so the caller's dq is untouched
    double *scratch = nullptr;
    CB2_TRY(check_cuda(cudaMalloc(&scratch, (size_t)z.L0.sz * p.n_var * sizeof(double))));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = check_cuda(cudaEventCreate(&e0));
    if (rc == CB2_OK) rc = check_cuda(cudaEventCreate(&e1));
    Zone zt = z;
    zt.dq = scratch;
    Profiler *saved = ctx->prof;
    ctx->prof = nullptr;  // the trial launches are not part of the profile
    ProfGuard pg(ctx);
    for (int d = 1; d < ndir && rc == CB2_OK; ++d) {
      float best_ms = 1e30f;
      int best = 0;
      zt.sweep_mask = 1u << d;
      for (int c = 0; c < 3 && rc == CB2_OK; ++c) {
        zt.tile_ni[d] = kTileNI[c];
        int nl = 0;
        rc = launch_inviscid_pv(zt, p, s, nl);  // warm-up (also sets the shared-memory limit)
        if (rc == CB2_OK) rc = check_cuda(cudaEventRecord(e0, s));
        for (int r = 0; r < 3 && rc == CB2_OK; ++r) rc = launch_inviscid_pv(zt, p, s, nl);
        if (rc == CB2_OK) rc = check_cuda(cudaEventRecord(e1, s));
        if (rc == CB2_OK) rc = check_cuda(cudaEventSynchronize(e1));
        float ms = 0;
        if (rc == CB2_OK) rc = check_cuda(cudaEventElapsedTime(&ms, e0, e1));
        if (rc == CB2_OK && ms < best_ms) {
          best_ms = ms;
          best = kTileNI[c];
        }
      }
      if (rc == CB2_OK) z.tile_ni[d] = best;
    }
    ctx->prof = saved;
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(scratch);
    if (rc != CB2_OK) return rc;
    ++ctx->bind_gen;  // a captured step graph holds the old tile widths
  }
  if (tile_ni_out)
    for (int d = 0; d < 3; ++d) tile_ni_out[d] = d == 0 ? 0 : (z.tile_ni[d] ? z.tile_ni[d] : kNI);
  return CB2_OK;
}

int cb2_set_tile_widths(cb2_ctx *ctx, int blk, const int *tile_ni) {
  Block *B = get_block(ctx, blk);
  if (!B || !tile_ni) return CB2_ERR_INVALID;
  for (int d = 1; d < 3; ++d) {
    bool ok = tile_ni[d] == 0;
    for (int c = 0; c < 3; ++c) ok = ok || tile_ni[d] == kTileNI[c];
    if (!ok) return CB2_ERR_INVALID;
  }
  for (int d = 1; d < 3; ++d) B->z.tile_ni[d] = tile_ni[d];
  ++ctx->bind_gen;
  return CB2_OK;
}

int cb2_vt_relaxation(cb2_ctx *ctx, int blk, double dt_stage, void *stream) {
  Block *B = get_block(ctx, blk);
  if (!B || !(dt_stage >= 0.0)) return CB2_ERR_INVALID;
  if (!two_temperature(ctx)) return CB2_ERR_UNSUPPORTED;
  ProfGuard pg(ctx);
  int nl = 0;
  CB2_TRY(launch_vt_relaxation(B->z, ctx->p, dt_stage, (cudaStream_t)stream, nl));
  return count(ctx, nl);
}

int cb2_boundary(cb2_ctx *ctx, int blk, void *stream) {
  Block *B = get_block(ctx, blk);
  if (!B) return CB2_ERR_INVALID;
  if (two_temperature(ctx) && !two_temperature_faces(*B)) return CB2_ERR_UNSUPPORTED;
  ProfGuard pg(ctx);
  int nl = 0;
  cudaStream_t s = (cudaStream_t)stream;
  CB2_TRY(launch_boundary(B->z, ctx->p, B->faces.data(), (int)B->faces.size(), s, nl));
  if (ctx->p.dim == 2 && B->z.mz == 1) CB2_TRY(launch_eliminate_k_gradient(B->z, ctx->p, s, nl));
  return count(ctx, nl);
}

int cb2_bind_inner_faces(cb2_ctx *ctx, int blk, const cb2_inner_face *faces, int n_faces) {
  Block *B = get_block(ctx, blk);
  if (!B || n_faces < 0 || (n_faces > 0 && !faces)) return CB2_ERR_INVALID;
  for (int f = 0; f < n_faces; ++f) {
    const cb2_inner_face &q = faces[f];
    if (q.face < 0 || q.face > 2 || (q.direction != 1 && q.direction != -1) || q.target_block < 0) return CB2_ERR_INVALID;
    for (int a = 0; a < 3; ++a) {
      if (q.src_tar[a] < 0 || q.src_tar[a] > 2 || (q.loop_dir[a] != 1 && q.loop_dir[a] != -1) ||
          (q.target_loop_dir[a] != 1 && q.target_loop_dir[a] != -1 && q.target_loop_dir[a] != 0) || q.n_point[a] < 1)
        return CB2_ERR_INVALID;
      if (q.range_end[a] - q.range_start[a] != q.loop_dir[a] * (q.n_point[a] - 1)) return CB2_ERR_INVALID;
    }
  }
  B->inner.assign(faces, faces + n_faces);
  ++ctx->bind_gen;
  return CB2_OK;
}

// Whether every node an inner face reads or writes lies inside both blocks' padded arrays.
static bool inner_face_in_range(const Zone &z, const Zone &zt, const cb2_inner_face &f) {
  const int ext[3] = {z.mx, z.my, z.mz}, extt[3] = {zt.mx, zt.my, zt.mz};
  for (int a = 0; a < 3; ++a) {
    const int lo = std::min(f.range_start[a], f.range_end[a]), hi = std::max(f.range_start[a], f.range_end[a]);
    if (lo < -z.ngg || hi > ext[a] - 1 + z.ngg) return false;
    // the target index along a moves with the step along src_tar[a]: check both ends
    const int b = f.src_tar[a];
    const int d0 = 0, d1 = f.loop_dir[b] * (f.n_point[b] - 1);
    const int t0 = f.target_start[a] + f.target_loop_dir[a] * d0, t1 = f.target_start[a] + f.target_loop_dir[a] * d1;
    if (std::min(t0, t1) < -zt.ngg || std::max(t0, t1) > extt[a] - 1 + zt.ngg) return false;
  }
  return true;
}

int cb2_halo(cb2_ctx *ctx, void *stream) {
  if (!ctx) return CB2_ERR_INVALID;
  ProfGuard pg(ctx);
  cudaStream_t s = (cudaStream_t)stream;
  int nl = 0;
  const int nb = (int)ctx->blocks.size();
  for (int b = 0; b < nb; ++b) {
    Block &B = ctx->blocks[b];
    if (!B.bound) continue;
    for (const cb2_inner_face &f : B.inner) {
      Block *T = get_block(ctx, f.target_block);
      if (!T || !inner_face_in_range(B.z, T->z, f)) return CB2_ERR_INVALID;
      CB2_TRY(launch_inner_exchange(B.z, T->z, ctx->p, f, s, nl));
    }
  }
  for (int b = 0; b < nb; ++b) {
    Block &B = ctx->blocks[b];
    if (B.bound && !B.inner.empty() && ctx->p.dim == 2 && B.z.mz == 1)
      CB2_TRY(launch_eliminate_k_gradient(B.z, ctx->p, s, nl));
  }
  return count(ctx, nl);
}

static bool any_inner_faces(const cb2_ctx *ctx) {
  for (const Block &B : ctx->blocks)
    if (B.bound && !B.inner.empty()) return true;
  return false;
}

int cb2_properties(cb2_ctx *ctx, int blk, void *stream) {
  Block *B = get_block(ctx, blk);
  if (!B) return CB2_ERR_INVALID;
  ProfGuard pg(ctx);
  int nl = 0;
  CB2_TRY(launch_properties(B->z, ctx->p, (cudaStream_t)stream, nl));
  return count(ctx, nl);
}

int cb2_cv_from_bv(cb2_ctx *ctx, int blk, void *stream) {
  Block *B = get_block(ctx, blk);
  if (!B) return CB2_ERR_INVALID;
  ProfGuard pg(ctx);
  int nl = 0;
  CB2_TRY(launch_cv_from_bv(B->z, ctx->p, (cudaStream_t)stream, nl));
  return count(ctx, nl);
}

// Enqueues the CFL dt of every bound block and their minimum into ctx->d_dtmin.
static int enqueue_cfl_dt(cb2_ctx *ctx, cudaStream_t s) {
  int nl = 0;
  CB2_TRY(launch_set_value(ctx->d_dtmin, 1e+6, s, nl));
  for (auto &B : ctx->blocks) {
    if (!B.bound) continue;
    if (!B.z.dtl) return CB2_ERR_INVALID;
    CB2_TRY(launch_local_dt(B.z, ctx->p, s, nl));
    const long long n = (long long)B.z.mx * B.z.my * B.z.mz;
    CB2_TRY(launch_min_reduce(B.z.dtl, n, ctx->d_partial, min_reduce_partials(n), ctx->d_dtmin, s, nl));
  }
  return count(ctx, nl);
}

int cb2_cfl_dt(cb2_ctx *ctx, double *dt_out, void *stream) {
  if (!ctx || !dt_out) return CB2_ERR_INVALID;
  ProfGuard pg(ctx);
  cudaStream_t s = (cudaStream_t)stream;
  CB2_TRY(enqueue_cfl_dt(ctx, s));
  double dt = 0;
  CB2_TRY(check_cuda(cudaMemcpyAsync(&dt, ctx->d_dtmin, sizeof(double), cudaMemcpyDeviceToHost, s)));
  CB2_TRY(check_cuda(cudaStreamSynchronize(s)));
  *dt_out = dt;
  ctx->p.dt = dt;  // the global step, as update_dt_global leaves it (src/RK.cuh:151)
  return CB2_OK;
}

}  // extern "C"

// qn <- cv and the shock sensor of every bound block: the part of a step before its dt.
static int enqueue_step_head(cb2_ctx *ctx, void *stream) {
  const int nb = (int)ctx->blocks.size();
  for (int b = 0; b < nb; ++b)
    if (ctx->blocks[b].bound) CB2_TRY(cb2_store_qn(ctx, b, stream));
  if (ctx->p.sensor_threshold > 1e-10)  // hybrid linear/WENO weights (src/RK.cuh:139-143)
    for (int b = 0; b < nb; ++b)
      if (ctx->blocks[b].bound) CB2_TRY(cb2_shock_sensor(ctx, b, stream));
  return CB2_OK;
}

// Branch streams and events for concurrent per-block work (created on first use).
constexpr int kMaxBranches = 8;

static int ensure_branches(cb2_ctx *ctx, int n) {
  if (!ctx->ev_fork) CB2_TRY(check_cuda(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming)));
  while ((int)ctx->branch.size() < n) {
    cudaStream_t st = nullptr;
    CB2_TRY(check_cuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)));
    ctx->branch.push_back(st);
    cudaEvent_t e = nullptr;
    CB2_TRY(check_cuda(cudaEventCreateWithFlags(&e, cudaEventDisableTiming)));
    ctx->ev_join.push_back(e);
  }
  return CB2_OK;
}

// Branches 0..n-1 start after everything enqueued on s so far.
static int fork_branches(cb2_ctx *ctx, cudaStream_t s, int n) {
  CB2_TRY(check_cuda(cudaEventRecord(ctx->ev_fork, s)));
  for (int i = 0; i < n; ++i) CB2_TRY(check_cuda(cudaStreamWaitEvent(ctx->branch[i], ctx->ev_fork, 0)));
  return CB2_OK;
}

// s continues after everything enqueued on branches 0..n-1.
static int join_branches(cb2_ctx *ctx, cudaStream_t s, int n) {
  for (int i = 0; i < n; ++i) {
    CB2_TRY(check_cuda(cudaEventRecord(ctx->ev_join[i], ctx->branch[i])));
    CB2_TRY(check_cuda(cudaStreamWaitEvent(s, ctx->ev_join[i], 0)));
  }
  return CB2_OK;
}

// The three stages of a step (src/RK.cuh:164-237).  With several blocks, each block's residual,
// stage update and boundary conditions -- and later its properties -- touch only that block's
// arrays, so they run on branch streams concurrently (the latency-bound face kernels and the
// sweeps of one block fill the SMs the others leave idle); the inner-face exchange, which reads
// other blocks, runs on the caller's stream after the join.  Under graph capture the branches
// become parallel paths of the graph.
static int enqueue_stages(cb2_ctx *ctx, double dt, void *stream) {
  const int nb = (int)ctx->blocks.size();
  const bool halo = any_inner_faces(ctx);
  cudaStream_t s = (cudaStream_t)stream;
  int nbound = 0;
  for (auto &B : ctx->blocks) nbound += B.bound ? 1 : 0;
  const int nbr = nbound > 1 ? std::min(nbound, kMaxBranches) : 0;
  if (nbr) CB2_TRY(ensure_branches(ctx, nbr));
  auto on = [&](int slot) { return nbr ? (void *)ctx->branch[slot % nbr] : stream; };
  // 8th-order viscous terms across inner faces: every block's viscous term first (cb2_viscous,
  // as the reference's compute_viscous_flux runs over the whole mesh), then the rest of each
  // block's residual added to it
  const bool visc_all = halo && ctx->p.viscous_order == 8;
  const unsigned mask = visc_all ? (CB2_RHS_CHEMISTRY | CB2_RHS_INVISCID | CB2_RHS_ACCUMULATE) : CB2_RHS_ALL;
  for (int rk = 0; rk < 3; ++rk) {
    if (visc_all) CB2_TRY(cb2_viscous(ctx, stream));
    if (nbr) CB2_TRY(fork_branches(ctx, s, nbr));
    for (int b = 0, slot = 0; b < nb; ++b) {
      if (!ctx->blocks[b].bound) continue;
      void *sb = on(slot++);
      CB2_TRY(cb2_rhs(ctx, b, mask, sb));
      CB2_TRY(cb2_stage_update(ctx, b, dt, rk, sb));
      CB2_TRY(cb2_boundary(ctx, b, sb));
    }
    if (nbr) CB2_TRY(join_branches(ctx, s, nbr));
    if (halo) CB2_TRY(cb2_halo(ctx, stream));  // data_communication (src/RK.cuh:216-226)
    if (nbr) CB2_TRY(fork_branches(ctx, s, nbr));
    for (int b = 0, slot = 0; b < nb; ++b)
      if (ctx->blocks[b].bound) CB2_TRY(cb2_properties(ctx, b, on(slot++)));
    if (nbr) CB2_TRY(join_branches(ctx, s, nbr));
  }
  return CB2_OK;
}

static void drop_step_graph(cb2_ctx *ctx) {
  auto &g = ctx->sg;
  if (g.exec) cudaGraphExecDestroy(g.exec);
  if (g.graph) cudaGraphDestroy(g.graph);
  g.exec = nullptr;
  g.graph = nullptr;
  g.gen = ~0ull;
  g.fixed_dt = -1;
}

// Builds the graph of cb2_rk3_run: a WHILE node whose body, captured from the same enqueue
// functions cb2_rk3_step uses, is one step followed by k_run_advance.  Inside the body every
// kernel reads the step's dt from the device (Param::dt_dev): RunState::dt in fixed mode, the
// CFL minimum otherwise.  Per-launch profiling is off inside the graph.
static int capture_step_graph(cb2_ctx *ctx, int fixed_dt) {
  auto &g = ctx->sg;
  drop_step_graph(ctx);
  if (!g.capture) CB2_TRY(check_cuda(cudaStreamCreateWithFlags(&g.capture, cudaStreamNonBlocking)));
  if (!ctx->d_run) CB2_TRY(check_cuda(cudaMalloc(&ctx->d_run, sizeof(RunState))));
  CB2_TRY(check_cuda(cudaGraphCreate(&g.graph, 0)));
  cudaGraphConditionalHandle h;
  int rc = check_cuda(cudaGraphConditionalHandleCreate(&h, g.graph, 1u, cudaGraphCondAssignDefault));
  cudaGraphNodeParams np{};
  cudaGraphNode_t node;
  if (rc == CB2_OK) {
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    rc = check_cuda(cudaGraphAddNode(&node, g.graph, nullptr, 0, &np));
  }
  if (rc != CB2_OK) {
    drop_step_graph(ctx);
    return rc;
  }
  const Param saved = ctx->p;
  Profiler *saved_prof = ctx->prof;
  const unsigned long long n0 = ctx->n_launch;
  ctx->prof = nullptr;
  ctx->p.dt_dev = fixed_dt ? &ctx->d_run->dt : ctx->d_dtmin;
  cudaStream_t s = g.capture;
  rc = check_cuda(cudaStreamBeginCaptureToGraph(s, np.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                                cudaStreamCaptureModeRelaxed));
  if (rc == CB2_OK) {
    rc = enqueue_step_head(ctx, s);
    if (rc == CB2_OK && !fixed_dt) rc = enqueue_cfl_dt(ctx, s);
    if (rc == CB2_OK) rc = enqueue_stages(ctx, 0.0, s);
    int nl = 0;
    if (rc == CB2_OK) rc = launch_run_advance(ctx->d_run, ctx->p.dt_dev, ctx->d_status, h, s, nl);
    cudaGraph_t body = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s, &body);
    if (rc == CB2_OK && e != cudaSuccess) rc = fail_cuda(e);
  }
  g.launches = ctx->n_launch - n0 + 1;  // the step's kernels and k_run_advance
  ctx->n_launch = n0;
  ctx->p = saved;
  ctx->prof = saved_prof;
  if (rc == CB2_OK) rc = check_cuda(cudaGraphInstantiate(&g.exec, g.graph, 0));
  if (rc != CB2_OK) {
    drop_step_graph(ctx);
    return rc;
  }
  g.gen = ctx->bind_gen;
  g.fixed_dt = fixed_dt;
  return CB2_OK;
}

extern "C" {

int cb2_rk3_step(cb2_ctx *ctx, double *dt_inout, int fixed_dt, void *stream) {
  if (!ctx || !dt_inout) return CB2_ERR_INVALID;
  if (two_temperature(ctx) && !two_temperature_step(ctx)) return CB2_ERR_UNSUPPORTED;
  ProfGuard pg(ctx);
  CB2_TRY(enqueue_step_head(ctx, stream));
  double dt = *dt_inout;
  if (!fixed_dt) {
    CB2_TRY(cb2_cfl_dt(ctx, &dt, stream));
    *dt_inout = dt;
  }
  ctx->p.dt = dt;
  ++ctx->p.step;  // the step this call takes (RK3 counts it before its stages)
  return enqueue_stages(ctx, dt, stream);
}

int cb2_set_step(cb2_ctx *ctx, long long step) {
  if (!ctx) return CB2_ERR_INVALID;
  ctx->p.step = step;
  return CB2_OK;
}

int cb2_rk3_run(cb2_ctx *ctx, double dt, int fixed_dt, long long max_steps, double t_end, double *time_inout,
                long long *steps_out, double *dt_last_out, void *stream) {
  if (!ctx || !time_inout || !steps_out || max_steps < 0 || std::isnan(t_end)) return CB2_ERR_INVALID;
  if (two_temperature(ctx) && !two_temperature_step(ctx)) return CB2_ERR_UNSUPPORTED;
  if (fixed_dt && !(dt > 0.0 && dt < 1e300)) return CB2_ERR_INVALID;
  *steps_out = 0;
  if (max_steps == 0 || !(*time_inout < t_end)) return CB2_OK;
  bool any = false;
  for (auto &B : ctx->blocks) {
    any = any || B.bound;
    if (B.bound && !fixed_dt && !B.z.dtl) return CB2_ERR_INVALID;
    // a blowing wall reads the step number, which the device-driven loop does not pass on
    if (B.bound)
      for (const FaceBC &f : B.faces)
        if (f.blow) return CB2_ERR_UNSUPPORTED;
  }
  if (!any) return CB2_ERR_INVALID;
  fixed_dt = fixed_dt ? 1 : 0;
  if (!ctx->sg.exec || ctx->sg.gen != ctx->bind_gen || ctx->sg.fixed_dt != fixed_dt)
    CB2_TRY(capture_step_graph(ctx, fixed_dt));
  cudaStream_t s = (cudaStream_t)stream;
  RunState h{*time_inout, t_end, fixed_dt ? dt : 0.0, 0, max_steps};
  CB2_TRY(check_cuda(cudaMemcpyAsync(ctx->d_run, &h, sizeof(h), cudaMemcpyHostToDevice, s)));
  CB2_TRY(check_cuda(cudaGraphLaunch(ctx->sg.exec, s)));
  unsigned status = 0;
  CB2_TRY(check_cuda(cudaMemcpyAsync(&h, ctx->d_run, sizeof(h), cudaMemcpyDeviceToHost, s)));
  CB2_TRY(check_cuda(cudaMemcpyAsync(&status, ctx->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, s)));
  CB2_TRY(check_cuda(cudaStreamSynchronize(s)));
  ctx->n_launch += (unsigned long long)h.step * ctx->sg.launches;
  *time_inout = h.time;
  *steps_out = h.step;
  if (dt_last_out) *dt_last_out = h.dt;
  ctx->p.dt = h.dt;
  if (status != 0u || !(h.dt > 0.0 && h.dt < 1e300)) return CB2_ERR_NONPHYSICAL;
  return CB2_OK;
}

int cb2_reactor_setup(cb2_ctx *ctx, cb2_reactor *reactors, int n, const double *T0, const double *p0,
                      const double *Y, const double *t_end, double h0, void *stream) {
  if (!ctx || !reactors || n < 0 || !T0 || !p0 || !Y || !t_end || !(h0 > 0)) return CB2_ERR_INVALID;
  if (two_temperature(ctx)) return CB2_ERR_UNSUPPORTED;
  if (ctx->p.n_spec == 0) return CB2_ERR_UNSUPPORTED;
  if (n == 0) return CB2_OK;
  ProfGuard pg(ctx);
  ++ctx->n_launch;
  return launch_reactor_setup(ctx->p, reactors, n, T0, p0, Y, t_end, h0, (cudaStream_t)stream);
}

int cb2_reactor_advance(cb2_ctx *ctx, cb2_reactor *reactors, int n, int max_attempts, double rtol, double atol,
                        void *stream) {
  if (!ctx || !reactors || n < 0 || max_attempts < 1 || !(rtol > 0) || !(atol > 0)) return CB2_ERR_INVALID;
  if (two_temperature(ctx)) return CB2_ERR_UNSUPPORTED;
  if (ctx->p.n_spec == 0) return CB2_ERR_UNSUPPORTED;
  if (n == 0) return CB2_OK;
  ProfGuard pg(ctx);
  ++ctx->n_launch;
  return launch_reactor_advance(ctx->p, reactors, n, max_attempts, rtol, atol, (cudaStream_t)stream);
}

int cb2_reactor_advance_krylov(cb2_ctx *ctx, cb2_reactor *reactors, int n, int max_attempts, double rtol,
                               double atol, void *stream) {
  if (!ctx || !reactors || n < 0 || max_attempts < 1 || !(rtol > 0) || !(atol > 0)) return CB2_ERR_INVALID;
  if (two_temperature(ctx)) return CB2_ERR_UNSUPPORTED;
  if (ctx->p.n_spec == 0) return CB2_ERR_UNSUPPORTED;
  if (n == 0) return CB2_OK;
  ProfGuard pg(ctx);
  ++ctx->n_launch;
  return launch_reactor_advance(ctx->p, reactors, n, max_attempts, rtol, atol, (cudaStream_t)stream, true);
}

int cb2_reactor_advance_fixed(cb2_ctx *ctx, cb2_reactor *reactors, int n, int max_steps, int scheme, void *stream) {
  if (!ctx || !reactors || n < 0 || max_steps < 1) return CB2_ERR_INVALID;
  if (two_temperature(ctx)) return CB2_ERR_UNSUPPORTED;
  if (ctx->p.n_spec == 0) return CB2_ERR_UNSUPPORTED;
  if (n == 0) return CB2_OK;
  ProfGuard pg(ctx);
  ++ctx->n_launch;
  return launch_reactor_fixed(ctx->p, reactors, n, max_steps, scheme, (cudaStream_t)stream);
}

}  // extern "C"

// Host records of a batch, largest block first (the persistent grid's work order), in
// ctx->d_batch; order[pos] is the caller's index of record pos.
static int build_block_batch(cb2_ctx *ctx, const cb2_block_case *cases, int n, std::vector<BlockCase> &h,
                             std::vector<int> &order) {
  const Param &p = ctx->p;
  const int need_g = p.reconstruction == CB2_REC_WENO7 ? 4 : 3;
  order.resize(n);
  for (int i = 0; i < n; ++i) {
    const cb2_zone_view &v = cases[i].zone;
    if (v.mx < 1 || v.my < 1 || v.mz < 1 || v.ngg < need_g) return CB2_ERR_INVALID;
    if (!v.cv || !v.bv || !v.qn || !v.dq || !v.metric || !v.jac || !v.mul) return CB2_ERR_INVALID;
    if (!(cases[i].dt >= 0.0)) return CB2_ERR_INVALID;
    if ((long long)(v.mx + 2 * v.ngg) * (v.my + 2 * v.ngg) >= (1LL << 31)) return CB2_ERR_UNSUPPORTED;
    const int ms[3] = {v.mx, v.my, v.mz};
    for (int d = 0; d < (v.mz > 1 ? 3 : 2); ++d)
      if (ms[d] < v.ngg + 2) return CB2_ERR_UNSUPPORTED;  // the periodic pair needs m >= g + 2
    order[i] = i;
  }
  auto work = [&](int i) { return (long long)cases[i].zone.mx * cases[i].zone.my * cases[i].zone.mz; };
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work(a) > work(b); });
  if (n > ctx->n_batch) {
    cudaFree(ctx->d_batch);
    ctx->d_batch = nullptr;
    ctx->n_batch = 0;
    CB2_TRY(check_cuda(cudaMalloc(&ctx->d_batch, sizeof(BlockCase) * n)));
    ctx->n_batch = n;
  }
  if (!ctx->d_queue) CB2_TRY(check_cuda(cudaMalloc(&ctx->d_queue, sizeof(int))));
  h.assign(n, BlockCase{});
  for (int pos = 0; pos < n; ++pos) {
    const cb2_block_case &c = cases[order[pos]];
    BlockCase &b = h[pos];
    b.z = make_zone(c.zone);
    b.p = p;
    b.p.dim = c.zone.mz == 1 ? 2 : 3;
    b.p.status = &ctx->d_batch[pos].flags;
    const int mx = c.zone.mx, my = c.zone.my, mz = c.zone.mz;
    b.n_pairs = 0;
    for (int d = 0; d < (mz > 1 ? 3 : 2); ++d) {
      // the low periodic face of direction d over the whole block (the register_face ranges)
      FaceBC f{};
      f.type = CB2_BC_PERIODIC;
      f.face = d;
      f.direction = -1;
      f.end[0] = d == 0 ? 0 : mx - 1;
      f.end[1] = d == 1 ? 0 : my - 1;
      f.end[2] = d == 2 ? 0 : mz - 1;
      b.pairs[b.n_pairs++] = f;
    }
    b.time = c.time;
    b.t_end = c.t_end;
    b.dt_fixed = c.dt;
    b.last_dt = 0.0;
    b.steps = 0;
    b.status = 0;
    b.flags = 0u;
  }
  return CB2_OK;
}

extern "C" {

int cb2_block_batch_advance(cb2_ctx *ctx, cb2_block_case *cases, int n, int max_steps, void *stream) {
  if (!ctx || (n > 0 && !cases) || n < 0 || max_steps < 0) return CB2_ERR_INVALID;
  if (!block_batch_supported(ctx->p)) return CB2_ERR_UNSUPPORTED;
  if (n == 0) return CB2_OK;
  std::vector<BlockCase> h;
  std::vector<int> order;
  CB2_TRY(build_block_batch(ctx, cases, n, h, order));
  ProfGuard pg(ctx);
  cudaStream_t s = (cudaStream_t)stream;
  CB2_TRY(check_cuda(cudaMemcpyAsync(ctx->d_batch, h.data(), sizeof(BlockCase) * n, cudaMemcpyHostToDevice, s)));
  CB2_TRY(launch_block_batch(ctx->d_batch, n, ctx->p, max_steps, 0, ctx->batch_ni, ctx->batch_cs, ctx->d_queue, s));
  ++ctx->n_launch;
  CB2_TRY(check_cuda(cudaMemcpyAsync(h.data(), ctx->d_batch, sizeof(BlockCase) * n, cudaMemcpyDeviceToHost, s)));
  CB2_TRY(check_cuda(cudaStreamSynchronize(s)));
  for (int pos = 0; pos < n; ++pos) {
    cb2_block_case &c = cases[order[pos]];
    c.time = h[pos].time;
    c.last_dt = h[pos].last_dt;
    c.steps = h[pos].steps;
    c.status = h[pos].status;
  }
  return CB2_OK;
}

int cb2_block_batch_autotune(cb2_ctx *ctx, cb2_block_case *cases, int n, int *tile_ni_out, void *stream) {
  if (!ctx || (n > 0 && !cases) || n < 0) return CB2_ERR_INVALID;
  if (!block_batch_supported(ctx->p)) return CB2_ERR_UNSUPPORTED;
  if (n > 0) {
    std::vector<BlockCase> h;
    std::vector<int> order;
    CB2_TRY(build_block_batch(ctx, cases, n, h, order));
    cudaStream_t s = (cudaStream_t)stream;
    CB2_TRY(check_cuda(cudaMemcpyAsync(ctx->d_batch, h.data(), sizeof(BlockCase) * n, cudaMemcpyHostToDevice, s)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = check_cuda(cudaEventCreate(&e0));
    if (rc == CB2_OK) rc = check_cuda(cudaEventCreate(&e1));
    float best_ms = 1e30f;
    int best = kNI, best_cs = 8;
    const int cluster[4] = {1, 2, 4, 8};
    for (int c = 0; c < 3 && rc == CB2_OK; ++c)
      for (int q = 0; q < 4 && rc == CB2_OK; ++q) {
        const int ni = kTileNI[c], cs = cluster[q];
        rc = launch_block_batch(ctx->d_batch, n, ctx->p, 0, 1, ni, cs, ctx->d_queue, s);  // warm-up
        if (rc == CB2_OK) rc = check_cuda(cudaEventRecord(e0, s));
        for (int r = 0; r < 2 && rc == CB2_OK; ++r)
          rc = launch_block_batch(ctx->d_batch, n, ctx->p, 0, 1, ni, cs, ctx->d_queue, s);
        if (rc == CB2_OK) rc = check_cuda(cudaEventRecord(e1, s));
        if (rc == CB2_OK) rc = check_cuda(cudaEventSynchronize(e1));
        float ms = 0;
        if (rc == CB2_OK) rc = check_cuda(cudaEventElapsedTime(&ms, e0, e1));
        if (rc == CB2_OK && ms < best_ms) {
          best_ms = ms;
          best = ni;
          best_cs = cs;
        }
      }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (rc != CB2_OK) return rc;
    ctx->batch_ni = best;
    ctx->batch_cs = best_cs;
  }
  if (tile_ni_out) {
    tile_ni_out[0] = ctx->batch_ni;
    tile_ni_out[1] = ctx->batch_cs;
  }
  return CB2_OK;
}

int cb2_block_batch_set_schedule(cb2_ctx *ctx, int tile_ni, int cluster_ctas) {
  if (!ctx || !(tile_ni == 4 || tile_ni == 8 || tile_ni == 16)) return CB2_ERR_INVALID;
  if (!(cluster_ctas == 1 || cluster_ctas == 2 || cluster_ctas == 4 || cluster_ctas == 8)) return CB2_ERR_INVALID;
  ctx->batch_ni = tile_ni;
  ctx->batch_cs = cluster_ctas;
  return CB2_OK;
}

int cb2_read_status(cb2_ctx *ctx, unsigned *flags_out, void *stream) {
  if (!ctx || !flags_out) return CB2_ERR_INVALID;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned f = 0;
  CB2_TRY(check_cuda(cudaMemcpyAsync(&f, ctx->d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, s)));
  CB2_TRY(check_cuda(cudaMemsetAsync(ctx->d_status, 0, sizeof(unsigned), s)));
  CB2_TRY(check_cuda(cudaStreamSynchronize(s)));
  *flags_out = f;
  return CB2_OK;
}

}  // extern "C"
