// Reference-kernel runner: drives the reference's OWN CUDA kernels, built from its sources for
// sm_100a, through the RK3 stage sequence of src/RK.cuh:107-237 on a synthetic case, and dumps
// the device arrays it produces.  TEST INFRASTRUCTURE ONLY: built into oracle/_ref/ by
// oracle/ref_gpu_build.py and run on a GPU by tests/golden/make_ref_kernels.py, whose dumps become
// the committed fixtures tests/golden/ref_kernels_*.npz.  The library never links or calls it.
//
// What is the reference's and what is this file's:
//   reference (linked from its sources, unmodified): cfd::Parameter (reads input/setup.txt),
//     cfd::Mesh (reads the ASCII grid, boundary and inner-face files, registers the faces and
//     computes metrics), cfd::Species / cfd::Reaction, cfd::Field::setup_device_memory (the DZone),
//     cfd::SinglePointStat (sizes the Field's statistics arrays), cfd::DBoundCond (every boundary
//     condition), cfd::DParameter, and every kernel of the stage:
//     compute_cv_from_bv, update_physical_properties, compute_viscous_flux, finite_rate_chemistry,
//     compute_inviscid_flux, update_cv_and_bv_rk, apply_vt_relaxation_rk, limit_flow,
//     apply_boundary_conditions, data_communication, eliminate_k_gradient, local_time_step,
//     global_time_step, compute_shock_sensor.
//   this file: the call sequence (the body of RK3<mix>, src/RK.cuh:107-237, without I/O,
//     residual monitoring, sponge layers and fluctuations), loading the case's initial primitive
//     state (and, when given, its metric and Jacobian) into the DZone arrays, the optional
//     constant viscosity of air (the reference has only Sutherland, src/FieldOperation.cuh:244;
//     the runner overwrites mul after every property update, the way a constant-mu case feeds the
//     kernels), and the dumps.
//
// Usage: ref_stage_runner <case-dir>
//   <case-dir>/input/setup.txt, input/grid/grid   0.grd, input/boundary_condition/{boundary,inner}   0.txt
//   <case-dir>/task.txt   : "key value" lines: mode (stages|steps|time), stages, n_steps, warmup, dt,
//                           fixed_dt, t_end, mul_constant, load_metric (0/1), init (file|reference),
//                           write_plt (0/1: the reference's output/flowfield.plt of the final state)
//   <case-dir>/state.bin  : per block, float64 padded arrays (ghost ngg): bv[6], sv[n_scalar],
//                           T_ve (two-temperature build), then metric[9] and jac when load_metric = 1
//   writes <case-dir>/out.bin : the layout is written out above the dump in run().
#include <unistd.h>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

#include "Parameter.h"
#include "Mesh.h"
#include "Field.h"
#include "ChemData.h"
#include "DParameter.cuh"
#include "BoundCond.h"
#include "BoundCond.cuh"
#include "InviscidScheme.cuh"
#include "ViscousScheme.cuh"
#include "FiniteRateChem.cuh"
#include "FieldOperation.cuh"
#include "DataCommunication.cuh"
#include "TimeAdvanceFunc.cuh"
#include "Initialize.cuh"
#include "SinglePointStat.cuh"
#include "RK.cuh"
#include "FieldIO.h"

namespace {

bool g_checks = true;  // off while a timed run measures the step sequence alone

void check(const char *where) {
  if (!g_checks) return;
  cudaError_t e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "ref_stage_runner: CUDA error after %s: %s\n", where, cudaGetErrorString(e));
    std::exit(3);
  }
}

std::map<std::string, std::string> read_task(const char *path) {
  std::map<std::string, std::string> t;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream s(line);
    std::string k, v;
    if (s >> k >> v) t[k] = v;
  }
  return t;
}

double tget(const std::map<std::string, std::string> &t, const char *k, double d) {
  auto it = t.find(k);
  return it == t.end() ? d : std::stod(it->second);
}

__global__ void fill_mul(cfd::DZone *zone, real mu) {
  const int ngg = zone->ngg;
  const int i = static_cast<int>(blockDim.x * blockIdx.x + threadIdx.x) - ngg;
  const int j = static_cast<int>(blockDim.y * blockIdx.y + threadIdx.y) - ngg;
  const int k = static_cast<int>(blockDim.z * blockIdx.z + threadIdx.z) - ngg;
  if (i >= zone->mx + ngg || j >= zone->my + ngg || k >= zone->mz + ngg) return;
  zone->mul(i, j, k) = mu;
}

struct Runner {
  cfd::Parameter &parameter;
  cfd::Mesh &mesh;
  std::vector<cfd::Field> &field;
  cfd::DBoundCond &bc;
  cfd::DParameter *param;
  double mul_constant;
  dim3 tpb;
  std::vector<dim3> bpg, bpg_all;
  std::vector<double> dt_hist;

  Runner(cfd::Parameter &p, cfd::Mesh &m, std::vector<cfd::Field> &f, cfd::DBoundCond &b, cfd::DParameter *dp,
         double mu)
      : parameter(p), mesh(m), field(f), bc(b), param(dp), mul_constant(mu) {
    // the launch shapes of RK3<mix> (src/RK.cuh:35-47, 53-56, 231-235)
    tpb = mesh.dimension == 2 ? dim3{16, 16, 1} : dim3{8, 8, 4};
    const int ng_1 = 2 * mesh[0].ngg - 1;
    for (int b = 0; b < mesh.n_block; ++b) {
      const int mx = mesh[b].mx, my = mesh[b].my, mz = mesh[b].mz;
      bpg.push_back(dim3((mx - 1) / tpb.x + 1, (my - 1) / tpb.y + 1, (mz - 1) / tpb.z + 1));
      bpg_all.push_back(dim3((mx + ng_1) / tpb.x + 1, (my + ng_1) / tpb.y + 1, (mz + ng_1) / tpb.z + 1));
    }
  }

  void override_mul() {
    if (mul_constant <= 0) return;
    for (int b = 0; b < mesh.n_block; ++b) {
      const int ngg = mesh[b].ngg;
      dim3 t{8, 8, 4};
      dim3 g((mesh[b].mx + 2 * ngg - 1) / t.x + 1, (mesh[b].my + 2 * ngg - 1) / t.y + 1,
             (mesh[b].mz + 2 * ngg - 1) / t.z + 1);
      fill_mul<<<g, t>>>(field[b].d_ptr, mul_constant);
    }
  }

  template <MixtureModel mix>
  void properties() {
    for (int b = 0; b < mesh.n_block; ++b)
      cfd::update_physical_properties<mix><<<bpg_all[b], tpb>>>(field[b].d_ptr, param);
    override_mul();
  }

  // Driver<mix>::initialize_computation (src/Driver.cu:126-210) after the primitive state is set.
  template <MixtureModel mix>
  void initialize(int step) {
    const int ng_1 = 2 * mesh[0].ngg - 1;
    if (mesh.dimension == 2) {
      for (int b = 0; b < mesh.n_block; ++b) {
        dim3 BPG{(unsigned)((mesh[b].mx + ng_1) / tpb.x + 1), (unsigned)((mesh[b].my + ng_1) / tpb.y + 1), 1};
        cfd::eliminate_k_gradient<<<BPG, tpb>>>(field[b].d_ptr, param);
      }
    }
    properties<mix>();
    for (int b = 0; b < mesh.n_block; ++b) bc.apply_boundary_conditions<mix>(mesh[b], field[b], param, step);
    cfd::data_communication<mix>(mesh, field, parameter, step, param);
    properties<mix>();
    // RK3 start: cv from bv over interior and ghosts (src/RK.cuh:49-58)
    for (int b = 0; b < mesh.n_block; ++b)
      cfd::compute_cv_from_bv<mix><<<bpg_all[b], tpb>>>(field[b].d_ptr, param);
    check("initialize");
  }

  // One SSP-RK3 step, stages [0, n_stages), as the body of RK3<mix> (src/RK.cuh:107-237).
  // Dumps dq after the residual of each stage into dq_out[stage] when given.
  template <MixtureModel mix>
  double step(int step_no, double dt, bool fixed_dt, int n_stages, std::vector<std::vector<double>> *dq_out) {
    const int n_var = parameter.get_int("n_var");
    for (int b = 0; b < mesh.n_block; ++b)
      cudaMemcpy(field[b].h_ptr->qn.data(), field[b].h_ptr->cv.data(), field[b].h_ptr->cv.size() * sizeof(real) * n_var,
                 cudaMemcpyDeviceToDevice);
    if (parameter.get_string("hybrid_inviscid_scheme") != "NO") {
      for (int b = 0; b < mesh.n_block; ++b) cfd::compute_shock_sensor<<<bpg[b], tpb>>>(field[b].d_ptr, param);
    }
    if (!fixed_dt) {
      for (int b = 0; b < mesh.n_block; ++b) cfd::local_time_step<mix><<<bpg[b], tpb>>>(field[b].d_ptr, param);
      dt = cfd::global_time_step(mesh, parameter, field);
      cfd::update_dt_global<<<1, 1>>>(param, dt);
    }
    check("pre-stage");
    [[maybe_unused]] constexpr real rk_stage_dt_scale[3]{1.0, 0.25, 2.0 / 3.0};
    for (int rk = 0; rk < n_stages; ++rk) {
      for (int b = 0; b < mesh.n_block; ++b)
        cudaMemset(field[b].h_ptr->dq.data(), 0, field[b].h_ptr->dq.size() * n_var * sizeof(real));
      cfd::compute_viscous_flux<mix>(mesh, field, param, parameter);
      for (int b = 0; b < mesh.n_block; ++b) {
        if (parameter.get_int("reaction") == 1) cfd::finite_rate_chemistry<<<bpg[b], tpb>>>(field[b].d_ptr, param);
        cfd::compute_inviscid_flux<mix>(mesh[b], field[b].d_ptr, param, n_var, parameter);
        // the non-reflecting outflows' correction of dq, before the dump (RK.cuh:190-193)
        bc.nonReflectingBoundary<mix>(mesh[b], field[b], param);
      }
      check("residual");
      if (dq_out) {
        for (int b = 0; b < mesh.n_block; ++b) {
          std::vector<double> h(static_cast<size_t>(field[b].h_ptr->dq.size()) * n_var);
          cudaMemcpy(h.data(), field[b].h_ptr->dq.data(), h.size() * sizeof(double), cudaMemcpyDeviceToHost);
          dq_out->push_back(std::move(h));
        }
      }
      for (int b = 0; b < mesh.n_block; ++b) {
        cfd::update_cv_and_bv_rk<mix><<<bpg[b], tpb>>>(field[b].d_ptr, param, dt, rk);
        if constexpr (cfd::kTwoTemperature) {
          cfd::apply_vt_relaxation_rk<<<bpg[b], tpb>>>(field[b].d_ptr, param, rk_stage_dt_scale[rk] * dt);
        }
        if (parameter.get_bool("limit_flow")) cfd::limit_flow<mix><<<bpg[b], tpb>>>(field[b].d_ptr, param);
        bc.apply_boundary_conditions<mix>(mesh[b], field[b], param, step_no);
      }
      cfd::data_communication<mix>(mesh, field, parameter, step_no, param);
      if (mesh.dimension == 2) {
        const int ng_1 = 2 * mesh[0].ngg - 1;
        for (int b = 0; b < mesh.n_block; ++b) {
          dim3 BPG{(unsigned)((mesh[b].mx + ng_1) / tpb.x + 1), (unsigned)((mesh[b].my + ng_1) / tpb.y + 1), 1};
          cfd::eliminate_k_gradient<<<BPG, tpb>>>(field[b].d_ptr, param);
        }
      }
      properties<mix>();
      check("stage");
    }
    return dt;
  }
};

void read_block_arrays(std::FILE *f, cfd::Field &fld, int n_scalar, bool load_metric) {
  auto *z = fld.h_ptr;
  auto load = [&](double *dev, size_t n, const char *what) {
    std::vector<double> h(n);
    if (std::fread(h.data(), sizeof(double), n, f) != n) {
      std::fprintf(stderr, "ref_stage_runner: state.bin too short reading %s\n", what);
      std::exit(4);
    }
    cudaMemcpy(dev, h.data(), n * sizeof(double), cudaMemcpyHostToDevice);
  };
  const size_t np = static_cast<size_t>(z->bv.size());
  load(z->bv.data(), np * 6, "bv");
  if (n_scalar > 0) load(z->sv.data(), np * n_scalar, "sv");
  if constexpr (cfd::kTwoTemperature) {
    if (z->temperature_ve.size() > 0) load(z->temperature_ve.data(), np, "temperature_ve");
  }
  if (load_metric) {
    std::vector<double> ref(np * 10);
    cudaMemcpy(ref.data(), z->metric.data(), np * 9 * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(ref.data() + np * 9, z->jac.data(), np * sizeof(double), cudaMemcpyDeviceToHost);
    std::FILE *m = std::fopen("ref_metric.bin", "ab");
    if (m) {
      std::fwrite(ref.data(), sizeof(double), ref.size(), m);
      std::fclose(m);
    }
    load(z->metric.data(), np * 9, "metric");
    load(z->jac.data(), np, "jac");
  }
}

void dump_array(std::FILE *f, const double *dev, size_t n) {
  std::vector<double> h(n);
  cudaMemcpy(h.data(), dev, n * sizeof(double), cudaMemcpyDeviceToHost);
  std::fwrite(h.data(), sizeof(double), n, f);
}

template <MixtureModel mix>
int run(cfd::Parameter &parameter, cfd::Mesh &mesh, cfd::Species &spec, cfd::Reaction &reac,
        const std::map<std::string, std::string> &task) {
  std::vector<cfd::Field> field;
  // the Driver's statistics collector (IOManager::stat_collector) is built before the fields and
  // sets the sizes of the statistics arrays that Field's constructor reads (src/SinglePointStat.cu:16-110)
  [[maybe_unused]] cfd::SinglePointStat stat_collector(parameter, mesh, field, spec);
  field.reserve(mesh.n_block);
  for (int b = 0; b < mesh.n_block; ++b) field.emplace_back(parameter, mesh[b]);
  for (int b = 0; b < mesh.n_block; ++b) field[b].setup_device_memory(parameter);
  check("setup_device_memory");
  cfd::DBoundCond bc;
  bc.initialize_bc_on_GPU(mesh, field, spec, parameter);
  check("initialize_bc_on_GPU");

  const bool from_reference = task.count("init") && task.at("init") == "reference";
  if (from_reference) {
    cfd::initialize_basic_variables<mix>(parameter, mesh, field, spec);
  } else {
    // the reference state that the WENO eps, limit_flow bounds and v_char read (src/BoundCond.cpp:331-357)
    [[maybe_unused]] cfd::Inflow reference(parameter.get_string("reference_state"), spec, parameter);
  }
  check("reference state");
  const cfd::DParameter d_param(parameter, spec, &reac);
  cfd::DParameter *param = nullptr;
  cudaMalloc(&param, sizeof(cfd::DParameter));
  cudaMemcpy(param, &d_param, sizeof(cfd::DParameter), cudaMemcpyHostToDevice);
  check("DParameter");

  if (!from_reference) {
    std::FILE *f = std::fopen("state.bin", "rb");
    if (!f) {
      std::fprintf(stderr, "ref_stage_runner: no state.bin\n");
      return 4;
    }
    std::remove("ref_metric.bin");
    for (int b = 0; b < mesh.n_block; ++b)
      read_block_arrays(f, field[b], parameter.get_int("n_scalar"), tget(task, "load_metric", 0) != 0);
    std::fclose(f);
  }

  Runner r(parameter, mesh, field, bc, param, tget(task, "mul_constant", 0.0));
  r.initialize<mix>(0);

  const std::string mode = task.count("mode") ? task.at("mode") : "stages";
  const bool fixed_dt = tget(task, "fixed_dt", 1) != 0;
  double dt = tget(task, "dt", 0.0);
  std::vector<std::vector<double>> dq;
  int steps = 0;
  double time = 0;
  if (mode == "stages") {
    dt = r.step<mix>(1, dt, fixed_dt, static_cast<int>(tget(task, "stages", 1)), &dq);
    steps = 1;
  } else if (mode == "time") {
    // warm-up steps, then n_steps steps between two CUDA events with no synchronisation of the
    // runner's own in between (the CFL step's global minimum still copies dt to the host, as RK3
    // does); the mean step time goes to time.txt
    const int n_warm = static_cast<int>(tget(task, "warmup", 3)), n_time = static_cast<int>(tget(task, "n_steps", 10));
    for (int s = 0; s < n_warm; ++s) dt = r.step<mix>(s + 1, dt, fixed_dt, 3, nullptr);
    check("warm-up");
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    g_checks = false;
    cudaEventRecord(e0);
    for (int s = 0; s < n_time; ++s) dt = r.step<mix>(n_warm + s + 1, dt, fixed_dt, 3, nullptr);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    g_checks = true;
    check("timed steps");
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    std::FILE *tf = std::fopen("time.txt", "w");
    if (tf) {
      std::fprintf(tf, "%d %.9g %.17g\n", n_time, ms / n_time, dt);
      std::fclose(tf);
    }
    std::printf("ref_stage_runner: %d timed step(s), %.6f ms per step, dt = %.17g\n", n_time, ms / n_time, dt);
    return 0;
  } else {
    const long long n_steps = static_cast<long long>(tget(task, "n_steps", 1));
    const double t_end = tget(task, "t_end", 1e300);
    while (steps < n_steps) {
      dt = r.step<mix>(steps + 1, dt, fixed_dt, 3, nullptr);
      r.dt_hist.push_back(dt);
      ++steps;
      time += dt;
      if (time >= t_end) break;  // physical_time >= total_simulation_time (src/RK.cuh:257)
    }
  }

  // out.bin: int32 n_block, steps, n_var, n_scalar, two_t, n_dq; float64 time, dt (last);
  //          float64 rho_inf, v_inf, p_inf, speed_of_sound (the reference state the kernels read);
  //          int32 n_dt + float64 dt history;
  //          per block: int32 mx, my, mz, ngg; float64 cv[n_var], bv[6], sv[n_scalar], (T_ve), padded
  //          (ghost ngg); then the n_dq dq dumps (each n_var x unpadded block, in block order per stage).
  std::FILE *o = std::fopen("out.bin", "wb");
  const int n_var = parameter.get_int("n_var"), n_scalar = parameter.get_int("n_scalar");
  const int two_t = cfd::kTwoTemperature ? 1 : 0;
  const int n_dq = static_cast<int>(dq.size());
  int hdr[6]{mesh.n_block, steps, n_var, n_scalar, two_t, n_dq};
  std::fwrite(hdr, sizeof(int), 6, o);
  double td[2]{time, dt};
  std::fwrite(td, sizeof(double), 2, o);
  double refs[4]{parameter.get_real("rho_inf"), parameter.get_real("v_inf"), parameter.get_real("p_inf"),
                 parameter.get_real("speed_of_sound")};
  std::fwrite(refs, sizeof(double), 4, o);
  const int n_dt = static_cast<int>(r.dt_hist.size());
  std::fwrite(&n_dt, sizeof(int), 1, o);
  std::fwrite(r.dt_hist.data(), sizeof(double), r.dt_hist.size(), o);
  for (int b = 0; b < mesh.n_block; ++b) {
    auto *z = field[b].h_ptr;
    int dims[4]{mesh[b].mx, mesh[b].my, mesh[b].mz, mesh[b].ngg};
    std::fwrite(dims, sizeof(int), 4, o);
    const size_t np = static_cast<size_t>(z->cv.size());
    dump_array(o, z->cv.data(), np * n_var);
    dump_array(o, z->bv.data(), np * 6);
    if (n_scalar > 0) dump_array(o, z->sv.data(), np * n_scalar);
    if constexpr (cfd::kTwoTemperature) {
      if (z->temperature_ve.size() > 0) dump_array(o, z->temperature_ve.data(), np);
    }
  }
  for (auto &d : dq) std::fwrite(d.data(), sizeof(double), d.size(), o);
  std::fclose(o);
  check("dump");
  if (tget(task, "write_plt", 0) != 0) {
    // the reference's own flowfield file of the final state (output/flowfield.plt, no ghost layers
    // as its drivers write it): FieldIO::initialize after copying the fields to the host
    for (int b = 0; b < mesh.n_block; ++b) field[b].copy_data_from_device(parameter);
    parameter.update_parameter("solution_time", time);
    cfd::FieldIO<mix> io(0, mesh, field, parameter, spec, 0);
    io.initialize();
    check("flowfield");
  }
  std::printf("ref_stage_runner: %d step(s), t = %.17g, dt = %.17g\n", steps, time, dt);
  return 0;
}

}  // namespace

int main(int argc, char **argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: ref_stage_runner <case-dir>\n");
    return 2;
  }
  std::setvbuf(stdout, nullptr, _IONBF, 0);
  if (chdir(argv[1]) != 0) {
    std::fprintf(stderr, "ref_stage_runner: cannot enter %s\n", argv[1]);
    return 2;
  }
  const auto task = read_task("task.txt");
  cfd::Parameter parameter(&argc, &argv);
  cfd::Mesh mesh(parameter);
  if (!parameter.get_bool("turbulence")) parameter.update_parameter("turbulence_method", 0);
  cfd::Species spec(parameter);
  cfd::Reaction reac(parameter, spec);
  parameter.deduce_sim_info(spec);
  if (parameter.get_int("species") == 1) return run<MixtureModel::Mixture>(parameter, mesh, spec, reac, task);
  return run<MixtureModel::Air>(parameter, mesh, spec, reac, task);
}
