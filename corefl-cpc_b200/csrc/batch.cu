// Batched 1-D cases: one CTA advances one case by whole SSP-RK3 steps, many cases of uneven
// size per launch.
//
// A case is a single i-line of mx nodes stored in the compact 1-D layout (g ghost nodes at each
// end, no ghost rows or planes).  One step runs the same per-node operations, in the same order,
// as cb2_rk3_step on a one-row block (src/RK.cuh:107-272):
//   qn <- cv; CFL dt = min over nodes of local_time_step (seed 1e6, no clamp to t_end: the
//   reference stops once the physical time reaches the end time); then three times:
//   dq <- 0, chemistry source, x sweep (tiles of the primitive-variable sweep), stage update,
//   outflow ghost fill of both ends, properties of every node.
// Against the block path on the same one-row case this omits only work whose result is exactly
// zero or unused: the y sweep of a row whose ghost rows copy it (every y-face flux is the same
// bitwise, so their difference is 0), the ghost rows themselves, and the transport properties of
// an inviscid case.  A case's results do not depend on which other cases share the launch.
#include "chem.cuh"
#include "point.cuh"
#include "inviscid_pv.cuh"
#include "batch.h"

namespace cb2 {

__device__ __forceinline__ double block_min_d(double v, double *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double m = 1e+6;
  for (int w = 0; w < kSweepThreads / 32; ++w) m = fmin(m, red[w]);
  return m;
}

template <int NS>
__device__ __forceinline__ void outflow_end(const Zone &z, const Param &p, int face_i, int dir, int gl) {
  const idx_t sz = z.L.sz;
  const idx_t gb = z.L.at(face_i, 0, 0), gg = z.L.at(face_i + gl * dir, 0, 0);
  for (int l = 0; l < 6; ++l) z.bv[gg + l * sz] = z.bv[gb + l * sz];
  for (int l = 0; l < p.n_scalar; ++l) z.sv[gg + l * sz] = z.sv[gb + l * sz];
  cv_point<NS>(z, p, gg);
}

template <int NS, int REC, int SOLVER>
__global__ void __launch_bounds__(kSweepThreads) k_line_batch(LineCase *cases, int n_cases, int max_steps) {
  extern __shared__ __align__(16) unsigned char line_smem[];
  __shared__ double red[kSweepThreads / 32];
  if ((int)blockIdx.x >= n_cases) return;
  LineCase &lc = cases[blockIdx.x];
  if (!lc.active || lc.status) return;
  const Zone &z = lc.z;
  const Param &p = lc.p;
  const int tid = threadIdx.x, nt = kSweepThreads;
  const int N = z.mx, g = z.ngg;
  constexpr int NV = 5 + NS;
  const idx_t sz = z.L.sz, sz0 = z.L0.sz;
  const idx_t run = (idx_t)z.L.my * z.L.disp2;
  const int ntile = (int)((run + (kSweepThreads - 2) - 1) / (kSweepThreads - 2));
  double time = lc.time;
  int step = lc.step;
  bool failed = false;
  for (int s = 0; s < max_steps && time < lc.t_end; ++s) {
    for (int i = tid; i < N; i += nt) {
      const idx_t gi = z.L.at(i, 0, 0);
      for (int l = 0; l < NV; ++l) z.qn[gi + l * sz] = z.cv[gi + l * sz];
    }
    double m = 1e+6;
    bool bad = false;
    for (int i = tid; i < N; i += nt) {
      const double d = local_dt_point<NS>(z, p, i, 0, 0);
      bad |= !(d > 0) || !isfinite(d);  // fmin would drop a NaN
      m = fmin(m, d);
    }
    const double dt = block_min_d(m, red);
    if (__syncthreads_or(bad)) {
      failed = true;
      break;
    }
    for (int rk = 0; rk < 3; ++rk) {
      for (int i = tid; i < N; i += nt)
        for (int l = 0; l < NV; ++l) z.dq[z.L0.at(i, 0, 0) + l * sz0] = 0.0;
      __syncthreads();
      if constexpr (NS > 0) {
        if (p.reaction) {
          for (int i = tid; i < N; i += nt) chemistry_point<NS>(z, p, i, 0, 0);
          __syncthreads();
        }
      }
      for (int t = 0; t < ntile; ++t) pv_tile<double, NS, 0, REC, SOLVER>(z, p, run, t, 0, 0, line_smem);
      for (int i = tid; i < N; i += nt) stage_update_point<NS>(z, p, dt, rk, i, 0, 0);
      __syncthreads();
      if (tid < g) outflow_end<NS>(z, p, 0, -1, tid + 1);
      else if (tid < 2 * g) outflow_end<NS>(z, p, N - 1, 1, tid - g + 1);
      __syncthreads();
      for (int i = tid - g; i < N + g; i += nt) properties_point<NS>(z, p, i, 0, 0, p.viscous_order > 0);
      __syncthreads();
    }
    time += dt;
    ++step;
    if (tid == 0) lc.last_dt = dt;
  }
  __syncthreads();
  if (tid == 0) {
    lc.time = time;
    lc.step = step;
    if (time >= lc.t_end) lc.status |= kLineDone;
    if (failed || (lc.flags & 3u)) lc.status |= kLineFailed;
  }
}

// Initial state of a two-state shock tube on the compact line: nodes at x = i dx, left state
// for x <= x_split, right state beyond; composition Y everywhere; metric d(xi)/dx = 1/dx,
// d(eta)/dy = d(zeta)/dz = 1, J = dx.  Covers the ghosts too.
template <int NS>
__global__ void k_line_setup(LineCase *cases, int slot, double TL, double pL, double TR, double pR, const double *Y,
                             double dx, double x_split) {
  const LineCase &lc = cases[slot];
  const Zone &z = lc.z;
  const Param &p = lc.p;
  const int i = blockIdx.x * blockDim.x + threadIdx.x - z.ngg;
  if (i >= z.mx + z.ngg) return;
  const idx_t g = z.L.at(i, 0, 0), sz = z.L.sz;
  const double x = i * dx;
  const bool left = x <= x_split;
  const double t = left ? TL : TR, pr = left ? pL : pR;
  double r = 0;
  for (int s = 0; s < NS; ++s) r += Y[s] * __ldg(p.mech.gas_const + s);
  const double rho = pr / (r * t);
  z.bv[g] = rho;
  z.bv[g + sz] = 0;
  z.bv[g + 2 * sz] = 0;
  z.bv[g + 3 * sz] = 0;
  z.bv[g + 4 * sz] = pr;
  z.bv[g + 5 * sz] = t;
  for (int s = 0; s < NS; ++s) z.sv[g + s * sz] = Y[s];
  for (int c = 0; c < 9; ++c) z.metric[g + c * sz] = 0;
  z.metric[g] = 1.0 / dx;
  z.metric[g + 4 * sz] = 1.0;
  z.metric[g + 8 * sz] = 1.0;
  z.jac[g] = dx;
  cv_point<NS>(z, p, g);
  properties_point<NS>(z, p, i, 0, 0, p.viscous_order > 0);
  if (z.rts) z.rts[g] = 1e+6;
}

// ---- launchers ------------------------------------------------------------------------------
template <int NS, int REC, int SOLVER>
static int line_batch_launch(LineCase *cases, int n, int max_steps, cudaStream_t s) {
  const size_t smem = pv_tile_smem<double, NS, REC, SOLVER>(0);
  auto kern = k_line_batch<NS, REC, SOLVER>;
  CB2_TRY(prepare_smem(kern, smem));
  kern<<<n, kSweepThreads, smem, s>>>(cases, n, max_steps);
  return check_launch();
}

int launch_line_batch(LineCase *cases, int n, const Param &p, int max_steps, cudaStream_t s) {
  if (n <= 0) return CB2_OK;
  ProfScope prof("line_batch", s);
  // the served cases: H2/air (9 species) with WENO5 and HLLC or AUSM+
  if (p.n_spec != 9 || p.reconstruction != CB2_REC_WENO5) return CB2_ERR_UNSUPPORTED;
  if (p.inviscid_scheme == CB2_INV_HLLC) return line_batch_launch<9, 5, CB2_INV_HLLC>(cases, n, max_steps, s);
  if (p.inviscid_scheme == CB2_INV_AUSMP) return line_batch_launch<9, 5, CB2_INV_AUSMP>(cases, n, max_steps, s);
  return CB2_ERR_UNSUPPORTED;
}

bool line_batch_supported(const Param &p) {
  return p.viscous_order == 0 && p.precision == CB2_PREC_FP64 && p.n_spec == 9 && p.i_eve < 0 &&
         p.reconstruction == CB2_REC_WENO5 && (p.inviscid_scheme == CB2_INV_HLLC || p.inviscid_scheme == CB2_INV_AUSMP);
}

int launch_line_setup(LineCase *cases, int slot, int mx, int g, const Param &p, double TL, double pL, double TR,
                      double pR, const double *Y, double dx, double x_split, cudaStream_t s) {
  const int n = mx + 2 * g;
  const unsigned blocks = (unsigned)((n + 127) / 128);
  if (p.n_spec != 9) return CB2_ERR_UNSUPPORTED;
  k_line_setup<9><<<blocks, 128, 0, s>>>(cases, slot, TL, pL, TR, pR, Y, dx, x_split);
  return check_launch();
}

}  // namespace cb2
