// Physical properties over interior and ghost nodes (update_physical_properties<mix>,
// src/FieldOperation.cuh:183-247), the local CFL time step (local_time_step<mix>,
// src/TimeAdvanceFunc.cuh:28-127) and its global minimum (min_of_arr + global_time_step,
// src/TimeAdvanceFunc.cu:114-164).
#include <algorithm>
#include "point.cuh"
#include "launch.h"

namespace cb2 {

constexpr int kPropThreads = 128;

// Bounded to 80 registers (6 CTAs of 128 threads per SM; the FP64 9-species transport otherwise
// takes 163): the exponential and logarithm chains are latency-bound (192^3 H2/air box: 29.9 -> 20.7
// ms per step).
template <int NS, bool F32T = false>
__global__ void __launch_bounds__(kPropThreads, 6) k_properties(Zone z, Param p) {
  const int g_ = z.ngg;
  const int i = blockIdx.x * kPropThreads + threadIdx.x - g_;
  const int j = blockIdx.y - g_, k = blockIdx.z - g_;
  if (i >= z.mx + g_) return;
  properties_point<NS, F32T>(z, p, i, j, k);
}

// A 2-D block (mz = 1) carries ngg ghost planes on each side of its one k plane.  The reference
// evaluates the properties on every one of them (src/RK.cuh:230-235); after eliminate_k_gradient
// their basic and scalar variables are copies of plane 0, so their properties are copies of
// plane 0's, which is how they are filled here: the transport evaluation runs once per (i, j)
// instead of 2 ngg + 1 times.  Only kappa_ve, which also depends on the plane's own T_ve (not
// copied by eliminate_k_gradient), is re-evaluated where that differs.
template <int NS, bool F32T = false>
__global__ void __launch_bounds__(kPropThreads) k_properties_planar(Zone z, Param p) {
  const int g_ = z.ngg;
  const int i = blockIdx.x * kPropThreads + threadIdx.x - g_;
  const int j = blockIdx.y - g_;
  if (i >= z.mx + g_) return;
  properties_point<NS, F32T>(z, p, i, j, 0);
  const idx_t sz = z.L.sz, g0 = z.L.at(i, j, 0);
  for (int kk = -g_; kk <= g_; ++kk) {
    if (kk == 0) continue;
    const idx_t gk = z.L.at(i, j, kk);
    z.mul[gk] = z.mul[g0];
    if (z.mach) z.mach[gk] = z.mach[g0];
    if constexpr (NS > 0) {
      z.gamma[gk] = z.gamma[g0];
      z.acoustic[gk] = z.acoustic[g0];
      z.kappa[gk] = z.kappa[g0];
#pragma unroll
      for (int s = 0; s < NS; ++s) z.rhoD[gk + s * sz] = z.rhoD[g0 + s * sz];
      if (p.i_eve >= 0) {
        if (z.tve[gk] <= 0) z.tve[gk] = z.bv[gk + 5 * sz];
        if (z.kappa_ve) {
          const double tk = z.tve[gk];
          if (tk == z.tve[g0]) {
            z.kappa_ve[gk] = z.kappa_ve[g0];
          } else {
            double y[NS], cp[NS], cv_ve, cpt = 0;
#pragma unroll
            for (int s = 0; s < NS; ++s) y[s] = z.sv[gk + s * sz];
            species_cp<NS>(z.bv[gk + 5 * sz], p.mech, cp);
#pragma unroll
            for (int s = 0; s < NS; ++s) cpt = fma(y[s], cp[s], cpt);
            mixture_ve_energy<NS>(tk, y, p.mech, &cv_ve);
            z.kappa_ve[gk] = z.kappa[g0] * cv_ve / fmax(cpt, 1e-8);
          }
        }
      }
    }
  }
}

int launch_properties(const Zone &z, const Param &p, cudaStream_t s, int &n_launch) {
  const int g = z.ngg;
  const bool planar = z.mz == 1 && p.dim == 2;
  const bool mixed = p.precision == CB2_PREC_MIXED;  // transport in FP32
  dim3 grid((z.mx + 2 * g + kPropThreads - 1) / kPropThreads, z.my + 2 * g, planar ? 1 : z.mz + 2 * g);
  ++n_launch;
  ProfScope prof("properties", s);
  switch (p.n_spec) {
    case 0:
      if (p.mu_constant > 0 && !z.mach) { --n_launch; return CB2_OK; }  // nothing changes
      if (planar) k_properties_planar<0><<<grid, kPropThreads, 0, s>>>(z, p);
      else k_properties<0><<<grid, kPropThreads, 0, s>>>(z, p);
      break;
    case 5:
      if (mixed) {
        if (planar) k_properties_planar<5, true><<<grid, kPropThreads, 0, s>>>(z, p);
        else k_properties<5, true><<<grid, kPropThreads, 0, s>>>(z, p);
      } else if (planar) {
        k_properties_planar<5><<<grid, kPropThreads, 0, s>>>(z, p);
      } else {
        k_properties<5><<<grid, kPropThreads, 0, s>>>(z, p);
      }
      break;
    case 9:
      if (mixed) {
        if (planar) k_properties_planar<9, true><<<grid, kPropThreads, 0, s>>>(z, p);
        else k_properties<9, true><<<grid, kPropThreads, 0, s>>>(z, p);
      } else if (planar) {
        k_properties_planar<9><<<grid, kPropThreads, 0, s>>>(z, p);
      } else {
        k_properties<9><<<grid, kPropThreads, 0, s>>>(z, p);
      }
      break;
    default: return CB2_ERR_UNSUPPORTED;
  }
  return check_launch();
}

// ---- local time step --------------------------------------------------------------------
template <int NS>
__global__ void __launch_bounds__(kPropThreads) k_local_dt(Zone z, Param p) {
  const int i = blockIdx.x * kPropThreads + threadIdx.x;
  const int j = blockIdx.y, k = blockIdx.z;
  if (i >= z.mx) return;
  z.dtl[z.L0.at(i, j, k)] = local_dt_point<NS>(z, p, i, j, k);
}

int launch_local_dt(const Zone &z, const Param &p, cudaStream_t s, int &n_launch) {
  dim3 grid((z.mx + kPropThreads - 1) / kPropThreads, z.my, z.mz);
  ++n_launch;
  ProfScope prof("local_dt", s);
  switch (p.n_spec) {
    case 0: k_local_dt<0><<<grid, kPropThreads, 0, s>>>(z, p); break;
    case 5: k_local_dt<5><<<grid, kPropThreads, 0, s>>>(z, p); break;
    case 9: k_local_dt<9><<<grid, kPropThreads, 0, s>>>(z, p); break;
    default: return CB2_ERR_UNSUPPORTED;
  }
  return check_launch();
}

// ---- min reduction: grid-stride partial minima, then one CTA over the partials ----------
constexpr int kRedThreads = 256;

__device__ __forceinline__ double warp_min(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double block_min(double v) {
  __shared__ double sw[kRedThreads / 32];
  v = warp_min(v);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) sw[wid] = v;
  __syncthreads();
  if (wid == 0) {
    v = lane < kRedThreads / 32 ? sw[lane] : 1e+6;
    v = warp_min(v);
  }
  return v;
}

// The reference seeds every thread with 1e+6 (src/TimeAdvanceFunc.cu:152), so a block
// whose every dt exceeds 1e6 reports 1e6; the same seed is kept here.
__global__ void __launch_bounds__(kRedThreads) k_min_partial(const double *src, long long n, double *partial) {
  double v = 1e+6;
  for (long long t = (long long)blockIdx.x * kRedThreads + threadIdx.x; t < n; t += (long long)gridDim.x * kRedThreads)
    v = fmin(v, src[t]);
  v = block_min(v);
  if (threadIdx.x == 0) partial[blockIdx.x] = v;
}

__global__ void __launch_bounds__(kRedThreads) k_min_final(const double *partial, int n, double *out) {
  double v = 1e+6;
  for (int t = threadIdx.x; t < n; t += kRedThreads) v = fmin(v, partial[t]);
  v = block_min(v);
  if (threadIdx.x == 0) *out = fmin(*out, v);
}

__global__ void k_set_value(double *dst, double v) { *dst = v; }

int launch_set_value(double *dst, double v, cudaStream_t s, int &n_launch) {
  k_set_value<<<1, 1, 0, s>>>(dst, v);
  ++n_launch;
  return check_launch();
}

// Grid-stride FP64 -> FP32 conversion (coalesced 8-byte loads and 4-byte stores).
__global__ void k_to_f32(const double *__restrict__ src, float *__restrict__ dst, size_t n) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = (float)src[i];
}

int launch_to_f32(const double *src, float *dst, size_t n, cudaStream_t s, int &n_launch) {
  if (n == 0) return CB2_OK;
  const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 32);
  k_to_f32<<<blocks, 256, 0, s>>>(src, dst, n);
  ++n_launch;
  return check_launch();
}

int min_reduce_partials(long long n) {
  long long b = (n + kRedThreads - 1) / kRedThreads;
  if (b > 148 * 8) b = 148 * 8;
  if (b < 1) b = 1;
  return (int)b;
}

// out must hold the running minimum on entry (the caller seeds it, e.g. with 1e6).
int launch_min_reduce(const double *src, long long n, double *partial, int n_partial, double *out, cudaStream_t s,
                      int &n_launch) {
  ProfScope prof("min_reduce", s);
  k_min_partial<<<n_partial, kRedThreads, 0, s>>>(src, n, partial);
  CB2_TRY(check_launch());
  k_min_final<<<1, kRedThreads, 0, s>>>(partial, n_partial, out);
  n_launch += 2;
  return check_launch();
}

}  // namespace cb2

namespace cb2 {

// ---- shock sensor (compute_shock_sensor, src/FieldOperation.cu:123-228) -------------------
// Computed on interior nodes once per step; the ghost values are never written (the
// reference's RK3 loop never exchanges them either), so the caller's zero fill stands there.
__global__ void __launch_bounds__(kPropThreads) k_shock_sensor(Zone z, Param p) {
  const int i = blockIdx.x * kPropThreads + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= z.mx) return;
  const Layout &L = z.L;
  const idx_t sz = L.sz, g = L.at(i, j, k);
  const idx_t st[3] = {1, L.disp2, L.disp1};
  const double *bv = z.bv;
  double sensor = 1;
  if (p.shock_sensor == 1) {  // modified Jameson (src/FieldOperation.cu:172-185)
    const double *pp = bv + 4 * sz + g;
    const double twoP = pp[0] * 2;
    double s = 0;
    for (int a = 0; a < 3; ++a) {
      const double pn = pp[st[a]] + pp[-st[a]];
      s += fabs(pn - twoP) / (pn + twoP);
    }
    sensor = s;
  } else if (p.shock_sensor == 2) {  // density / pressure jump (src/FieldOperation.cu:187-205)
    const double rho = bv[g], rhoI = 1.0 / rho, pr = bv[g + 4 * sz], pI = 1.0 / pr;
    double s = 0;
    for (int a = 0; a < 3; ++a) s = fmax(s, fabs(bv[g + st[a]] - rho) * rhoI);
    for (int a = 0; a < 3; ++a) s = fmax(s, fabs(bv[g + 4 * sz + st[a]] - pr) * pI);
    sensor = s;
  } else {  // modified Ducros (src/FieldOperation.cu:123-170)
    constexpr double c12 = 1.0 / 12.0, c23 = 2.0 / 3.0;
    double d[3][3];  // d[var u,v,w][dir]
    for (int c = 0; c < 3; ++c) {
      const double *f = bv + (1 + c) * sz + g;
      for (int a = 0; a < 3; ++a)
        d[c][a] = c12 * f[-2 * st[a]] - c23 * f[-st[a]] + c23 * f[st[a]] - c12 * f[2 * st[a]];
    }
    const double *M = z.metric + g;
    auto cart = [&](int c, int x) { return d[c][0] * M[x * sz] + d[c][1] * M[(3 + x) * sz] + d[c][2] * M[(6 + x) * sz]; };
    double div = cart(0, 0) + cart(1, 1) + cart(2, 2);
    if (div > 0) sensor = 0;
    else {
      const double duDy = cart(0, 1), duDz = cart(0, 2), dvDx = cart(1, 0), dvDz = cart(1, 2);
      const double dwDx = cart(2, 0), dwDy = cart(2, 1);
      div *= div;
      const double curl2 = (dwDy - dvDz) * (dwDy - dvDz) + (duDz - dwDx) * (duDz - dwDx) + (dvDx - duDy) * (dvDx - duDy);
      sensor = div / (div + curl2 + p.sensor_eps);
    }
  }
  z.shock[g] = sensor;
}

int launch_shock_sensor(const Zone &z, const Param &p, cudaStream_t s, int &n_launch) {
  dim3 grid((z.mx + kPropThreads - 1) / kPropThreads, z.my, z.mz);
  ProfScope prof("shock_sensor", s);
  k_shock_sensor<<<grid, kPropThreads, 0, s>>>(z, p);
  ++n_launch;
  return check_launch();
}

}  // namespace cb2
