// Batched closed blocks: many 2-D / 3-D blocks of uneven size advanced by whole SSP-RK3 steps in
// one persistent launch.  Each CTA takes the next block from a work queue ordered by decreasing
// size, runs its steps with the block path's per-node functions (the sweep tiles of
// inviscid_pv.cuh, stage_update_point, the periodic pair items of boundary.cuh,
// properties_point), CTA barriers standing in for the kernel boundaries of cb2_rk3_step, and then
// takes the next block.  The order of every phase is the block path's (RK3<mix>, src/RK.cuh:
// 107-237 for an inviscid air case with periodic faces), so a block's results are bitwise those
// of cb2_rk3_step on it.
#include <algorithm>
#include <vector>
#include <cooperative_groups.h>
#include "point.cuh"
#include "inviscid_pv.cuh"
#include "boundary.cuh"
#include "sweep.cuh"
#include "block_batch.h"

namespace cb2 {

__device__ __forceinline__ double cta_min(double v, double *red) {
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

// One phase: the y/z tiles of direction DIR over the whole block, tile t on cluster rank t % cs.
template <int DIR, int REC, int SOLVER, int NI>
__device__ __forceinline__ void sweep_yz(const Zone &z, const Param &p, unsigned char *smem, int rank, int cs) {
  constexpr int NSW = kSweepThreads / NI;
  const int nit = (z.mx + NI - 1) / NI;
  const int ms = DIR == 1 ? z.my : z.mz;
  const int nst = (ms + NSW - 3) / (NSW - 2);
  const int other = DIR == 1 ? z.mz : z.my;
  for (int t = rank; t < nit * nst * other; t += cs) {
    const int bx = t % nit, r = t / nit;
    pv_tile<double, 0, DIR, REC, SOLVER, NI>(z, p, 0, bx, r % nst, r / nst, smem);
  }
}

// A thread-block cluster advances one block at a time: cluster rank 0 takes the next block from
// the work queue, every phase spreads its tiles and nodes over the cluster's CTAs, and cluster
// barriers (release/acquire at cluster scope, which orders the global-memory writes) separate
// the phases.  All CTAs of a cluster follow the same control flow, so every barrier is reached
// by all of them.  mode 0: whole steps; mode 1: only the residual of one stage, for timing.
template <int REC, int SOLVER, int NI>
__global__ void __launch_bounds__(kSweepThreads) k_block_batch(BlockCase *cases, int n_cases, int max_steps,
                                                                int mode, int *queue) {
  namespace cg = cooperative_groups;
  extern __shared__ __align__(16) unsigned char bb_smem[];
  __shared__ double red[kSweepThreads / 32];
  __shared__ double s_part;
  __shared__ int s_case;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank(), cs = (int)cl.num_blocks();
  const int tid = threadIdx.x, nt = kSweepThreads;
  const long long g0 = (long long)rank * nt + tid, gs = (long long)cs * nt;  // cluster-wide thread index
  for (;;) {
    if (rank == 0 && tid == 0) s_case = atomicAdd(queue, 1);
    cl.sync();
    const int c = *cl.map_shared_rank(&s_case, 0);
    cl.sync();  // every CTA has read the case before rank 0 takes the next one
    if (c >= n_cases) return;
    BlockCase &bc = cases[c];
    if (bc.status) continue;
    const Zone &z = bc.z;
    const Param &p = bc.p;
    constexpr int NV = 5;
    const idx_t sz = z.L.sz, sz0 = z.L0.sz;
    const idx_t run = (idx_t)z.L.my * z.L.disp2;
    const int ntx = (int)((run + (kSweepThreads - 2) - 1) / (kSweepThreads - 2));
    const int g = z.ngg;
    const int px = z.mx + 2 * g, py = z.my + 2 * g, pz = z.mz + 2 * g;
    const long long npad = (long long)px * py * pz;
    const long long nint = (long long)z.mx * z.my * z.mz;
    auto residual = [&]() {
      for (long long e = g0; e < sz0 * NV; e += gs) z.dq[e] = 0.0;
      cl.sync();
      for (int t = rank; t < ntx * z.mz; t += cs) pv_tile<double, 0, 0, REC, SOLVER>(z, p, run, t % ntx, 0, t / ntx, bb_smem);
      cl.sync();
      sweep_yz<1, REC, SOLVER, NI>(z, p, bb_smem, rank, cs);
      cl.sync();
      if (z.mz > 1) {
        sweep_yz<2, REC, SOLVER, NI>(z, p, bb_smem, rank, cs);
        cl.sync();
      }
    };
    if (mode == 1) {
      residual();
      continue;
    }
    double time = bc.time;
    int step = 0;
    bool failed = false;
    double last = bc.last_dt;
    for (int s = 0; s < max_steps && time < bc.t_end; ++s) {
      for (long long e = g0; e < sz * NV; e += gs) z.qn[e] = z.cv[e];
      double dt = bc.dt_fixed;
      if (!(dt > 0)) {
        double m = 1e+6;
        bool bad = false;
        for (long long e = g0; e < nint; e += gs) {
          const int i = (int)(e % z.mx), r = (int)(e / z.mx);
          const double d = local_dt_point<0>(z, p, i, r % z.my, r / z.my);
          bad |= !(d > 0) || !isfinite(d);
          m = fmin(m, d);
        }
        m = cta_min(bad ? -1.0 : m, red);  // a bad step shows as a negative minimum
        if (tid == 0) s_part = m;
        cl.sync();
        dt = 1e+6;
        for (int r = 0; r < cs; ++r) dt = fmin(dt, *cl.map_shared_rank(&s_part, r));
        cl.sync();  // the partial minima are read before they are written again
        if (!(dt > 0)) {
          failed = true;
          break;
        }
      } else {
        cl.sync();  // qn is copied before any stage update overwrites cv
      }
      for (int rk = 0; rk < 3; ++rk) {
        residual();
        for (long long e = g0; e < nint; e += gs) {
          const int i = (int)(e % z.mx), r = (int)(e / z.mx);
          stage_update_point<0>(z, p, dt, rk, i, r % z.my, r / z.my);
        }
        cl.sync();
        for (int f = 0; f < bc.n_pairs; ++f) {
          const FaceBC &fb = bc.pairs[f];
          const long long items = (long long)(2 * g + 1) * (fb.end[0] - fb.start[0] + 1) *
                                  (fb.end[1] - fb.start[1] + 1) * (fb.end[2] - fb.start[2] + 1);
          for (long long t = g0; t < items; t += gs) bc_periodic_pair_item<0>(z, p, fb, t);
          cl.sync();
        }
        if (p.dim == 2 && z.mz == 1) {
          for (long long e = g0; e < (long long)px * py; e += gs)
            eliminate_k_gradient_point(z, p, (int)(e % px) - g, (int)(e / px) - g);
          cl.sync();
        }
        if (!(p.mu_constant > 0 && !z.mach)) {
          for (long long e = g0; e < npad; e += gs) {
            const int i = (int)(e % px) - g;
            const long long r = e / px;
            properties_point<0>(z, p, i, (int)(r % py) - g, (int)(r / py) - g);
          }
          cl.sync();
        }
      }
      time += dt;
      ++step;
      last = dt;
    }
    cl.sync();
    if (rank == 0 && tid == 0) {
      bc.time = time;
      bc.steps = step;
      bc.last_dt = last;
      int st = 0;
      if (time >= bc.t_end) st |= CB2_BLOCK_DONE;
      if (failed || bc.flags) st |= CB2_BLOCK_FAILED;
      bc.status = st;
    }
  }
}

template <int REC, int SOLVER, int NI>
static int batch_launch(BlockCase *cases, int n, int max_steps, int mode, int cs, int *queue, cudaStream_t s) {
  const size_t smem = std::max(pv_tile_smem<double, 0, REC, SOLVER>(0), pv_tile_smem<double, 0, REC, SOLVER>(1, NI));
  auto kern = k_block_batch<REC, SOLVER, NI>;
  CB2_TRY(prepare_smem(kern, smem));
  cudaLaunchConfig_t cfg{};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = (unsigned)cs;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.blockDim = dim3(kSweepThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3((unsigned)cs);
  int clusters = 0;
  CB2_TRY(check_cuda(cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg)));
  clusters = std::max(1, std::min(n, clusters));
  cfg.gridDim = dim3((unsigned)(clusters * cs));
  CB2_TRY(check_cuda(cudaMemsetAsync(queue, 0, sizeof(int), s)));
  CB2_TRY(check_cuda(cudaLaunchKernelEx(&cfg, kern, cases, n, max_steps, mode, queue)));
  return check_launch();
}

template <int REC, int SOLVER>
static int batch_launch_ni(BlockCase *cases, int n, int max_steps, int mode, int ni, int cs, int *queue,
                           cudaStream_t s) {
  if (ni == 4) return batch_launch<REC, SOLVER, 4>(cases, n, max_steps, mode, cs, queue, s);
  if (ni == 16) return batch_launch<REC, SOLVER, 16>(cases, n, max_steps, mode, cs, queue, s);
  return batch_launch<REC, SOLVER, 8>(cases, n, max_steps, mode, cs, queue, s);
}

bool block_batch_supported(const Param &p) {
  return p.n_spec == 0 && p.i_eve < 0 && p.viscous_order == 0 && p.precision == CB2_PREC_FP64 && !p.limit_flow &&
         (p.reconstruction == CB2_REC_WENO5 || p.reconstruction == CB2_REC_WENO7) &&
         (p.inviscid_scheme == CB2_INV_AUSMP || p.inviscid_scheme == CB2_INV_HLLC);
}

int launch_block_batch(BlockCase *cases, int n, const Param &p, int max_steps, int mode, int ni, int cs,
                       int *queue, cudaStream_t s) {
  if (cs < 1 || cs > 8) return CB2_ERR_INVALID;
  if (n <= 0) return CB2_OK;
  if (!block_batch_supported(p)) return CB2_ERR_UNSUPPORTED;
  ProfScope prof(mode == 1 ? "block_batch_residual" : "block_batch", s);
  const bool w7 = p.reconstruction == CB2_REC_WENO7, ausm = p.inviscid_scheme == CB2_INV_AUSMP;
  if (w7 && ausm) return batch_launch_ni<7, CB2_INV_AUSMP>(cases, n, max_steps, mode, ni, cs, queue, s);
  if (w7) return batch_launch_ni<7, CB2_INV_HLLC>(cases, n, max_steps, mode, ni, cs, queue, s);
  if (ausm) return batch_launch_ni<5, CB2_INV_AUSMP>(cases, n, max_steps, mode, ni, cs, queue, s);
  return batch_launch_ni<5, CB2_INV_HLLC>(cases, n, max_steps, mode, ni, cs, queue, s);
}

}  // namespace cb2
