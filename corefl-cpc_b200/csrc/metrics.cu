// Metrics and Jacobian of a block from its node coordinates (Block::compute_jac_metric,
// src/Mesh.cpp:244-528, the 2nd-order branch): half central differences of x, y, z along
// xi, eta, zeta, the Jacobian as their determinant, and the nine metric terms as the cofactors
// over it.  The reference computes them on the host once its ghost coordinates are in place
// (init_ghost_grid, src/Mesh.cpp:1013-1163); here the same arithmetic runs on the device, one
// thread per node of the ghost-ngg lattice, from coordinates carried with g1 >= ngg + 1 ghost
// layers (so every node's neighbours exist).
#include "common.cuh"
#include "launch.h"

namespace cb2 {

constexpr int kMetThreads = 128;

__global__ void __launch_bounds__(kMetThreads) k_metrics(const double *__restrict__ x, const double *__restrict__ y,
                                                        const double *__restrict__ z, Layout Lc, Layout Lm, int ngg,
                                                        double *__restrict__ metric, double *__restrict__ jac,
                                                        int *bad) {
  const int i = blockIdx.x * kMetThreads + threadIdx.x - ngg;
  const int j = blockIdx.y - ngg, k = blockIdx.z - ngg;
  if (i >= Lm.mx + ngg) return;
  const idx_t c = Lc.at(i, j, k);
  const idx_t s1 = 1, s2 = Lc.disp2, s3 = Lc.disp1;
  const double dxd1 = (x[c + s1] - x[c - s1]) * 0.5, dyd1 = (y[c + s1] - y[c - s1]) * 0.5,
               dzd1 = (z[c + s1] - z[c - s1]) * 0.5;
  const double dxd2 = (x[c + s2] - x[c - s2]) * 0.5, dyd2 = (y[c + s2] - y[c - s2]) * 0.5,
               dzd2 = (z[c + s2] - z[c - s2]) * 0.5;
  const double dxd3 = (x[c + s3] - x[c - s3]) * 0.5, dyd3 = (y[c + s3] - y[c - s3]) * 0.5,
               dzd3 = (z[c + s3] - z[c - s3]) * 0.5;
  const double J = dxd1 * dyd2 * dzd3 + dxd2 * dyd3 * dzd1 + dxd3 * dyd1 * dzd2 - dxd1 * dyd3 * dzd2 -
                   dxd2 * dyd1 * dzd3 - dxd3 * dyd2 * dzd1;
  const idx_t g = Lm.at(i, j, k), sz = Lm.sz;
  jac[g] = J;
  if (!(J > 0)) atomicAdd(bad, 1);  // the reference logs and aborts on a non-positive Jacobian
  metric[g] = (dyd2 * dzd3 - dyd3 * dzd2) / J;
  metric[g + sz] = (dxd3 * dzd2 - dxd2 * dzd3) / J;
  metric[g + 2 * sz] = (dxd2 * dyd3 - dxd3 * dyd2) / J;
  metric[g + 3 * sz] = (dyd3 * dzd1 - dyd1 * dzd3) / J;
  metric[g + 4 * sz] = (dxd1 * dzd3 - dxd3 * dzd1) / J;
  metric[g + 5 * sz] = (dxd3 * dyd1 - dxd1 * dyd3) / J;
  metric[g + 6 * sz] = (dyd1 * dzd2 - dyd2 * dzd1) / J;
  metric[g + 7 * sz] = (dxd2 * dzd1 - dxd1 * dzd2) / J;
  metric[g + 8 * sz] = (dxd1 * dyd2 - dxd2 * dyd1) / J;
}

}  // namespace cb2

using namespace cb2;

extern "C" int cb2_metrics(const double *x, const double *y, const double *z, int mx, int my, int mz, int g_coord,
                           int ngg, double *metric, double *jac, void *stream) {
  if (!x || !y || !z || !metric || !jac || mx < 1 || my < 1 || mz < 1 || ngg < 0 || g_coord < ngg + 1)
    return CB2_ERR_INVALID;
  const Layout Lc = make_layout(mx, my, mz, g_coord), Lm = make_layout(mx, my, mz, ngg);
  cudaStream_t s = (cudaStream_t)stream;
  int *bad = nullptr;
  CB2_TRY(check_cuda(cudaMalloc(&bad, sizeof(int))));
  int rc = check_cuda(cudaMemsetAsync(bad, 0, sizeof(int), s));
  if (rc == CB2_OK) {
    dim3 grid((mx + 2 * ngg + kMetThreads - 1) / kMetThreads, my + 2 * ngg, mz + 2 * ngg);
    k_metrics<<<grid, kMetThreads, 0, s>>>(x, y, z, Lc, Lm, ngg, metric, jac, bad);
    rc = check_launch();
  }
  int nbad = 0;
  if (rc == CB2_OK) rc = check_cuda(cudaMemcpyAsync(&nbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s));
  if (rc == CB2_OK) rc = check_cuda(cudaStreamSynchronize(s));
  cudaFree(bad);
  if (rc == CB2_OK && nbad > 0) rc = CB2_ERR_NONPHYSICAL;
  return rc;
}
