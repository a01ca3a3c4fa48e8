// Explicit finite-rate chemistry source over a block (the launch of finite_rate_chemistry,
// src/FiniteRateChem.cu:1406-1488); the per-node arithmetic is in chem.cuh.
#include "chem.cuh"
#include "launch.h"

namespace cb2 {

constexpr int kChemThreads = 128;

// Bounded to 128 registers (4 CTAs of 128 threads per SM): the 9-species kernel otherwise takes
// 168 and runs 3 CTAs; its latency-bound exponentials gain more from the extra warps than the
// few spills cost (192^3 H2/air box: 27.0 -> 22.7 ms per step).
template <int NS>
__global__ void __launch_bounds__(kChemThreads, 4) k_chemistry(Zone z, Param p) {
  const int i = blockIdx.x * kChemThreads + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
  if (i >= z.mx) return;
  chemistry_point<NS>(z, p, i, j, k);
}

int launch_chemistry(const Zone &z, const Param &p, cudaStream_t s, int &n_launch) {
  dim3 grid((z.mx + kChemThreads - 1) / kChemThreads, z.my, z.mz);
  ProfScope prof("chemistry", s);
  ++n_launch;
  switch (p.n_spec) {
    case 5: k_chemistry<5><<<grid, kChemThreads, 0, s>>>(z, p); break;
    case 9: k_chemistry<9><<<grid, kChemThreads, 0, s>>>(z, p); break;
    default: return CB2_ERR_UNSUPPORTED;
  }
  return check_launch();
}

}  // namespace cb2
