// The 8th-order central first derivative along one index direction with the reference's
// one-sided closures on the four nodes next to a physical boundary (d_dXi / d_dEta / d_dZeta,
// src/ViscousScheme.cu:140-468), and the physical-boundary flags of a node.  Shared by the
// viscous kernels and the primitive-variable sweeps that take the viscous divergence along their
// direction.
#pragma once
#include "common.cuh"

namespace cb2 {

// ---- 8th-order derivative along one index direction ---------------------------------
// f(m) returns the field at offset m along the direction; n = node index, nx = extent.
template <typename T, typename F>
__device__ __forceinline__ T d8(F f, int n, int nx, bool bl, bool br) {
  if (bl) {
    if (n == 0) return T(-25.0 / 12) * f(0) + T(4.0) * f(1) - 3 * f(2) + T(4.0 / 3) * f(3) - T(0.25) * f(4);
    if (n == 1) return T(-0.25) * f(-1) - T(5.0 / 6) * f(0) + T(1.5) * f(1) - T(0.5) * f(2) + T(1.0 / 12) * f(3);
    if (n == 2) return T(-1.0 / 12) * (f(2) - f(-2)) + T(2.0 / 3) * (f(1) - f(-1));
    if (n == 3) return T(0.75) * (f(1) - f(-1)) - T(0.15) * (f(2) - f(-2)) + T(1.0 / 60) * (f(3) - f(-3));
  }
  if (br) {
    if (n == nx - 1) return T(25.0 / 12) * f(0) - T(4.0) * f(-1) + 3 * f(-2) - T(4.0 / 3) * f(-3) + T(0.25) * f(-4);
    if (n == nx - 2) return T(0.25) * f(1) + T(5.0 / 6) * f(0) - T(1.5) * f(-1) + T(0.5) * f(-2) - T(1.0 / 12) * f(-3);
    if (n == nx - 3) return T(-1.0 / 12) * (f(2) - f(-2)) + T(2.0 / 3) * (f(1) - f(-1));
    if (n == nx - 4) return T(0.75) * (f(1) - f(-1)) - T(0.15) * (f(2) - f(-2)) + T(1.0 / 60) * (f(3) - f(-3));
  }
  return T(0.8) * (f(1) - f(-1)) + T(-0.2) * (f(2) - f(-2)) + T(4.0 / 105) * (f(3) - f(-3)) +
         T(-1.0 / 280) * (f(4) - f(-4));
}

struct BFlags {
  bool il, ir, jl, jr, kl, kr;
};

__device__ __forceinline__ BFlags bflags(const Zone &z, int i, int j, int k) {
  BFlags b;
  b.il = z.bt.il[j + k * z.my] != 0;
  b.ir = z.bt.ir[j + k * z.my] != 0;
  b.jl = z.bt.jl[i + k * z.mx] != 0;
  b.jr = z.bt.jr[i + k * z.mx] != 0;
  b.kl = z.bt.kl[i + j * z.mx] != 0;
  b.kr = z.bt.kr[i + j * z.mx] != 0;
  return b;
}

}  // namespace cb2
