// Per-item device functions of the periodic and 2-D ghost fills, shared by the block kernels
// (boundary.cu) and the batched block kernel (block_batch.cu).
#pragma once
#include "common.cuh"
#include "launch.h"
#include "point.cuh"

namespace cb2 {

// 2-D blocks: copy the k = 0 plane into every k ghost plane (eliminate_k_gradient,
// src/FieldOperation.cu:96-121).
__device__ __forceinline__ void eliminate_k_gradient_point(const Zone &z, const Param &p, int i, int j) {
  const int g_ = z.ngg;
  const idx_t sz = z.L.sz;
  const idx_t g0 = z.L.at(i, j, 0);
  for (int kk = 1; kk <= g_; ++kk) {
    const idx_t gp = z.L.at(i, j, kk), gm = z.L.at(i, j, -kk);
    for (int l = 0; l < 6; ++l) { z.bv[gp + l * sz] = z.bv[g0 + l * sz]; z.bv[gm + l * sz] = z.bv[g0 + l * sz]; }
    for (int l = 0; l < p.n_scalar; ++l) { z.sv[gp + l * sz] = z.sv[g0 + l * sz]; z.sv[gm + l * sz] = z.sv[g0 + l * sz]; }
    for (int l = 0; l < p.n_var; ++l) { z.cv[gp + l * sz] = z.cv[g0 + l * sz]; z.cv[gm + l * sz] = z.cv[g0 + l * sz]; }
  }
}

// ---- both periodic faces of one direction in one launch -----------------------------------
// Work item p of a face line: p = 0 averages the two coincident end nodes, p in [1, g] fills
// left ghost -p from node m-1-p, p in [g+1, 2g] fills right ghost m-1+(p-g) from node p-g.
// Applying the two faces one after the other gives exactly this when no copy source is an end
// node (m >= g + 2) and both faces span the same tangential range; the launcher checks both.
// Items are ordered so that consecutive threads touch consecutive addresses: along x the item
// index runs fastest, along y/z the i index does.
struct PairItem {
  int p, i, j, k;  // i, j, k of the left face node
};

__device__ __forceinline__ bool pair_item(const FaceBC &f, int g, long long t, PairItem &it) {
  const int P = 2 * g + 1;
  const int n0 = f.end[0] - f.start[0] + 1, n1 = f.end[1] - f.start[1] + 1, n2 = f.end[2] - f.start[2] + 1;
  if (t >= (long long)P * n0 * n1 * n2) return false;
  if (f.face == 0) {
    it.p = (int)(t % P); t /= P;
    it.i = f.start[0];
    it.j = f.start[1] + (int)(t % n1);
    it.k = f.start[2] + (int)(t / n1);
  } else {
    it.i = f.start[0] + (int)(t % n0); t /= n0;
    it.p = (int)(t % P); t /= P;
    if (f.face == 1) { it.j = f.start[1]; it.k = f.start[2] + (int)t; }
    else { it.j = f.start[1] + (int)t; it.k = f.start[2]; }
  }
  return true;
}

// Node at offset `off` along the face direction from node (i,j,k) with the direction index
// replaced by `e`.
__device__ __forceinline__ idx_t along(const Layout &L, int face, int i, int j, int k, int e) {
  if (face == 0) return L.at(e, j, k);
  if (face == 1) return L.at(i, e, k);
  return L.at(i, j, e);
}

template <int NS>
__device__ __forceinline__ void bc_periodic_pair_item(const Zone &z, const Param &p, const FaceBC &f, long long t) {
  PairItem it;
  const int g = z.ngg;
  if (!pair_item(f, g, t, it)) return;
  const int m = f.face == 0 ? z.mx : (f.face == 1 ? z.my : z.mz);
  const idx_t sz = z.L.sz;
  if (it.p == 0) {
    const idx_t ga = along(z.L, f.face, it.i, it.j, it.k, 0), gb = along(z.L, f.face, it.i, it.j, it.k, m - 1);
    for (int l = 0; l < 6; ++l) {
      const double ave = 0.5 * (z.bv[ga + l * sz] + z.bv[gb + l * sz]);
      z.bv[ga + l * sz] = ave;
      z.bv[gb + l * sz] = ave;
    }
    for (int l = 0; l < p.n_scalar; ++l) {
      const double ave = 0.5 * (z.sv[ga + l * sz] + z.sv[gb + l * sz]);
      z.sv[ga + l * sz] = ave;
      z.sv[gb + l * sz] = ave;
    }
    cv_point<NS>(z, p, ga);
    cv_point<NS>(z, p, gb);
    return;
  }
  const bool left = it.p <= g;
  const int dst = left ? -it.p : m - 1 + (it.p - g);
  const int src = left ? m - 1 - it.p : it.p - g;
  const idx_t gg = along(z.L, f.face, it.i, it.j, it.k, dst), gs = along(z.L, f.face, it.i, it.j, it.k, src);
  for (int l = 0; l < 6; ++l) z.bv[gg + l * sz] = z.bv[gs + l * sz];
  for (int l = 0; l < p.n_scalar; ++l) z.sv[gg + l * sz] = z.sv[gs + l * sz];
  cv_point<NS>(z, p, gg);
}

}  // namespace cb2
