// Tiling of one directional sweep (x, y or z) for the pencil kernels.
//
// A CTA of kSweepThreads threads owns kSweepThreads consecutive interfaces and updates the
// kSweepThreads-1 nodes between them (CTAs overlap by one interface), so every thread
// computes exactly one interface flux in one pass and the flux difference is taken from
// shared memory.
//
// x sweep: positions are taken along the padded k-slab as a 1-D array (consecutive
//   j-lines are adjacent in the padded layout), so a CTA streams one contiguous range of
//   cv/bv/metric; interfaces whose i falls outside [-1, mx-1] are skipped.
// y/z sweep: a CTA owns kTI consecutive i (coalesced) x kTS interfaces along the sweep.
#pragma once
#include "common.cuh"

namespace cb2 {

constexpr int kSweepThreads = 256;
constexpr int kTI = 16;                  // i-columns per y/z tile
constexpr int kTS = kSweepThreads / kTI; // interfaces per column in a y/z tile

struct SweepGeom {
  int dir;
  // x sweep
  idx_t run;       // number of padded positions of the interior j-lines of one k-slab
  // y/z sweep
  int n_itile;     // tiles along i
  int n_stile;     // tiles along the sweep direction
};

// Number of shared-memory node slots a tile needs for a stencil half-width r.
__host__ __device__ __forceinline__ int sweep_nodes(int dir, int r) {
  return dir == 0 ? (kSweepThreads + 2 * r - 1) : kTI * (kTS + 2 * r - 1);
}

// Node-centred tiling: a CTA of kSweepThreads threads owns kSweepThreads consecutive nodes
// along the sweep; each thread reconstructs both faces of its node, the interfaces between
// neighbouring threads are formed from shared memory, and the kSweepThreads-2 inner nodes are
// updated (CTAs overlap by two nodes).  x sweep: one contiguous padded run as above.  y/z
// sweep: kNI consecutive i x kNS nodes along the sweep.
constexpr int kNI = 8;
constexpr int kNS = kSweepThreads / kNI;

__host__ __device__ __forceinline__ int node_sweep_nodes(int dir, int r) {
  return dir == 0 ? (kSweepThreads + 2 * r) : kNI * (kNS + 2 * r);
}

// ni: i-columns of a y/z tile (kSweepThreads / ni nodes along the sweep); the autotuner picks
// it per block and direction among kTileNI.
constexpr int kTileNI[3] = {4, 8, 16};

inline dim3 node_sweep_grid(int dir, const Layout &L, SweepGeom &g, int ni = kNI) {
  g.dir = dir;
  if (dir == 0) {
    g.run = (idx_t)L.my * L.disp2;
    const idx_t per = kSweepThreads - 2;
    return dim3((unsigned)((g.run + per - 1) / per), 1, (unsigned)L.mz);
  }
  const int ns = kSweepThreads / ni;
  g.n_itile = (L.mx + ni - 1) / ni;
  const int ms = dir == 1 ? L.my : L.mz;
  g.n_stile = (ms + ns - 3) / (ns - 2);
  const int other = dir == 1 ? L.mz : L.my;
  return dim3((unsigned)g.n_itile, (unsigned)g.n_stile, (unsigned)other);
}

inline dim3 sweep_grid(int dir, const Layout &L, SweepGeom &g) {
  g.dir = dir;
  if (dir == 0) {
    g.run = (idx_t)L.my * L.disp2;
    const idx_t per = kSweepThreads - 1;
    return dim3((unsigned)((g.run + per - 1) / per), 1, (unsigned)L.mz);
  }
  g.n_itile = (L.mx + kTI - 1) / kTI;
  const int ms = dir == 1 ? L.my : L.mz;
  g.n_stile = (ms + kTS - 2) / (kTS - 1);
  const int other = dir == 1 ? L.mz : L.my;
  return dim3((unsigned)g.n_itile, (unsigned)g.n_stile, (unsigned)other);
}

}  // namespace cb2
