// Batched closed blocks (block_batch.cu): the device record of one block and the launcher.
#pragma once
#include "common.cuh"
#include "launch.h"
#include "cb200_serve.h"

namespace cb2 {

struct BlockCase {
  Zone z;
  Param p;           // the context's settings, dim set by the block, status -> flags
  FaceBC pairs[3];   // the left face of each periodic direction, in face-list order
  int n_pairs;
  double time, t_end, dt_fixed, last_dt;
  int steps, status;
  unsigned flags;    // non-physical-state bits of this block's stage updates
};

bool block_batch_supported(const Param &p);
// mode 0: advance by up to max_steps steps; mode 1: one residual (dq) of every block, for timing.
// cs: CTAs per thread-block cluster, which shares one block (1..8).  queue: one device int, the
// work counter of the persistent grid.
int launch_block_batch(BlockCase *cases, int n, const Param &p, int max_steps, int mode, int ni, int cs,
                       int *queue, cudaStream_t s);

}  // namespace cb2
