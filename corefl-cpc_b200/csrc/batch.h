// Batched 1-D cases (batch.cu) and the serving loop (serve.cu).
#pragma once
#include "common.cuh"
#include "launch.h"

namespace cb2 {

// One 1-D case of a batch, in device memory.  The arrays of z live in the server's pool.
struct LineCase {
  Zone z;
  Param p;          // the scheme settings, with p.status pointing at `flags` of this case
  double time, t_end, last_dt;
  int step, status, active;
  unsigned flags;   // non-physical-state bits of this case's stage updates
};
constexpr int kLineDone = 1;
constexpr int kLineFailed = 2;  // a non-finite or non-positive time step, or a non-physical state

// Advances every active, unfinished case of cases[0..n) by up to max_steps RK3 steps, one CTA
// per case.  p selects the kernel instantiation; each case carries its own copy of the settings.
int launch_line_batch(LineCase *cases, int n, const Param &p, int max_steps, cudaStream_t s);
bool line_batch_supported(const Param &p);
// Initial two-state shock tube of case `slot` (its arrays and settings already assigned).
int launch_line_setup(LineCase *cases, int slot, int mx, int g, const Param &p, double TL, double pL, double TR,
                      double pR, const double *Y, double dx, double x_split, cudaStream_t s);

}  // namespace cb2
