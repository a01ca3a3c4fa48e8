// Loop control of the device-driven step loop: the last node of the step graph that the WHILE
// node of cb2_rk3_run repeats.  The reference advances physical_time on the host after every
// step and stops once it reaches total_simulation_time or total_step (src/RK.cuh:240,257);
// here the same test runs on the device and sets the WHILE node's condition.
#include "launch.h"

namespace cb2 {

__global__ void k_run_advance(RunState *r, const double *dt, const unsigned *status, cudaGraphConditionalHandle h) {
  const double d = *dt;
  r->dt = d;
  r->time += d;
  r->step += 1;
  const bool ok = d > 0.0 && d < 1e300 && (status == nullptr || *status == 0u);
  cudaGraphSetConditional(h, (ok && r->step < r->max_steps && r->time < r->t_end) ? 1u : 0u);
}

int launch_run_advance(RunState *r, const double *dt, const unsigned *status, cudaGraphConditionalHandle h,
                       cudaStream_t s, int &n_launch) {
  k_run_advance<<<1, 1, 0, s>>>(r, dt, status, h);
  ++n_launch;
  return check_launch();
}

}  // namespace cb2
