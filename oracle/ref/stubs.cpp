// Host stand-ins for the reference's runtime hooks that the parser links against.
// TEST INFRASTRUCTURE ONLY.
#include <cstdio>
#include <cstdlib>
#include "Parallel.h"
#include "kernels.h"

double cfd::MpiParallel::get_wall_time() { return 0.0; }
void cfd::MpiParallel::barrier() {}
void cfd::MpiParallel::exit() {
  std::fprintf(stderr, "reference parser requested exit\n");
  std::exit(1);
}
cfd::MpiParallel::~MpiParallel() = default;
void cfd::setup_gpu_device(int, int) {}
