// D2Q9 instantiations of the AA kernel family (with the fused D2Q5 tracers).
#include "aa_launch.cuh"

namespace lbm {
cudaError_t launch_step_d2q9(const lbm_sim& sim, bool even, bool write_moments) {
  return launch_lattice<D2Q9>(sim, even, write_moments);
}
}  // namespace lbm
