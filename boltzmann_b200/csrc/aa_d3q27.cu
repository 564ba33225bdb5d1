// D3Q27 instantiations of the AA kernel family (with the fused D3Q7 tracers).
#include "aa_launch.cuh"

namespace lbm {
cudaError_t launch_step_d3q27(const lbm_sim& sim, bool even, bool write_moments) {
  return launch_lattice<D3Q27>(sim, even, write_moments);
}
}  // namespace lbm
