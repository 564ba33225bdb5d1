// Host-side dispatch of the AA kernel family for one fluid lattice. Included by one .cu file per
// lattice so the instantiations compile in parallel.
#pragma once

#include "aa_step.cuh"
#include "sim.h"

namespace lbm {

template <class Real>
StepArgs<Real> make_step_args(const lbm_sim& s, bool write_moments) {
  StepArgs<Real> a{};
  a.f = s.f;
  a.rho = static_cast<Real*>(s.rho);
  a.vel = static_cast<Real*>(s.vel);
  a.flags = s.flags;
  if (s.dim == 3) {
    a.nx = (int)s.counts[0];
    a.ny = (int)s.counts[1];
    a.nz = (int)s.counts[2];
  } else {
    a.nx = 1;
    a.ny = (int)s.counts[0];
    a.nz = (int)s.counts[1];
  }
  a.n = s.n;
  a.om_pos = s.om_pos;
  a.om_neg = s.om_neg;
  const int off = 3 - s.dim;
  // Acceleration source, as src/simulation.rs:326-373 leaves it for the fluid kernel: any
  // Boussinesq coupling overwrites the constant acceleration every step, the last one winning.
  if (!s.couplings.empty()) {
    const lbm_sim::Coupling& c = s.couplings.back();
    a.acc_mode = kAccBoussinesq;
    for (int k = 0; k < s.dim; ++k) a.acc[off + k] = c.g[k];
    a.alpha = c.alpha;
    a.c0 = c.c0;
    a.coupled = c.tracer;
    a.coupled_val = static_cast<const Real*>(s.tracers[c.tracer].val);
  } else if (s.has_gravity) {
    a.acc_mode = kAccConstant;
    for (int k = 0; k < s.dim; ++k) a.acc[off + k] = s.gravity[k];
  }
  a.ntracers = (int)s.tracers.size();
  for (int t = 0; t < a.ntracers; ++t) {
    a.tr[t].g = static_cast<Real*>(s.tracers[t].g);
    a.tr[t].val = static_cast<Real*>(s.tracers[t].val);
    a.tr[t].omega = s.tracers[t].omega;
  }
  a.write_moments = write_moments ? 1 : 0;
  a.status = s.status;
  return a;
}

template <class Real>
void step_geometry(const StepArgs<Real>& a, dim3& grid, dim3& block) {
  const int bx = a.nz >= 256 ? 256 : ((a.nz + 31) / 32) * 32;
  block = dim3(bx, 1, 1);
  grid = dim3((a.nz + bx - 1) / bx, a.ny < 65535 ? a.ny : 65535, a.nx < 65535 ? a.nx : 65535);
}

template <class L, bool TRT, int K>
cudaError_t launch_typed(const lbm_sim& s, bool even, bool write_moments) {
  using Real = typename Pop<K>::real;
  const StepArgs<Real> a = make_step_args<Real>(s, write_moments);
  dim3 grid, block;
  step_geometry(a, grid, block);
  const bool tracers = a.ntracers > 0;
  if (even) {
    if (tracers)
      aa_step_kernel<L, TRT, K, true, true><<<grid, block, 0, s.stream>>>(a);
    else
      aa_step_kernel<L, TRT, K, true, false><<<grid, block, 0, s.stream>>>(a);
  } else {
    if (tracers)
      aa_step_kernel<L, TRT, K, false, true><<<grid, block, 0, s.stream>>>(a);
    else
      aa_step_kernel<L, TRT, K, false, false><<<grid, block, 0, s.stream>>>(a);
  }
  return cudaGetLastError();
}

template <class L>
cudaError_t launch_lattice(const lbm_sim& s, bool even, bool write_moments) {
  const bool trt = s.collision == 1;
  switch (s.storage) {
    case kF32:
      return trt ? launch_typed<L, true, kF32>(s, even, write_moments)
                 : launch_typed<L, false, kF32>(s, even, write_moments);
    case kF16:
      return trt ? launch_typed<L, true, kF16>(s, even, write_moments)
                 : launch_typed<L, false, kF16>(s, even, write_moments);
    case kBF16:
      return trt ? launch_typed<L, true, kBF16>(s, even, write_moments)
                 : launch_typed<L, false, kBF16>(s, even, write_moments);
    case kF64:
      return trt ? launch_typed<L, true, kF64>(s, even, write_moments)
                 : launch_typed<L, false, kF64>(s, even, write_moments);
  }
  return cudaErrorInvalidValue;
}

}  // namespace lbm
