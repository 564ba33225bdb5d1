/*
 * TEST INFRASTRUCTURE (the checker, never the product).
 *
 * Host loop around the reference's own OpenCL kernels, compiled as C++:
 *   - src/lib.cl (djbarker/boltzmann), included unmodified from the reference tree;
 *   - update_d3q27_trt, update_d2q5_trt and update_d3q7_trt, which the reference never
 *     registers (src/opencl.rs:123-129) but whose source its generator
 *     python/boltzmann/kernel_gen.py:250-462 produces; oracle/build.py writes them to
 *     oracle/_ref/gen/ at build time.
 *
 * The loop restates Simulation::iterate (src/simulation.rs:278-446): the constant-acceleration
 * pass once per call, then per step every Boussinesq pass (last one wins), the fluid kernel,
 * then every tracer kernel, with even = 1 - step % 2. Work-items run in-range only
 * (x, y[, z] < counts); OpenMP splits the slow x axis over host threads.
 *
 * Built only by oracle/build.py into oracle/_ref/, only where the reference tree exists.
 */
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <omp.h>

#include "ref_shim.h"

#include "lib.cl"
#include "update_d3q27_trt.cl"
#include "update_d2q5_trt.cl"
#include "update_d3q7_trt.cl"

namespace {

thread_local std::string g_err;

int fail(const char* msg) {
  g_err = msg;
  return 1;
}

// Runs fn(ix, iy, iz) once per in-range work-item, x split over threads.
template <class Fn>
void for_each_work_item(int dim, const int* s, int nthreads, Fn fn) {
  const long nx = s[0];
  const long ny = dim > 1 ? s[1] : 1;
  const long nz = dim > 2 ? s[2] : 1;
#pragma omp parallel for schedule(static) num_threads(nthreads)
  for (long ix = 0; ix < nx; ++ix) {
    for (long iy = 0; iy < ny; ++iy) {
      for (long iz = 0; iz < nz; ++iz) {
        ref_work_item_id[0] = (size_t)ix;
        ref_work_item_id[1] = (size_t)iy;
        ref_work_item_id[2] = (size_t)iz;
        fn();
      }
    }
  }
}

}  // namespace

extern "C" {

const char* lbm_ref_last_error(void) { return g_err.c_str(); }

/* One call == Simulation::iterate(iters) after the upload (src/simulation.rs:278-446).
 * Arrays are the reference's host layouts: f [N, q], rho [N], vel [N, dim], acc [N, dim],
 * tracer g [N, q_t], C [N]; N = prod(counts) in row-major order (x slowest).
 * collision (fluid and each tracer): 0 = BGK, 1 = TRT; a tracer's rates are t_om (omega or
 * omega+) and t_om_neg. */
int lbm_ref_iterate(int dim, const int64_t* counts, int32_t* flags, int q, int collision,
                    float om_pos, float om_neg, float* f, float* rho, float* vel, float* acc,
                    int use_acc, const float* gravity, int ncouplings, const int32_t* c_tracer,
                    const float* c_alpha, const float* c_c0, const float* c_g, int ntracers,
                    const int32_t* t_q, const int32_t* t_collision, const float* t_om,
                    const float* t_om_neg, float* const* t_g, float* const* t_C, int64_t iters,
                    int nthreads) {
  if (iters % 2 != 0) return fail("iters must be even");
  if (dim < 2 || dim > 3) return fail("no update kernel for this dimension");
  if (nthreads <= 0) nthreads = omp_get_max_threads();

  int s[3] = {(int)counts[0], dim > 1 ? (int)counts[1] : 1, dim > 2 ? (int)counts[2] : 1};
  float dummy[4] = {0, 0, 0, 0};
  float* acc_arg = use_acc ? acc : dummy;
  float* grav = const_cast<float*>(gravity);

  const bool fluid_ok = (dim == 2 && q == 9) || (dim == 3 && q == 27);
  if (!fluid_ok) return fail("Kernel not found (fluid)");
  for (int t = 0; t < ntracers; ++t) {
    const bool ok = (t_collision[t] == 0 || t_collision[t] == 1) &&
                    ((dim == 2 && t_q[t] == 5) || (dim == 3 && t_q[t] == 7));
    if (!ok) return fail("Kernel not found (tracer)");
  }

  // Constant acceleration, once per iterate call (src/simulation.rs:326-342).
  if (gravity != nullptr) {
    if (!use_acc) return fail("gravity without an acceleration buffer");
    if (dim == 2)
      for_each_work_item(dim, s, nthreads, [&] { set_constant_acc_2d(s, acc_arg, grav); });
    else
      for_each_work_item(dim, s, nthreads, [&] { set_constant_acc_3d(s, acc_arg, grav); });
  }

  for (int64_t it = 0; it < iters; ++it) {
    const int even = (int)(1 - it % 2);

    // Boussinesq sources, in coupling order (src/simulation.rs:352-373).
    for (int k = 0; k < ncouplings; ++k) {
      float* conc = t_C[c_tracer[k]];
      float alpha = c_alpha[k], c0 = c_c0[k];
      float* g = const_cast<float*>(c_g + (size_t)k * dim);
      if (dim == 2)
        for_each_work_item(dim, s, nthreads,
                           [&] { set_boussinesq_acc_2d(s, acc_arg, conc, alpha, c0, g); });
      else
        for_each_work_item(dim, s, nthreads,
                           [&] { set_boussinesq_acc_3d(s, acc_arg, conc, alpha, c0, g); });
    }

    // Fluid (src/simulation.rs:375-408).
    if (dim == 2 && collision == 0)
      for_each_work_item(dim, s, nthreads, [&] {
        update_d2q9_bgk(s, even, om_pos, f, rho, vel, acc_arg, use_acc, flags);
      });
    else if (dim == 2)
      for_each_work_item(dim, s, nthreads, [&] {
        update_d2q9_trt(s, even, om_pos, om_neg, f, rho, vel, acc_arg, use_acc, flags);
      });
    else if (collision == 0)
      for_each_work_item(dim, s, nthreads, [&] {
        update_d3q27_bgk(s, even, om_pos, f, rho, vel, acc_arg, use_acc, flags);
      });
    else
      for_each_work_item(dim, s, nthreads, [&] {
        update_d3q27_trt(s, even, om_pos, om_neg, f, rho, vel, acc_arg, use_acc, flags);
      });

    // Tracers (src/simulation.rs:410-432).
    for (int t = 0; t < ntracers; ++t) {
      float* g = t_g[t];
      float* C = t_C[t];
      float om = t_om[t], om_n = t_om_neg[t];
      if (t_collision[t] == 0 && dim == 2)
        for_each_work_item(dim, s, nthreads,
                           [&] { update_d2q5_bgk(s, even, om, g, C, vel, flags); });
      else if (t_collision[t] == 0)
        for_each_work_item(dim, s, nthreads,
                           [&] { update_d3q7_bgk(s, even, om, g, C, vel, flags); });
      else if (dim == 2)
        for_each_work_item(dim, s, nthreads,
                           [&] { update_d2q5_trt(s, even, om, om_n, g, C, vel, flags); });
      else
        for_each_work_item(dim, s, nthreads,
                           [&] { update_d3q7_trt(s, even, om, om_n, g, C, vel, flags); });
    }
  }
  return 0;
}

}  // extern "C"
