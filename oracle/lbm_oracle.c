/*
 * TEST INFRASTRUCTURE: the CPU oracle (checker) for the CUDA lattice-Boltzmann path.
 * Nothing in the product links or calls this file; tests, smoke() and the bench's CPU
 * baseline leg use it only to check or to time against.
 *
 * A table-driven C restatement of the reference's hot path (djbarker/boltzmann):
 *   - equilibrium initialisation, src/velocities.rs:43-52 (FP32, same operation order);
 *   - the AA-pattern fused stream+collide kernels of src/lib.cl (D2Q9/D3Q27 BGK, D2Q9 TRT,
 *     D2Q5/D3Q7 advection-diffusion) and the D3Q27 TRT and D2Q5/D3Q7 TRT kernels its generator
 *     python/boltzmann/kernel_gen.py:250-462 writes, as one generic routine over a velocity set;
 *   - the constant and Boussinesq acceleration passes, src/lib.cl:14-44 and 60-92;
 *   - the host step loop, src/simulation.rs:278-446.
 *
 * Two precisions are built from lbm_oracle_impl.h:
 *   _f32: fields stored as float, moments in float and the collision evaluated in double and
 *         rounded on store -- the pattern the reference's double literals produce
 *         (e.g. src/lib.cl:266-274);
 *   _f64: every field and every operation in double (the FP64 oracle).
 *
 * Pinned against the reference's own kernels (oracle/_ref) by tests/golden fixtures.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <string.h>

#include <omp.h>

/* A velocity set: directions c_i and exact rational weights w_i, in the reference's slot order
 * (src/velocities.rs:66-191; the same order as src/lib.cl:195-196, 411-417). */
typedef struct {
  int d, q;
  int c[27][3];
  int w_num[27], w_den[27];
  int opp[27];
} vset;

static vset make_vset(int d, int q, const int* dirs, const int* wn, const int* wd) {
  /* dirs: q rows of d components in {-1, 0, 1} */
  vset v;
  memset(&v, 0, sizeof v);
  v.d = d;
  v.q = q;
  for (int i = 0; i < q; ++i) {
    for (int k = 0; k < d; ++k) v.c[i][k] = dirs[i * d + k];
    v.w_num[i] = wn[i];
    v.w_den[i] = wd[i];
  }
  for (int i = 0; i < q; ++i)
    for (int j = 0; j < q; ++j) {
      int match = 1;
      for (int k = 0; k < d; ++k) match &= v.c[j][k] == -v.c[i][k];
      if (match) v.opp[i] = j;
    }
  return v;
}

static int lookup_vset(int d, int q, vset* out) {
  /* src/velocities.rs:55-64 */
  if (d == 1 && q == 3) {
    static const int c[3] = {0, 1, -1};
    static const int n[3] = {4, 1, 1}, m[3] = {6, 6, 6};
    *out = make_vset(1, 3, c, n, m);
  } else if (d == 2 && q == 9) {
    static const int c[18] = {0, 0, 1, 0, -1, 0, 0, 1, 0, -1, 1, 1, -1, -1, 1, -1, -1, 1};
    static const int n[9] = {4, 1, 1, 1, 1, 1, 1, 1, 1}, m[9] = {9, 9, 9, 9, 9, 36, 36, 36, 36};
    *out = make_vset(2, 9, c, n, m);
  } else if (d == 2 && q == 5) {
    static const int c[10] = {0, 0, 1, 0, -1, 0, 0, 1, 0, -1};
    static const int n[5] = {1, 1, 1, 1, 1}, m[5] = {3, 6, 6, 6, 6};
    *out = make_vset(2, 5, c, n, m);
  } else if (d == 3 && q == 7) {
    static const int c[21] = {0, 0, 0, 1, 0, 0, -1, 0, 0, 0, 1, 0, 0, -1, 0, 0, 0, 1, 0, 0, -1};
    static const int n[7] = {1, 19, 19, 19, 19, 19, 19}, m[7] = {20, 120, 120, 120, 120, 120, 120};
    *out = make_vset(3, 7, c, n, m);
  } else if (d == 3 && q == 27) {
    static const int c[81] = {
        0,  0,  0,  1,  0,  0,  -1, 0,  0,  0,  1,  0,  0,  -1, 0,  0,  0,  1,  0,  0,  -1,
        1,  1,  0,  -1, -1, 0,  1,  -1, 0,  -1, 1,  0,  1,  0,  1,  -1, 0,  -1, 0,  1,  1,
        0,  -1, -1, 1,  0,  -1, -1, 0,  1,  0,  1,  -1, 0,  -1, 1,  1,  1,  1,  -1, -1, -1,
        1,  -1, 1,  -1, 1,  -1, 1,  1,  -1, -1, -1, 1,  1,  -1, -1, -1, 1,  1};
    static const int n[27] = {8, 2, 2, 2, 2, 2, 2, 1, 1, 1, 1, 1, 1, 1,
                              1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1};
    static const int m[27] = {27, 27, 27, 27, 27, 27, 27, 54,  54,  54,  54,  54,  54, 54,
                              54, 54, 54, 54, 54, 216, 216, 216, 216, 216, 216, 216, 216};
    *out = make_vset(3, 27, c, n, m);
  } else {
    return 1;
  }
  return 0;
}

static __thread const char* g_err = "";

const char* lbm_oracle_last_error(void) { return g_err; }

/* Exported for the tests: the velocity table the oracle uses. */
int lbm_oracle_velocity_set(int d, int q, int32_t* c_out, int32_t* w_num, int32_t* w_den,
                            int32_t* opp) {
  vset v;
  if (lookup_vset(d, q, &v)) return 1;
  for (int i = 0; i < q; ++i) {
    for (int k = 0; k < d; ++k) c_out[i * d + k] = v.c[i][k];
    w_num[i] = v.w_num[i];
    w_den[i] = v.w_den[i];
    opp[i] = v.opp[i];
  }
  return 0;
}

/* Equilibrium for one velocity set over n cells, FP32 in the operation order of
 * src/velocities.rs:43-52 (ndarray's dot is a plain running sum for these lengths):
 *   out = (rho * w) * (((1 + 3 vq) + (4.5 vq) vq) - 1.5 vv). */
int lbm_oracle_equilibrate_f32(int d, int q, int64_t n, const float* rho, const float* vel,
                               float* out) {
  vset v;
  if (lookup_vset(d, q, &v)) {
    g_err = "Unknown model";
    return 1;
  }
  float w[27];
  for (int i = 0; i < q; ++i) w[i] = (float)v.w_num[i] / (float)v.w_den[i];
#pragma omp parallel for schedule(static)
  for (int64_t cell = 0; cell < n; ++cell) {
    const float* u = vel + cell * d;
    float vv = 0.0f;
    for (int k = 0; k < d; ++k) vv = vv + u[k] * u[k];
    for (int i = 0; i < q; ++i) {
      float vq = 0.0f;
      for (int k = 0; k < d; ++k) vq = vq + u[k] * (float)v.c[i][k];
      float poly = 1.0f + 3.0f * vq;
      poly = poly + 4.5f * vq * vq;
      poly = poly - 1.5f * vv;
      out[cell * q + i] = rho[cell] * w[i] * poly;
    }
  }
  return 0;
}

/* Same in double (the FP64 oracle's initial state). */
int lbm_oracle_equilibrate_f64(int d, int q, int64_t n, const double* rho, const double* vel,
                               double* out) {
  vset v;
  if (lookup_vset(d, q, &v)) {
    g_err = "Unknown model";
    return 1;
  }
#pragma omp parallel for schedule(static)
  for (int64_t cell = 0; cell < n; ++cell) {
    const double* u = vel + cell * d;
    double vv = 0.0;
    for (int k = 0; k < d; ++k) vv += u[k] * u[k];
    for (int i = 0; i < q; ++i) {
      double vq = 0.0;
      for (int k = 0; k < d; ++k) vq += u[k] * v.c[i][k];
      double w = (double)v.w_num[i] / (double)v.w_den[i];
      out[cell * q + i] = rho[cell] * w * (1.0 + 3.0 * vq + 4.5 * vq * vq - 1.5 * vv);
    }
  }
  return 0;
}

#define REAL float
#define FN(name) name##_f32
#include "lbm_oracle_impl.h"
#undef REAL
#undef FN

#define REAL double
#define FN(name) name##_f64
#include "lbm_oracle_impl.h"
#undef REAL
#undef FN
