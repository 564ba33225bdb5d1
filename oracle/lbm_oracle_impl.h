/*
 * TEST INFRASTRUCTURE: body of the CPU oracle, included by lbm_oracle.c once per precision
 * with REAL (storage and moment type) and FN(name) (symbol suffix) defined.
 * The collision is evaluated in double for both precisions.
 */

typedef struct {
  int dim;
  long n[3]; /* counts, padded with 1 up to 3 axes */
  const int32_t* flags;
  vset lat;
  double w[27];
} FN(grid_t);

/* Cell index of coords (x, y, z) minus direction c with periodic wrap (src/lib.cl:218-223). */
static inline long FN(upstream)(const FN(grid_t) * g, long x, long y, long z, const int* c) {
  long xs = x - c[0], ys = y - c[1], zs = z - c[2];
  if (xs < 0) xs += g->n[0];
  if (xs >= g->n[0]) xs -= g->n[0];
  if (ys < 0) ys += g->n[1];
  if (ys >= g->n[1]) ys -= g->n[1];
  if (zs < 0) zs += g->n[2];
  if (zs >= g->n[2]) zs -= g->n[2];
  return (xs * g->n[1] + ys) * g->n[2] + zs;
}

/* AA-pattern load (src/lib.cl:225-246): even steps pull slot i from the cell upstream of c_i,
 * odd steps read slot opp(i) of this cell. Returns the slot addresses for the matching store. */
static inline void FN(aa_load)(const FN(grid_t) * g, const REAL* f, long cell, long x, long y,
                               long z, int even, REAL* fl, long* at) {
  const int q = g->lat.q;
  for (int i = 0; i < q; ++i) {
    at[i] = even ? FN(upstream)(g, x, y, z, g->lat.c[i]) * q + i : cell * q + g->lat.opp[i];
    fl[i] = f[at[i]];
  }
}

/* AA-pattern store (src/lib.cl:276-296): even steps write post-collision f_opp(i) into slot i
 * upstream of c_i (the slot that was read); odd steps write f_i into slot i of this cell. */
static inline void FN(aa_store)(const FN(grid_t) * g, REAL* f, long cell, int even,
                                const REAL* fl, const long* at) {
  const int q = g->lat.q;
  for (int i = 0; i < q; ++i) {
    if (even)
      f[at[i]] = fl[g->lat.opp[i]];
    else
      f[cell * q + i] = fl[i];
  }
}

static inline double FN(feq)(const FN(grid_t) * g, int i, double r, const double* v, double vv) {
  double cu = 0.0;
  for (int k = 0; k < g->dim; ++k) cu += g->lat.c[i][k] * v[k];
  return r * g->w[i] * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * vv);
}

typedef struct {
  FN(grid_t) g;
  int trt;
  REAL om_pos, om_neg;
  REAL *f, *rho, *vel;
  const REAL* acc;
  int use_acc;
} FN(fluid_t);

/* One fluid cell: src/lib.cl:191-301 (D2Q9 BGK), 407-618 (D3Q27 BGK), 620-748 (D2Q9 TRT),
 * kernel_gen.py:385-420 (TRT for any velocity set). */
static void FN(fluid_cell)(const FN(fluid_t) * a, long x, long y, long z, int even) {
  const FN(grid_t)* g = &a->g;
  const int q = g->lat.q, d = g->dim;
  const long cell = (x * g->n[1] + y) * g->n[2] + z;
  const int32_t flag = g->flags[cell];
  if (flag & 1) return;               /* wall: never updated (src/lib.cl:207-213) */
  const int fixed = (flag & 6) != 0; /* FIXED_FLUID_VELOCITY | FIXED_FLUID_DENSITY (208) */

  REAL fl[27];
  long at[27];
  FN(aa_load)(g, a->f, cell, x, y, z, even, fl, at);

  /* moments (src/lib.cl:249-251) */
  REAL r = 0, m[3] = {0, 0, 0}, v[3] = {0, 0, 0};
  for (int i = 0; i < q; ++i) r += fl[i];
  for (int i = 0; i < q; ++i)
    for (int k = 0; k < d; ++k) {
      if (g->lat.c[i][k] > 0) m[k] += fl[i];
      if (g->lat.c[i][k] < 0) m[k] -= fl[i];
    }
  for (int k = 0; k < d; ++k) v[k] = m[k] / r;

  REAL om_p = a->om_pos, om_n = a->om_neg;
  /* force: velocity shift by acc / omega (TRT: omega+) (src/lib.cl:253-256, 682-685) */
  if (a->use_acc)
    for (int k = 0; k < d; ++k) v[k] += a->acc[cell * d + k] / om_p;
  if (fixed) { /* src/lib.cl:257-262, 687-693 */
    om_p = 1;
    om_n = 1;
    r = a->rho[cell];
    for (int k = 0; k < d; ++k) v[k] = a->vel[cell * d + k];
  }
  REAL vv = 0;
  for (int k = 0; k < d; ++k) vv += v[k] * v[k];

  const double rd = r, vvd = vv, vd[3] = {v[0], v[1], v[2]};
  if (!a->trt) {
    /* BGK: f_i += omega (feq_i - f_i) (src/lib.cl:266-274) */
    for (int i = 0; i < q; ++i)
      fl[i] = (REAL)((double)fl[i] + (double)om_p * (FN(feq)(g, i, rd, vd, vvd) - (double)fl[i]));
  } else {
    /* TRT over the pairs (i, opp i) (src/lib.cl:697-719). The rest direction has no odd part. */
    for (int i = 0; i < q; ++i) {
      const int j = g->lat.opp[i];
      if (j < i) continue;
      const double fe_i = FN(feq)(g, i, rd, vd, vvd), fe_j = FN(feq)(g, j, rd, vd, vvd);
      const double sym = (double)(REAL)(fl[i] + fl[j]) * 0.5;
      const double asym = (double)(REAL)(fl[i] - fl[j]) * 0.5;
      const double fpos = (double)om_p * ((fe_i + fe_j) * 0.5 - sym);
      const double fneg = (double)om_n * ((fe_i - fe_j) * 0.5 - asym);
      fl[i] = (REAL)((double)fl[i] + (fpos + fneg));
      if (j != i) fl[j] = (REAL)((double)fl[j] + (fpos - fneg));
    }
  }

  FN(aa_store)(g, a->f, cell, even, fl, at);
  a->rho[cell] = r; /* src/lib.cl:298-300 */
  for (int k = 0; k < d; ++k) a->vel[cell * d + k] = v[k];
}

typedef struct {
  FN(grid_t) g;
  int trt;
  REAL om, om_neg; /* omega (BGK) or omega+, omega- (TRT) */
  REAL *f, *val;
  const REAL* vel; /* the fluid velocity written this step */
} FN(tracer_t);

/* One tracer cell: src/lib.cl:102-189 (D2Q5 BGK), 303-405 (D3Q7 BGK); TRT as the reference's
 * generator writes it for a scalar (python/boltzmann/kernel_gen.py:368-421: the fixed-value
 * override sets both rates to 1, then the pair update of the fluid's TRT). */
static void FN(tracer_cell)(const FN(tracer_t) * a, long x, long y, long z, int even) {
  const FN(grid_t)* g = &a->g;
  const int q = g->lat.q, d = g->dim;
  const long cell = (x * g->n[1] + y) * g->n[2] + z;
  const int32_t flag = g->flags[cell];
  if (flag & 1) return;               /* wall (src/lib.cl:116-122) */
  const int fixed = (flag & 8) != 0; /* FIXED_SCALAR_VALUE (117) */

  REAL fl[27];
  long at[27];
  FN(aa_load)(g, a->f, cell, x, y, z, even, fl, at);

  REAL r = 0, v[3] = {0, 0, 0};
  for (int i = 0; i < q; ++i) r += fl[i];
  for (int k = 0; k < d; ++k) v[k] = a->vel[cell * d + k];
  REAL om = a->om, om_n = a->om_neg;
  if (fixed) { /* src/lib.cl:156-161 */
    om = 1;
    om_n = 1;
    r = a->val[cell];
  }
  REAL vv = 0;
  for (int k = 0; k < d; ++k) vv += v[k] * v[k];
  const double rd = r, vvd = vv, vd[3] = {v[0], v[1], v[2]};
  if (!a->trt) {
    for (int i = 0; i < q; ++i)
      fl[i] = (REAL)((double)fl[i] + (double)om * (FN(feq)(g, i, rd, vd, vvd) - (double)fl[i]));
  } else {
    for (int i = 0; i < q; ++i) {
      const int j = g->lat.opp[i];
      if (j < i) continue;
      const double fe_i = FN(feq)(g, i, rd, vd, vvd), fe_j = FN(feq)(g, j, rd, vd, vvd);
      const double sym = (double)(REAL)(fl[i] + fl[j]) * 0.5;
      const double asym = (double)(REAL)(fl[i] - fl[j]) * 0.5;
      const double fpos = (double)om * ((fe_i + fe_j) * 0.5 - sym);
      const double fneg = (double)om_n * ((fe_i - fe_j) * 0.5 - asym);
      fl[i] = (REAL)((double)fl[i] + (fpos + fneg));
      if (j != i) fl[j] = (REAL)((double)fl[j] + (fpos - fneg));
    }
  }

  FN(aa_store)(g, a->f, cell, even, fl, at);
  a->val[cell] = r; /* src/lib.cl:188 */
}

static int FN(make_grid)(FN(grid_t) * g, int dim, const int64_t* counts, const int32_t* flags,
                         int q) {
  memset(g, 0, sizeof *g);
  g->dim = dim;
  for (int k = 0; k < 3; ++k) g->n[k] = k < dim ? (long)counts[k] : 1;
  g->flags = flags;
  if (lookup_vset(dim, q, &g->lat)) return 1;
  for (int i = 0; i < q; ++i) g->w[i] = (double)g->lat.w_num[i] / (double)g->lat.w_den[i];
  return 0;
}

/* Simulation::iterate after the upload (src/simulation.rs:278-446). Same argument list as
 * lbm_ref_iterate in oracle/ref_driver.cpp, with fields of type REAL. */
int FN(lbm_oracle_iterate)(int dim, const int64_t* counts, const int32_t* flags, int q,
                           int collision, REAL om_pos, REAL om_neg, REAL* f, REAL* rho, REAL* vel,
                           REAL* acc, int use_acc, const REAL* gravity, int ncouplings,
                           const int32_t* c_tracer, const REAL* c_alpha, const REAL* c_c0,
                           const REAL* c_g, int ntracers, const int32_t* t_q,
                           const int32_t* t_collision, const REAL* t_om,
                           const REAL* t_om_neg, REAL* const* t_g, REAL* const* t_C,
                           int64_t iters, int nthreads) {
  if (iters % 2 != 0) { /* src/simulation.rs:279-281 */
    g_err = "iters must be even";
    return 1;
  }
  if (nthreads <= 0) nthreads = omp_get_max_threads();
  const int fluid_ok = (dim == 2 && q == 9) || (dim == 3 && q == 27);
  if (!fluid_ok) {
    g_err = "Kernel not found (fluid)";
    return 1;
  }
  FN(fluid_t) fa;
  FN(make_grid)(&fa.g, dim, counts, flags, q);
  fa.trt = collision == 1;
  fa.om_pos = om_pos;
  fa.om_neg = om_neg;
  fa.f = f;
  fa.rho = rho;
  fa.vel = vel;
  fa.acc = acc;
  fa.use_acc = use_acc;

  FN(tracer_t) ta[8];
  if (ntracers > 8) {
    g_err = "too many tracers";
    return 1;
  }
  for (int t = 0; t < ntracers; ++t) {
    const int ok = (t_collision[t] == 0 || t_collision[t] == 1) &&
                   ((dim == 2 && t_q[t] == 5) || (dim == 3 && t_q[t] == 7));
    if (!ok) {
      g_err = "Kernel not found (tracer)";
      return 1;
    }
    FN(make_grid)(&ta[t].g, dim, counts, flags, t_q[t]);
    ta[t].trt = t_collision[t] == 1;
    ta[t].om = t_om[t];
    ta[t].om_neg = t_om_neg[t];
    ta[t].f = t_g[t];
    ta[t].val = t_C[t];
    ta[t].vel = vel;
  }
  const FN(grid_t)* G = &fa.g;
  const long N = G->n[0] * G->n[1] * G->n[2];

  /* constant acceleration once per call (src/simulation.rs:326-342, src/lib.cl:14-44) */
  if (gravity) {
    if (!use_acc) {
      g_err = "gravity without an acceleration buffer";
      return 1;
    }
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (long c = 0; c < N; ++c)
      for (int k = 0; k < dim; ++k) acc[c * dim + k] = gravity[k];
  }

  for (int64_t it = 0; it < iters; ++it) {
    const int even = (int)(1 - it % 2); /* src/simulation.rs:350 */
    /* Boussinesq sources in coupling order; the last one wins (src/simulation.rs:352-373,
     * src/lib.cl:60-92) */
    for (int k = 0; k < ncouplings; ++k) {
      const REAL* conc = t_C[c_tracer[k]];
      const REAL alpha = c_alpha[k], c0 = c_c0[k];
      const REAL* gk = c_g + (long)k * dim;
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (long c = 0; c < N; ++c) {
        const REAL b = alpha * (conc[c] - c0);
        for (int a = 0; a < dim; ++a) acc[c * dim + a] = gk[a] * b;
      }
    }
#pragma omp parallel for schedule(static) num_threads(nthreads)
    for (long x = 0; x < G->n[0]; ++x)
      for (long y = 0; y < G->n[1]; ++y)
        for (long z = 0; z < G->n[2]; ++z) FN(fluid_cell)(&fa, x, y, z, even);
    for (int t = 0; t < ntracers; ++t) {
      const FN(tracer_t)* tp = &ta[t];
#pragma omp parallel for schedule(static) num_threads(nthreads)
      for (long x = 0; x < G->n[0]; ++x)
        for (long y = 0; y < G->n[1]; ++y)
          for (long z = 0; z < G->n[2]; ++z) FN(tracer_cell)(tp, x, y, z, even);
    }
  }
  return 0;
}
