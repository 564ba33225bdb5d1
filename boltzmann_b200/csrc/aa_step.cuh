// The AA-pattern in-place fused stream+collide kernel family.
//
// One kernel template covers the reference's update kernels (djbarker/boltzmann src/lib.cl:
// update_d2q9_bgk 191-301, update_d2q9_trt 620-748, update_d3q27_bgk 407-618, and the D3Q27 TRT
// kernel that python/boltzmann/kernel_gen.py:250-462 generates), fused with
//   - the advection-diffusion tracer kernels (update_d2q5_bgk 102-189, update_d3q7_bgk 303-405):
//     each tracer reads the fluid velocity this thread has just computed, so the fluid velocity
//     never goes through HBM between the two;
//   - the acceleration passes (set_constant_acc 14-44, set_boussinesq_acc 60-92): the constant
//     acceleration is a kernel argument and the Boussinesq acceleration is computed in registers
//     from the coupled tracer's value of the previous step.
//
// Memory layout in HBM (N = cell count, cell = (x*ny + y)*nz + z, the reference's row-major
// index, x slowest):
//   populations  f[i*N + cell]  structure-of-arrays, slot order of the reference;
//   flags        u8[N]          the low four CellFlags bits;
//   rho, vel     [N], [N][D]    the reference's host layout (only written on the step that ends
//                               an iterate call; fixed cells only read them);
//   tracers      g[i*N + cell], val[N].
// Consecutive threads own consecutive cells along the contiguous axis, so every population
// access of a warp is one contiguous run (shifted by at most one cell on even steps).
//
// AA semantics (src/lib.cl:225-246, 276-296): an even step reads slot i of the cell upstream of
// c_i and writes the post-collision f_opp(i) back into that same slot; an odd step reads slot
// opp(i) of its own cell and writes f_i into slot i. Every slot is read and written by exactly
// one thread per step, so the update is in place and race-free.
#pragma once

#include <cstdint>

#include "lattice.cuh"
#include "storage.cuh"

namespace lbm {

constexpr int kMaxTracers = 4;

template <class Real>
struct TracerArgs {
  void* g;    // [Qt][N] in the tracer storage type (TracerPop)
  Real* val;  // [N]
  Real omega;      // omega (BGK) or omega+ (TRT)
  Real omega_neg;  // omega- (TRT)
  int trt;
};

template <class Real>
struct StepArgs {
  void* f;             // [Q][N] in the storage type
  Real* rho;           // [N]
  Real* vel;           // [N][D]
  const uint8_t* flags;
  int nx, ny, nz;      // 2D domains use nx = 1, (ny, nz) = the reference's (x, y) counts
  long long n;         // cell count
  Real om_pos, om_neg; // BGK uses om_pos
  int acc_mode;        // 0: none, 1: constant acceleration acc[], 2: Boussinesq
  Real force[3];       // velocity shift per unit buoyancy: acc / om_pos (constant acceleration,
                       // the reference's per-cell division done once) or g / om_pos (Boussinesq)
  Real alpha, c0;      // Boussinesq coupling
  int coupled;         // index of the coupled tracer
  const Real* coupled_val;  // its val[] (read for the Boussinesq term)
  int ntracers;
  TracerArgs<Real> tr[kMaxTracers];
  int write_moments;   // 1 on the last step of an iterate call
  int path;            // kernel choice: 0 automatic, 1 direct, 2 TMA-staged (when the shape allows)
  const float* omega_field;  // per-cell om_pos (a learned closure's relaxation field), or null
  int* status;         // bit 0 set when a non-finite density or velocity is produced
  unsigned spin_limit; // polls of a staged kernel's pipeline waits before it gives up (bit 1)
};

enum AccMode : int { kAccNone = 0, kAccConstant = 1, kAccBoussinesq = 2 };

// Velocity component along internal axis a (0 = x, 1 = y, 2 = z). 2D sets map the reference's
// (x, y) onto the internal (y, z).
template <class L>
__host__ __device__ constexpr int comp(int i, int a) {
  if constexpr (L::D == 3)
    return L::c(i, a);
  else
    return a == 0 ? 0 : L::c(i, a - 1);
}

// comp<L>(i, A) for a slot index known only at run time (a producer lane's job), selected from
// the compile-time entries so that the velocity table is never materialised in local memory.
template <class L, int A>
__device__ __forceinline__ int comp_rt(int i) {
  int v = 0;
#pragma unroll
  for (int k = 0; k < L::Q; ++k)
    if (k == i) v = comp<L>(k, A);
  return v;
}

// Upstream coordinate along one axis for a velocity component cc (coordinate - cc, wrapped).
__device__ __forceinline__ int upstream_coord(int cc, int minus1, int same, int plus1) {
  return cc > 0 ? minus1 : (cc < 0 ? plus1 : same);
}

// A cell and its periodic neighbourhood as 32-bit element offsets per axis:
//   ox = {x-1, x, x+1} * ny * nz,  oy = {y-1, y, y+1} * nz,  oz = {z-1, z, z+1} (wrapped),
// so the cell upstream of c_i is ox[.] + oy[.] + oz[.] (one three-input add) and every access is
// a uniform per-direction base pointer plus a 32-bit offset. Cell counts stay below 2^32.
struct CellPos {
  unsigned cell;
  unsigned ox[3], oy[3], oz[3];

  template <class L>
  __device__ __forceinline__ unsigned upstream(int i) const {
    // index 0: coordinate - 1 (component +1), 1: same, 2: coordinate + 1 (component -1)
    return ox[1 - comp<L>(i, 0)] + oy[1 - comp<L>(i, 1)] + oz[1 - comp<L>(i, 2)];
  }
};

// AA load of one velocity set's populations for this cell: deviations d_i = f_i - W_i when DEV,
// full values otherwise.
template <class L, class P, bool EVEN, bool DEV>
__device__ __forceinline__ void aa_load(const typename P::type* __restrict__ f, long long n,
                                        const CellPos& c, typename P::real (&v)[L::Q]) {
  using Real = typename P::real;
#pragma unroll
  for (int i = 0; i < L::Q; ++i) {
    const typename P::type* p =
        EVEN ? (f + (size_t)i * n) + c.upstream<L>(i) : (f + (size_t)opp(i) * n) + c.cell;
    // Slot i (even) and slot opp(i) (odd) share the weight of direction i.
    if constexpr (DEV)
      v[i] = P::load_dev(p, weight<L, Real>(i));
    else
      v[i] = P::load(p, weight<L, Real>(i));
  }
}

// AA store matching aa_load.
template <class L, class P, bool EVEN, bool DEV>
__device__ __forceinline__ void aa_store(typename P::type* __restrict__ f, long long n,
                                         const CellPos& c, const typename P::real (&v)[L::Q]) {
  using Real = typename P::real;
#pragma unroll
  for (int i = 0; i < L::Q; ++i) {
    typename P::type* p = (f + (size_t)i * n) + (EVEN ? c.upstream<L>(i) : c.cell);
    const Real val = EVEN ? v[opp(i)] : v[i];
    if constexpr (DEV)
      P::store_dev(p, val, weight<L, Real>(i));
    else
      P::store(p, val, weight<L, Real>(i));
  }
}

// Where update_cell puts the post-collision populations: the AA store straight to HBM. (The
// TMA kernel passes a sink that writes them into its shared-memory stage instead, from where whole
// row segments go back with bulk copies.)
struct GlobalSink {
  template <class L, class P, bool EVEN, bool DEV>
  __device__ __forceinline__ void fluid(typename P::type* f, long long n, const CellPos& c,
                                        const typename P::real (&v)[L::Q]) const {
    aa_store<L, P, EVEN, DEV>(f, n, c, v);
  }
  template <class TL, class TP, bool EVEN>
  __device__ __forceinline__ void tracer(typename TP::type* g, long long n, const CellPos& c,
                                         const typename TP::real (&v)[TL::Q]) const {
    aa_store<TL, TP, EVEN, false>(g, n, c, v);
  }
};

// BGK or TRT collision against the second-order equilibrium
//   feq_i = w_i r (1 + 3 c_i.u + 4.5 (c_i.u)^2 - 1.5 u.u),
// evaluated per opposite pair (i, i+1) as feq = A +- B (symmetric and antisymmetric parts).
// TRT relaxes the symmetric part with om_pos and the antisymmetric part with om_neg
// (src/lib.cl:697-719); BGK relaxes both with om_pos (src/lib.cl:266-274).
//
// DEV: v holds deviations d_i = f_i - W_i and dr = r - 1, and the equilibrium is formed as
// the deviation e_i = feq_i - W_i = w_i r X_i + (w_i dr + (w_i - W_i)),
// X_i = 3cu + 4.5cu^2 - 1.5uu. Every term is small, so the stored f_i = W_i + d_i carries about
// one rounding, like the reference's double-precision update. The constant w_i - W_i (below one
// ulp of e_i) is added to the small w_i dr term first: added last it would be rounded away in
// the same direction every step, a mass drift of ~4e-9 per cell and step.
// Otherwise v holds full values (the tracers, whose concentration is not near a fixed offset).
// The weights enter as exact integers k_i times r / kDen (one unbiased rounding per cell):
// float-rounded weights do not sum to one (D2Q9: 1 + 7.5e-9), which would otherwise add a
// systematic mass and momentum drift of that size per step.
template <class L, bool TRT, bool DEV, class Real>
__device__ __forceinline__ void collide(Real (&v)[L::Q], Real r, Real dr, const Real (&u)[3],
                                        Real uu, Real om_pos, Real om_neg) {
  const Real ru = over_den<L>(r);
  const Real unit = DEV ? over_den<L>(dr) : ru;  // the w_i (r or dr) term per unit weight
  const Real quad = Real(-1.5) * uu;
  {
    const Real k0 = Real(L::wk(0));
    const Real e0 = k0 * ru * quad + (k0 * unit + (DEV ? weight_gap<L, Real>(0) : Real(0)));
    v[0] += om_pos * (e0 - v[0]);
  }
#pragma unroll
  for (int i = 1; i < L::Q; i += 2) {
    Real cu = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (comp<L>(i, a) > 0) cu += u[a];
      if (comp<L>(i, a) < 0) cu -= u[a];
    }
    const Real k = Real(L::wk(i));
    const Real A =
        k * ru * (quad + Real(4.5) * cu * cu) + (k * unit + (DEV ? weight_gap<L, Real>(i) : Real(0)));
    const Real B = k * ru * Real(3) * cu;
    if constexpr (TRT) {
      const Real s = Real(0.5) * (v[i] + v[i + 1]);
      const Real d = Real(0.5) * (v[i] - v[i + 1]);
      const Real fp = om_pos * (A - s);
      const Real fn = om_neg * (B - d);
      v[i] += fp + fn;
      v[i + 1] += fp - fn;
    } else {
      v[i] += om_pos * (A + B - v[i]);
      v[i + 1] += om_pos * (A - B - v[i + 1]);
    }
  }
}

// Fused multiply-add in the compute precision, written out so that the operation sequence of the
// FP32 cell update is fixed in the source (the two-cells-a-thread path repeats it lane for lane
// on packed instructions and must round identically).
__device__ __forceinline__ float fma_r(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_r(double a, double b, double c) { return fma(a, b, c); }
// A product and a sum that are never contracted into a fused multiply-add.
__device__ __forceinline__ float mul_r(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_r(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float add_r(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double add_r(double a, double b) { return __dadd_rn(a, b); }

// ---- Packed FP32 (Blackwell FADD2 / FMUL2 / FFMA2): two independent FP32 operations per
// instruction, each lane rounded exactly as the scalar operation (round to nearest even).
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
  return __fadd2_rn(a, make_float2(-b.x, -b.y));
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 splat(float s) { return make_float2(s, s); }

// c_i . u for direction i (components in {-1, 0, 1}).
template <class L, class Real>
__device__ __forceinline__ Real c_dot(int i, const Real (&u)[3]) {
  Real cu = 0;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (comp<L>(i, a) > 0) cu += u[a];
    if (comp<L>(i, a) < 0) cu -= u[a];
  }
  return cu;
}

// The collision of `collide` for FP32, with the opposite pairs (2p+1, 2p+2) and (2p+3, 2p+4)
// processed together on packed instructions: lane x holds pair p, lane y pair p+1, and every
// lane performs the scalar version's operations in the same order (same roundings). A last
// unpaired pair (D3Q27 has 13, D3Q7 3) runs on scalar instructions.
template <class L, bool TRT, bool DEV>
__device__ __forceinline__ void collide_packed(float (&v)[L::Q], float r, float dr,
                                               const float (&u)[3], float uu, float om_pos,
                                               float om_neg) {
  constexpr int P = (L::Q - 1) / 2;
  const float ru = over_den<L>(r);
  const float unit = DEV ? over_den<L>(dr) : ru;
  const float quad = __fmul_rn(-1.5f, uu);
  {
    const float k0 = float(L::wk(0));
    const float e0 = __fmaf_rn(__fmul_rn(k0, ru), quad,
                               __fmaf_rn(k0, unit, DEV ? weight_gap<L, float>(0) : 0.0f));
    v[0] = __fmaf_rn(om_pos, __fsub_rn(e0, v[0]), v[0]);
  }
#pragma unroll
  for (int p = 0; p + 1 < P; p += 2) {
    const int i = 2 * p + 1, j = 2 * p + 3;
    const float ki = float(L::wk(i)), kj = float(L::wk(j));
    const float2 cu = make_float2(c_dot<L>(i, u), c_dot<L>(j, u));
    const float2 kru = make_float2(__fmul_rn(ki, ru), __fmul_rn(kj, ru));
    const float2 ku = make_float2(__fmaf_rn(ki, unit, DEV ? weight_gap<L, float>(i) : 0.0f),
                                  __fmaf_rn(kj, unit, DEV ? weight_gap<L, float>(j) : 0.0f));
    const float2 X = fma2(mul2(splat(4.5f), cu), cu, splat(quad));
    const float2 A = fma2(kru, X, ku);
    const float2 B = mul2(mul2(kru, splat(3.0f)), cu);
    float2 F = make_float2(v[i], v[j]), G = make_float2(v[i + 1], v[j + 1]);
    if constexpr (TRT) {
      const float2 S = mul2(splat(0.5f), add2(F, G));
      const float2 D = mul2(splat(0.5f), sub2(F, G));
      const float2 fp = mul2(splat(om_pos), sub2(A, S));
      const float2 fn = mul2(splat(om_neg), sub2(B, D));
      F = add2(F, add2(fp, fn));
      G = add2(G, sub2(fp, fn));
    } else {
      F = fma2(splat(om_pos), sub2(add2(A, B), F), F);
      G = fma2(splat(om_pos), sub2(sub2(A, B), G), G);
    }
    v[i] = F.x;
    v[j] = F.y;
    v[i + 1] = G.x;
    v[j + 1] = G.y;
  }
  if constexpr (P % 2 == 1) {
    constexpr int i = 2 * (P - 1) + 1;
    const float cu = c_dot<L>(i, u);
    const float k = float(L::wk(i));
    const float kr = __fmul_rn(k, ru);
    const float X = __fmaf_rn(__fmul_rn(4.5f, cu), cu, quad);
    const float A = __fmaf_rn(kr, X, __fmaf_rn(k, unit, DEV ? weight_gap<L, float>(i) : 0.0f));
    const float B = __fmul_rn(__fmul_rn(kr, 3.0f), cu);
    if constexpr (TRT) {
      const float sp = __fmul_rn(0.5f, __fadd_rn(v[i], v[i + 1]));
      const float dp = __fmul_rn(0.5f, __fsub_rn(v[i], v[i + 1]));
      const float fp = __fmul_rn(om_pos, __fsub_rn(A, sp));
      const float fn = __fmul_rn(om_neg, __fsub_rn(B, dp));
      v[i] = __fadd_rn(v[i], __fadd_rn(fp, fn));
      v[i + 1] = __fadd_rn(v[i + 1], __fsub_rn(fp, fn));
    } else {
      v[i] = __fmaf_rn(om_pos, __fsub_rn(__fadd_rn(A, B), v[i]), v[i]);
      v[i + 1] = __fmaf_rn(om_pos, __fsub_rn(__fsub_rn(A, B), v[i + 1]), v[i + 1]);
    }
  }
}

// Whether the FP32 collision of lattice L (fluid or tracer) runs on packed pairs, with storage
// kind K of the fluid: D3Q27 (13 pairs, +5% MLUPS on the 256^3 Taylor-Green run), and every
// lattice of a simulation with 16-bit populations, whose staged kernels update two cells a
// thread and must round as this one-cell path does (aa_pair.cuh). With FP32 storage the packed
// and scalar D2Q9 / tracer collisions measured within 2% of each other.
template <class L, int K>
__host__ __device__ constexpr bool pack_collide() {
  return L::Q >= 27 || dev_in<K>();
}

// Moments of one cell for FP32. In: v full values (or deviations when DL). Out: v deviations,
// dr = r - 1 = sum of deviations + (sum of the offsets - 1), and the momentum from the pair
// differences f_i - f_opp(i): for full values within a factor two of each other that
// difference is exact (Sterbenz), so the momentum carries only the rounding of its own sum.
template <class L, bool DL>
__device__ __forceinline__ void moments_packed(float (&v)[L::Q], float& dr, float (&m)[3]) {
  constexpr int P = (L::Q - 1) / 2;
  float del[P];
  float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int p = 0; p + 1 < P; p += 2) {
    const int i = 2 * p + 1, j = 2 * p + 3;
    float2 F = make_float2(v[i], v[j]), G = make_float2(v[i + 1], v[j + 1]);
    const float2 D = sub2(F, G);
    del[p] = D.x;
    del[p + 1] = D.y;
    if constexpr (!DL) {
      const float2 W = make_float2(weight<L, float>(i), weight<L, float>(j));
      F = sub2(F, W);
      G = sub2(G, W);
      v[i] = F.x;
      v[j] = F.y;
      v[i + 1] = G.x;
      v[j + 1] = G.y;
    }
    acc = add2(acc, add2(F, G));
  }
  float sig_last = 0.0f;
  if constexpr (P % 2 == 1) {
    constexpr int i = 2 * (P - 1) + 1;
    del[P - 1] = v[i] - v[i + 1];
    if constexpr (!DL) {
      v[i] -= weight<L, float>(i);
      v[i + 1] -= weight<L, float>(i);
    }
    sig_last = v[i] + v[i + 1];
  }
  if constexpr (!DL) v[0] -= weight<L, float>(0);
  dr = v[0] + (acc.x + acc.y) + sig_last + weight_defect<L, float>();
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) m[ax] = 0.0f;
#pragma unroll
  for (int p = 0; p < P; ++p) {
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      if (comp<L>(2 * p + 1, ax) > 0) m[ax] += del[p];
      if (comp<L>(2 * p + 1, ax) < 0) m[ax] -= del[p];
    }
  }
}

// Advection-diffusion update of one tracer cell in the fluid velocity u just computed
// (src/lib.cl:102-189, 303-405), with its populations already loaded into g. TRT tracers take
// the pair update of the fluid's TRT with their own rates, both 1 on fixed-value cells (the
// D2Q5 / D3Q7 TRT kernels of python/boltzmann/kernel_gen.py:368-421).
template <class TL, class TP, bool EVEN, bool PACK, class Real, class Sink = GlobalSink>
__device__ __forceinline__ void tracer_update(const TracerArgs<Real>& tr, long long n,
                                              const CellPos& c, int flag, Real (&g)[TL::Q],
                                              const Real (&u)[3], Real uu, bool keep,
                                              const Sink& sink = Sink()) {
  Real rt = 0;
#pragma unroll
  for (int i = 0; i < TL::Q; ++i) rt += g[i];
  Real om = tr.omega, om_n = tr.omega_neg;
  const bool tfixed = (flag & 8) != 0;  // FIXED_SCALAR_VALUE (src/lib.cl:156-161)
  if (tfixed) {
    om = 1;
    om_n = 1;
    rt = tr.val[c.cell];
  }
  if constexpr (sizeof(Real) == 4 && PACK) {
    if (tr.trt)
      collide_packed<TL, true, false>(g, rt, rt, u, uu, om, om_n);
    else
      collide_packed<TL, false, false>(g, rt, rt, u, uu, om, om);
  } else {
    if (tr.trt)
      collide<TL, true, false>(g, rt, rt, u, uu, om, om_n);
    else
      collide<TL, false, false>(g, rt, rt, u, uu, om, om);
  }
  sink.template tracer<TL, TP, EVEN>(static_cast<typename TP::type*>(tr.g), n, c, g);
  if (keep && !tfixed) tr.val[c.cell] = rt;
}

template <class Real>
__device__ __forceinline__ CellPos make_cellpos(const StepArgs<Real>& a, int x, int y, int z,
                                                bool neighbours) {
  CellPos c;
  const unsigned plane = (unsigned)a.ny * (unsigned)a.nz;
  c.ox[1] = (unsigned)x * plane;
  c.oy[1] = (unsigned)y * (unsigned)a.nz;
  c.oz[1] = (unsigned)z;
  c.cell = c.ox[1] + c.oy[1] + c.oz[1];
  if (neighbours) {
    c.ox[0] = (unsigned)(x == 0 ? a.nx - 1 : x - 1) * plane;
    c.ox[2] = (unsigned)(x == a.nx - 1 ? 0 : x + 1) * plane;
    c.oy[0] = (unsigned)(y == 0 ? a.ny - 1 : y - 1) * (unsigned)a.nz;
    c.oy[2] = (unsigned)(y == a.ny - 1 ? 0 : y + 1) * (unsigned)a.nz;
    c.oz[0] = (unsigned)(z == 0 ? a.nz - 1 : z - 1);
    c.oz[2] = (unsigned)(z == a.nz - 1 ? 0 : z + 1);
  }
  return c;
}

// Everything after the loads for one cell: moments, forcing, fixed-cell override, collision,
// AA store, end-of-call moments and the fused tracers. f holds the population values of the AA
// load (full values; deviations for 16-bit storage, see dev_in), g the first tracer's
// (NT == 1), cval the coupled tracer's previous value.
// om_pos / om_neg are the relaxation rates of the cell's domain (a.om_pos / a.om_neg for a single
// simulation; per domain in an ensemble).
// KT: storage kind of the fused tracers' populations (TracerPop).
// UNFORCED: no body force, coupling or relaxation field by construction (batched ensembles), so
// their per-cell checks are left out (+5% on the FP16 ensemble kernel).
template <class L, bool TRT, int K, bool EVEN, int NT, class Sink = GlobalSink,
          int KT = default_tracer_kind<K>(), bool UNFORCED = false>
__device__ __forceinline__ void update_cell(const StepArgs<typename Pop<K>::real>& a,
                                            const CellPos& c, int flag,
                                            typename Pop<K>::real (&f)[L::Q],
                                            typename Pop<K>::real (&g)[NT == 1 ? TracerLattice<L::D>::type::Q : 1],
                                            typename Pop<K>::real cval,
                                            typename Pop<K>::real om_pos,
                                            typename Pop<K>::real om_neg,
                                            const Sink& sink = Sink()) {
  using P = Pop<K>;
  using Real = typename P::real;
  using T = typename P::type;
  using TL = typename TracerLattice<L::D>::type;
  using TP = TracerPop<KT>;
  constexpr int Q = L::Q;

  if (flag & 1) return;  // WALL: never updated (src/lib.cl:210-213)
  constexpr bool DL = dev_in<K>();  // f holds deviations already (16-bit storage)

  // Moments (src/lib.cl:249-251). The density is taken from the deviations d_i = f_i - W_i
  // (exact for values near W_i): r = 1 + (sum d_i + (sum W_i - 1)). A float sum of the full
  // values loses ~1e-7 of r per step for D3Q27 (27 terms near 1), which the collision turns into
  // density noise; the deviation sum keeps r to about one rounding. The momentum is the sum of
  // the opposite-pair differences f_i - f_opp(i) of the values as loaded (FP32: exact
  // differences of the stored full values; rounded deviations d_i instead bias it in float,
  // measured on a periodic shear layer. With 16-bit storage the deviations are all there is,
  // and the bias is far below their rounding.) FP64 keeps the slot-order sums.
  Real u[3] = {0, 0, 0};
  Real dr = 0;
  if constexpr (sizeof(Real) == 4) {
    moments_packed<L, DL>(f, dr, u);
  } else {
#pragma unroll
    for (int i = 0; i < Q; ++i) {
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        if (comp<L>(i, ax) > 0) u[ax] += f[i];
        if (comp<L>(i, ax) < 0) u[ax] -= f[i];
      }
    }
#pragma unroll
    for (int i = 0; i < Q; ++i) f[i] -= weight<L, Real>(i);  // now the deviations d_i
#pragma unroll
    for (int i = 0; i < Q; ++i) dr += f[i];
    dr += weight_defect<L, Real>();
  }
  Real r = Real(1) + dr;
  if constexpr (DL) {
    const Real rinv = __frcp_rn(r);  // one correctly rounded reciprocal; u within 1.5 ulp
#pragma unroll
    for (int ax = 3 - L::D; ax < 3; ++ax) u[ax] = mul_r(u[ax], rinv);
  } else if constexpr (sizeof(Real) == 4) {
    // u = m / r, correctly rounded, from one correctly rounded reciprocal y = 1/r shared by the
    // components: q = m y, then Markstein's quotient correction q + (m - r q) y, both steps
    // fused multiply-adds (P. Markstein, "Computation of elementary functions on the IBM
    // RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990). With y correctly rounded the
    // corrected q is the correctly rounded quotient, so the bits are those of a division
    // (tests/test_quotient_cpu.py checks the method against exact arithmetic); two divisions
    // cost the issue-bound FP32 ensemble kernel 4.7%. (m y alone is biased for r near 1.)
    const float y = __frcp_rn(r);
#pragma unroll
    for (int ax = 3 - L::D; ax < 3; ++ax) {
      const float q = __fmul_rn(u[ax], y);
      u[ax] = __fmaf_rn(__fmaf_rn(-r, q, u[ax]), y, q);
    }
  } else {
#pragma unroll
    for (int ax = 3 - L::D; ax < 3; ++ax) u[ax] = u[ax] / r;
  }

  // A per-cell relaxation field replaces the domain's om_pos (the force shift keeps the domain's).
  if (!UNFORCED && a.omega_field != nullptr) om_pos = (Real)__ldg(a.omega_field + c.cell);
  // Force as a velocity shift acc / omega (src/lib.cl:253-256; TRT: omega+, 682-685).
  if (UNFORCED) {
  } else if (a.acc_mode == kAccConstant) {
#pragma unroll
    for (int ax = 3 - L::D; ax < 3; ++ax) u[ax] = add_r(u[ax], a.force[ax]);
  } else if (a.acc_mode == kAccBoussinesq) {
    const Real b = a.alpha * (cval - a.c0);  // src/lib.cl:71
#pragma unroll
    for (int ax = 3 - L::D; ax < 3; ++ax) u[ax] = fma_r(b, a.force[ax], u[ax]);
  }
  const bool fixed = (flag & 6) != 0;  // FIXED_FLUID_VELOCITY | FIXED_FLUID_DENSITY
  if (fixed) {                         // src/lib.cl:257-262
    om_pos = 1;
    om_neg = 1;
    r = a.rho[c.cell];
    dr = r - Real(1);
#pragma unroll
    for (int ax = 3 - L::D; ax < 3; ++ax) u[ax] = a.vel[(size_t)c.cell * L::D + ax - (3 - L::D)];
  }
  Real uu = u[3 - L::D] * u[3 - L::D];
#pragma unroll
  for (int ax = 4 - L::D; ax < 3; ++ax) uu = fma_r(u[ax], u[ax], uu);

  if constexpr (sizeof(Real) == 4 && pack_collide<L, K>())
    collide_packed<L, TRT, true>(f, r, dr, u, uu, om_pos, om_neg);
  else
    collide<L, TRT, true>(f, r, dr, u, uu, om_pos, om_neg);
  sink.template fluid<L, P, EVEN, true>(static_cast<T*>(a.f), a.n, c, f);

  if (a.write_moments && !fixed) {
    a.rho[c.cell] = r;
#pragma unroll
    for (int ax = 3 - L::D; ax < 3; ++ax) a.vel[(size_t)c.cell * L::D + ax - (3 - L::D)] = u[ax];
    if (!isfinite(r) || !isfinite(uu)) atomicOr(a.status, 1);  // rho or any velocity component
  }

  if constexpr (NT == 1) {
    const bool keep = a.write_moments || (a.acc_mode == kAccBoussinesq && a.coupled == 0);
    tracer_update<TL, TP, EVEN, pack_collide<TL, K>()>(a.tr[0], a.n, c, flag, g, u, uu, keep,
                                                        sink);
  } else if constexpr (NT < 0) {
    for (int t = 0; t < a.ntracers; ++t) {
      Real gt[TL::Q];
      aa_load<TL, TP, EVEN, false>(static_cast<const typename TP::type*>(a.tr[t].g), a.n, c, gt);
      const bool keep = a.write_moments || (a.acc_mode == kAccBoussinesq && t == a.coupled);
      tracer_update<TL, TP, EVEN, pack_collide<TL, K>()>(a.tr[t], a.n, c, flag, gt, u, uu, keep);
    }
  }
}

// Direct variant: one cell per thread and grid row, loads straight into registers.
// NT: number of fused tracers known at compile time (0 or 1), or -1 for a runtime count.
// Every load a cell needs is issued before the first branch on any loaded value, so each thread
// has one memory phase (walls load populations they then ignore; they are a small fraction).
template <class L, bool TRT, int K, bool EVEN, int NT, int KT = default_tracer_kind<K>()>
__global__ void __launch_bounds__(256)
    aa_step_kernel(const __grid_constant__ StepArgs<typename Pop<K>::real> a) {
  using P = Pop<K>;
  using Real = typename P::real;
  using T = typename P::type;
  using TL = typename TracerLattice<L::D>::type;
  using TP = TracerPop<KT>;

  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= a.nz) return;

  for (int x = blockIdx.z; x < a.nx; x += gridDim.z) {
    for (int y = blockIdx.y; y < a.ny; y += gridDim.y) {
      const CellPos c = make_cellpos(a, x, y, z, EVEN);
      const int flag = a.flags[c.cell];
      Real f[L::Q];
      aa_load<L, P, EVEN, dev_in<K>()>(static_cast<const T*>(a.f), a.n, c, f);
      Real g[NT == 1 ? TL::Q : 1];
      if constexpr (NT == 1)
        aa_load<TL, TP, EVEN, false>(static_cast<const typename TP::type*>(a.tr[0].g), a.n, c, g);
      Real cval = 0;
      if (a.acc_mode == kAccBoussinesq) cval = a.coupled_val[c.cell];
      update_cell<L, TRT, K, EVEN, NT, GlobalSink, KT>(a, c, flag, f, g, cval, a.om_pos,
                                                      a.om_neg);
    }
  }
}

}  // namespace lbm
