// Two cells a thread for the TMA-staged kernel with 16-bit populations: consumer thread t
// updates cells t and t + 128 of its 256-cell tile, with every FP32 operation of the cell update
// on Blackwell's packed instructions (lane x: cell t, lane y: cell t + 128). Each lane performs
// exactly the operations of update_cell / moments_packed / collide_packed / tracer_update in the
// same order (the packed instructions round each lane as the scalar one), so the results are
// the bits of the one-cell path; the operation count per cell drops because every operation is
// packed, not only the ones that pair opposite directions.
// Used for D3Q27 BGK without a tracer (results through the stage; +1.4% on the 256^3
// Taylor-Green run, whose kernel is close to its memory time) and for D2Q9 BGK / TRT with none or
// one fused tracer (both parities: results through the stage, or straight to HBM on even steps
// of rows longer than one tile), whose one-cell kernels are issue-bound.
#pragma once

#include "aa_step.cuh"

namespace lbm {

__device__ __forceinline__ float2 over_den2_hi_lo(float2 x, float hi, float lo) {
  return fma2(x, splat(hi), mul2(x, splat(lo)));
}

// c_i . u for both cells, the additions of c_dot in its order.
template <class L>
__device__ __forceinline__ float2 c_dot2(int i, const float2 (&u)[3]) {
  float2 cu = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (comp<L>(i, a) > 0) cu = add2(cu, u[a]);
    if (comp<L>(i, a) < 0) cu = sub2(cu, u[a]);
  }
  return cu;
}

// moments_packed<L, true> for two cells: v holds deviations.
template <class L>
__device__ __forceinline__ void moments2(const float2 (&v)[L::Q], float2& dr, float2 (&m)[3]) {
  constexpr int P = (L::Q - 1) / 2;
  float2 del[P];
  float2 acc_even = make_float2(0.0f, 0.0f), acc_odd = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int p = 0; p + 1 < P; p += 2) {
    const int i = 2 * p + 1, j = 2 * p + 3;
    del[p] = sub2(v[i], v[i + 1]);
    del[p + 1] = sub2(v[j], v[j + 1]);
    acc_even = add2(acc_even, add2(v[i], v[i + 1]));
    acc_odd = add2(acc_odd, add2(v[j], v[j + 1]));
  }
  float2 sig_last = make_float2(0.0f, 0.0f);
  if constexpr (P % 2 == 1) {
    constexpr int i = 2 * (P - 1) + 1;
    del[P - 1] = sub2(v[i], v[i + 1]);
    sig_last = add2(v[i], v[i + 1]);
  }
  dr = add2(add2(add2(v[0], add2(acc_even, acc_odd)), sig_last), splat(weight_defect<L, float>()));
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) m[ax] = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int p = 0; p < P; ++p) {
#pragma unroll
    for (int ax = 3 - L::D; ax < 3; ++ax) {
      if (comp<L>(2 * p + 1, ax) > 0) m[ax] = add2(m[ax], del[p]);
      if (comp<L>(2 * p + 1, ax) < 0) m[ax] = sub2(m[ax], del[p]);
    }
  }
}

// One opposite pair (i, i + 1) of collide_packed<L, TRT, DEV> for two cells.
template <class L, bool TRT, bool DEV>
__device__ __forceinline__ void collide_pair2(float2 (&v)[L::Q], int i, float2 ru, float2 unit,
                                              float2 quad, const float2 (&u)[3], float2 om_pos,
                                              float2 om_neg) {
  const float k = float(L::wk(i));
  const float2 cu = c_dot2<L>(i, u);
  const float2 kr = mul2(splat(k), ru);
  const float2 ku = fma2(splat(k), unit, splat(DEV ? weight_gap<L, float>(i) : 0.0f));
  const float2 X = fma2(mul2(splat(4.5f), cu), cu, quad);
  const float2 A = fma2(kr, X, ku);
  const float2 B = mul2(mul2(kr, splat(3.0f)), cu);
  float2 F = v[i], G = v[i + 1];
  if constexpr (TRT) {
    const float2 S = mul2(splat(0.5f), add2(F, G));
    const float2 D = mul2(splat(0.5f), sub2(F, G));
    const float2 fp = mul2(om_pos, sub2(A, S));
    const float2 fn = mul2(om_neg, sub2(B, D));
    F = add2(F, add2(fp, fn));
    G = add2(G, sub2(fp, fn));
  } else {
    F = fma2(om_pos, sub2(add2(A, B), F), F);
    G = fma2(om_pos, sub2(sub2(A, B), G), G);
  }
  v[i] = F;
  v[i + 1] = G;
}

// collide_packed<L, TRT, DEV> for two cells (r: densities, dr: r - 1; the tracers pass their
// concentration as both).
template <class L, bool TRT, bool DEV>
__device__ __forceinline__ void collide2(float2 (&v)[L::Q], float2 r, float2 dr,
                                         const float2 (&u)[3], float2 uu, float2 om_pos,
                                         float2 om_neg) {
  const float2 ru = over_den2_hi_lo(r, inv_den_hi<L, float>(), inv_den_lo<L, float>());
  const float2 unit =
      DEV ? over_den2_hi_lo(dr, inv_den_hi<L, float>(), inv_den_lo<L, float>()) : ru;
  const float2 quad = mul2(splat(-1.5f), uu);
  {
    const float k0 = float(L::wk(0));
    const float2 e0 = fma2(mul2(splat(k0), ru), quad,
                           fma2(splat(k0), unit, splat(DEV ? weight_gap<L, float>(0) : 0.0f)));
    v[0] = fma2(om_pos, sub2(e0, v[0]), v[0]);
  }
#pragma unroll
  for (int i = 1; i < L::Q; i += 2) collide_pair2<L, TRT, DEV>(v, i, ru, unit, quad, u, om_pos, om_neg);
}

// Where update_cell2 puts its results: into the stage the operands came from, at StageSink's
// positions (slot i of the cell on odd steps, the very position read on even steps); walls
// (skip) leave theirs untouched.
template <class St, int TILE>
struct PairSink {
  unsigned char* st;
  int tid;  // cell A's column; cell B is tid + TILE / 2

  template <class L, class P, bool EVEN>
  __device__ __forceinline__ void fluid(bool skipA, bool skipB, const float2 (&v)[L::Q]) const {
    using T = typename P::type;
    T* base = reinterpret_cast<T*>(st);
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
      const int cz = comp<L>(i, 2);
      const int pa = stage_pos<St::kWR, EVEN>(St::H, tid, cz);
      const int pb = stage_pos<St::kWR, EVEN>(St::H, tid + TILE / 2, cz);
      const float2 val = EVEN ? v[opp(i)] : v[i];
      if (!skipA) P::store_dev(base + i * St::SEG + pa, val.x, 0.0f);
      if (!skipB) P::store_dev(base + i * St::SEG + pb, val.y, 0.0f);
    }
    if constexpr (EVEN && St::QP > L::Q) {
      // The padding rows of the last four-row group repeat slot Q - 1.
      constexpr int i = L::Q - 1;
      const int pa = stage_pos<St::kWR, EVEN>(St::H, tid, comp<L>(i, 2));
      const int pb = stage_pos<St::kWR, EVEN>(St::H, tid + TILE / 2, comp<L>(i, 2));
      const T wa = base[i * St::SEG + pa], wb = base[i * St::SEG + pb];
#pragma unroll
      for (int rr = L::Q; rr < St::QP; ++rr) {
        base[rr * St::SEG + pa] = wa;
        base[rr * St::SEG + pb] = wb;
      }
    }
  }

  template <class TL, class TP, bool EVEN>
  __device__ __forceinline__ void tracer(bool skipA, bool skipB, const float2 (&v)[TL::Q]) const {
    using TT = typename TP::type;
#pragma unroll
    for (int i = 0; i < TL::Q; ++i) {
      const float2 val = EVEN ? v[opp(i)] : v[i];
      TT* base = reinterpret_cast<TT*>(st + St::off_trc) + i * St::SEGG;
      const int cz = comp<TL>(i, 2);
      if (!skipA) TP::store(base + stage_pos<St::kWR, EVEN>(St::HG, tid, cz), val.x, 0.0f);
      if (!skipB) TP::store(base + stage_pos<St::kWR, EVEN>(St::HG, tid + TILE / 2, cz), val.y, 0.0f);
    }
  }
};

// tracer_update<TL, TP, EVEN, true> for two cells: the concentration, the fixed-value override,
// the packed collision and the AA store. Wall cells (skip) are computed but not stored.
template <class TL, class TP, bool EVEN, class Sink>
__device__ __forceinline__ void tracer_update2(const TracerArgs<float>& tr, long long n,
                                               const CellPos& cA, const CellPos& cB, int flagA,
                                               int flagB, bool wallA, bool wallB,
                                               float2 (&g)[TL::Q], const float2 (&u)[3],
                                               float2 uu, bool keep, const Sink& sink) {
  float2 rt = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int i = 0; i < TL::Q; ++i) rt = add2(rt, g[i]);
  float2 om = splat(tr.omega), om_n = splat(tr.omega_neg);
  const bool tfA = (flagA & 8) != 0, tfB = (flagB & 8) != 0;  // FIXED_SCALAR_VALUE
  if (tfA) {
    om.x = 1.0f;
    om_n.x = 1.0f;
    rt.x = tr.val[cA.cell];
  }
  if (tfB) {
    om.y = 1.0f;
    om_n.y = 1.0f;
    rt.y = tr.val[cB.cell];
  }
  if (tr.trt)
    collide2<TL, true, false>(g, rt, rt, u, uu, om, om_n);
  else
    collide2<TL, false, false>(g, rt, rt, u, uu, om, om);
  sink.template tracer<TL, TP, EVEN>(wallA, wallB, g);
  if (keep) {
    if (!wallA && !tfA) tr.val[cA.cell] = rt.x;
    if (!wallB && !tfB) tr.val[cB.cell] = rt.y;
  }
}

// update_cell<L, TRT, K, EVEN, NT, ..., KT> for two cells whose deviations were loaded into f
// (and, NT == 1, the first tracer's populations into g); cA / cB: the cells' positions (with
// their neighbourhoods when the sink stores to HBM on even steps); flagA / flagB their flags;
// cval: the coupled values.
template <class L, bool TRT, int K, bool EVEN, int NT, int KT, class Sink>
__device__ __forceinline__ void update_cell2(const StepArgs<float>& a, const Sink& sink,
                                             const CellPos& cA, const CellPos& cB, int flagA,
                                             int flagB, float2 (&f)[L::Q],
                                             float2 (&g)[NT == 1 ? TracerLattice<L::D>::type::Q : 1],
                                             float2 cval) {
  using P = Pop<K>;
  using TL = typename TracerLattice<L::D>::type;
  using TP = TracerPop<KT>;
  constexpr int D = L::D;
  static_assert(dev_in<K>(), "two cells a thread: 16-bit storage");
  const bool wallA = (flagA & 1) != 0, wallB = (flagB & 1) != 0;
  if (wallA && wallB) return;
  const unsigned cellA = cA.cell, cellB = cB.cell;

  float2 dr, m[3];
  moments2<L>(f, dr, m);
  float2 r = add2(splat(1.0f), dr);
  const float2 rinv = make_float2(__frcp_rn(r.x), __frcp_rn(r.y));
  float2 u[3];
  u[0] = make_float2(0.0f, 0.0f);
#pragma unroll
  for (int ax = 3 - D; ax < 3; ++ax) u[ax] = mul2(m[ax], rinv);

  float2 om_pos = splat(a.om_pos), om_neg = splat(a.om_neg);
  if (a.omega_field != nullptr)
    om_pos = make_float2(__ldg(a.omega_field + cellA), __ldg(a.omega_field + cellB));
  if (a.acc_mode == kAccConstant) {
#pragma unroll
    for (int ax = 3 - D; ax < 3; ++ax) u[ax] = add2(u[ax], splat(a.force[ax]));
  } else if (a.acc_mode == kAccBoussinesq) {
    const float2 b = mul2(splat(a.alpha), sub2(cval, splat(a.c0)));
#pragma unroll
    for (int ax = 3 - D; ax < 3; ++ax) u[ax] = fma2(b, splat(a.force[ax]), u[ax]);
  }
  const bool fixedA = (flagA & 6) != 0, fixedB = (flagB & 6) != 0;
  if (fixedA) {
    om_pos.x = 1.0f;
    om_neg.x = 1.0f;
    r.x = a.rho[cellA];
    dr.x = r.x - 1.0f;
#pragma unroll
    for (int ax = 3 - D; ax < 3; ++ax) u[ax].x = a.vel[(size_t)cellA * D + ax - (3 - D)];
  }
  if (fixedB) {
    om_pos.y = 1.0f;
    om_neg.y = 1.0f;
    r.y = a.rho[cellB];
    dr.y = r.y - 1.0f;
#pragma unroll
    for (int ax = 3 - D; ax < 3; ++ax) u[ax].y = a.vel[(size_t)cellB * D + ax - (3 - D)];
  }
  float2 uu = mul2(u[3 - D], u[3 - D]);
#pragma unroll
  for (int ax = 4 - D; ax < 3; ++ax) uu = fma2(u[ax], u[ax], uu);

  collide2<L, TRT, true>(f, r, dr, u, uu, om_pos, om_neg);
  sink.template fluid<L, P, EVEN>(wallA, wallB, f);

  if (a.write_moments) {
    if (!wallA && !fixedA) {
      a.rho[cellA] = r.x;
#pragma unroll
      for (int ax = 3 - D; ax < 3; ++ax) a.vel[(size_t)cellA * D + ax - (3 - D)] = u[ax].x;
      if (!isfinite(r.x) || !isfinite(uu.x)) atomicOr(a.status, 1);
    }
    if (!wallB && !fixedB) {
      a.rho[cellB] = r.y;
#pragma unroll
      for (int ax = 3 - D; ax < 3; ++ax) a.vel[(size_t)cellB * D + ax - (3 - D)] = u[ax].y;
      if (!isfinite(r.y) || !isfinite(uu.y)) atomicOr(a.status, 1);
    }
  }

  if constexpr (NT == 1) {
    const bool keep = a.write_moments || (a.acc_mode == kAccBoussinesq && a.coupled == 0);
    tracer_update2<TL, TP, EVEN>(a.tr[0], a.n, cA, cB, flagA, flagB, wallA, wallB, g, u, uu, keep,
                                 sink);
  }
}

}  // namespace lbm
