// Two cells a thread for the TMA-staged kernel with 16-bit populations (D3Q27, no fused
// tracer): consumer thread t updates cells t and t + 128 of its 256-cell tile, with every FP32
// operation of the cell update on Blackwell's packed instructions (lane x: cell t, lane y: cell
// t + 128). Each lane performs exactly the operations of update_cell / moments_packed /
// collide_packed in the same order (the packed instructions round each lane as the scalar one),
// so the results are the bits of the one-cell path; the operation count per cell drops because
// every operation is packed, not only the ones that pair opposite directions. Measured +1.4% on
// the 256^3 Taylor-Green run with FP16 populations (the kernel is close to its memory time).
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
    for (int ax = 0; ax < 3; ++ax) {
      if (comp<L>(2 * p + 1, ax) > 0) m[ax] = add2(m[ax], del[p]);
      if (comp<L>(2 * p + 1, ax) < 0) m[ax] = sub2(m[ax], del[p]);
    }
  }
}

// One opposite pair (i, i + 1) of collide_packed<L, TRT, true> for two cells.
template <class L, bool TRT>
__device__ __forceinline__ void collide_pair2(float2 (&v)[L::Q], int i, float2 ru, float2 unit,
                                              float2 quad, const float2 (&u)[3], float2 om_pos,
                                              float2 om_neg) {
  const float k = float(L::wk(i));
  const float2 cu = c_dot2<L>(i, u);
  const float2 kr = mul2(splat(k), ru);
  const float2 ku = fma2(splat(k), unit, splat(weight_gap<L, float>(i)));
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

// update_cell<L, TRT, K, EVEN, 0> for two cells whose deviations were loaded into f, results
// into the stage: slot i of each cell at the position it was read from (see StageSink).
// cellA / cellB: the cells' indices; flagA / flagB their flags; cval: the coupled value.
template <class St, class L, bool TRT, int K, bool EVEN, int TILE>
__device__ __forceinline__ void update_cell2(const StepArgs<float>& a, unsigned char* st, int tid,
                                             unsigned cellA, unsigned cellB, int flagA, int flagB,
                                             float2 (&f)[L::Q], float2 cval) {
  using P = Pop<K>;
  using T = typename P::type;
  constexpr int Q = L::Q;
  static_assert(L::D == 3 && dev_in<K>(), "two cells a thread: D3Q27 with 16-bit storage");
  const bool wallA = (flagA & 1) != 0, wallB = (flagB & 1) != 0;
  if (wallA && wallB) return;

  float2 dr, m[3];
  moments2<L>(f, dr, m);
  float2 r = add2(splat(1.0f), dr);
  const float2 rinv = make_float2(__frcp_rn(r.x), __frcp_rn(r.y));
  float2 u[3];
#pragma unroll
  for (int ax = 0; ax < 3; ++ax) u[ax] = mul2(m[ax], rinv);

  float2 om_pos = splat(a.om_pos), om_neg = splat(a.om_neg);
  if (a.omega_field != nullptr)
    om_pos = make_float2(__ldg(a.omega_field + cellA), __ldg(a.omega_field + cellB));
  if (a.acc_mode == kAccConstant) {
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) u[ax] = add2(u[ax], splat(a.force[ax]));
  } else if (a.acc_mode == kAccBoussinesq) {
    const float2 b = mul2(splat(a.alpha), sub2(cval, splat(a.c0)));
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) u[ax] = fma2(b, splat(a.force[ax]), u[ax]);
  }
  const bool fixedA = (flagA & 6) != 0, fixedB = (flagB & 6) != 0;
  if (fixedA) {
    om_pos.x = 1.0f;
    om_neg.x = 1.0f;
    r.x = a.rho[cellA];
    dr.x = r.x - 1.0f;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) u[ax].x = a.vel[(size_t)cellA * 3 + ax];
  }
  if (fixedB) {
    om_pos.y = 1.0f;
    om_neg.y = 1.0f;
    r.y = a.rho[cellB];
    dr.y = r.y - 1.0f;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) u[ax].y = a.vel[(size_t)cellB * 3 + ax];
  }
  float2 uu = mul2(u[0], u[0]);
  uu = fma2(u[1], u[1], uu);
  uu = fma2(u[2], u[2], uu);

  // collide_packed<L, TRT, true>
  const float2 ru = over_den2_hi_lo(r, inv_den_hi<L, float>(), inv_den_lo<L, float>());
  const float2 unit = over_den2_hi_lo(dr, inv_den_hi<L, float>(), inv_den_lo<L, float>());
  const float2 quad = mul2(splat(-1.5f), uu);
  {
    const float k0 = float(L::wk(0));
    const float2 e0 = fma2(mul2(splat(k0), ru), quad,
                           fma2(splat(k0), unit, splat(weight_gap<L, float>(0))));
    f[0] = fma2(om_pos, sub2(e0, f[0]), f[0]);
  }
#pragma unroll
  for (int i = 1; i < Q; i += 2) collide_pair2<L, TRT>(f, i, ru, unit, quad, u, om_pos, om_neg);

  // The results into the stage (StageSink's positions), walls skipped.
  T* base = reinterpret_cast<T*>(st);
#pragma unroll
  for (int i = 0; i < Q; ++i) {
    const int cz = comp<L>(i, 2);
    const int pa = EVEN ? St::H + ((tid - cz) & (TILE - 1)) : tid;
    const int pb = EVEN ? St::H + ((tid + TILE / 2 - cz) & (TILE - 1)) : tid + TILE / 2;
    const float2 val = EVEN ? f[opp(i)] : f[i];
    if (!wallA) P::store_dev(base + i * St::SEG + pa, val.x, 0.0f);
    if (!wallB) P::store_dev(base + i * St::SEG + pb, val.y, 0.0f);
  }
  if constexpr (EVEN && St::QP > Q) {
    // The padding rows of the last four-row group repeat slot Q - 1.
    constexpr int i = Q - 1;
    const int pa = St::H + ((tid - comp<L>(i, 2)) & (TILE - 1));
    const int pb = St::H + ((tid + TILE / 2 - comp<L>(i, 2)) & (TILE - 1));
    const T wa = base[i * St::SEG + pa], wb = base[i * St::SEG + pb];
#pragma unroll
    for (int rr = Q; rr < St::QP; ++rr) {
      base[rr * St::SEG + pa] = wa;
      base[rr * St::SEG + pb] = wb;
    }
  }

  if (a.write_moments) {
    if (!wallA && !fixedA) {
      a.rho[cellA] = r.x;
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) a.vel[(size_t)cellA * 3 + ax] = u[ax].x;
      if (!isfinite(r.x) || !isfinite(uu.x)) atomicOr(a.status, 1);
    }
    if (!wallB && !fixedB) {
      a.rho[cellB] = r.y;
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) a.vel[(size_t)cellB * 3 + ax] = u[ax].y;
      if (!isfinite(r.y) || !isfinite(uu.y)) atomicOr(a.status, 1);
    }
  }
}

}  // namespace lbm
