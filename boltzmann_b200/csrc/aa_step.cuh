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
  Real* g;    // [Qt][N]
  Real* val;  // [N]
  Real omega;
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
  Real acc[3];         // constant acceleration, or the Boussinesq gravity vector
  Real alpha, c0;      // Boussinesq coupling
  int coupled;         // index of the coupled tracer
  const Real* coupled_val;  // its val[] (read for the Boussinesq term)
  int ntracers;
  TracerArgs<Real> tr[kMaxTracers];
  int write_moments;   // 1 on the last step of an iterate call
  int* status;         // bit 0 set when a non-finite density is produced
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

// Upstream coordinate along one axis for a velocity component cc (coordinate - cc, wrapped).
__device__ __forceinline__ int upstream_coord(int cc, int minus1, int same, int plus1) {
  return cc > 0 ? minus1 : (cc < 0 ? plus1 : same);
}

struct CellPos {
  long long cell;
  int x, y, z;
  int xm, xp, ym, yp, zm, zp;  // wrapped neighbour coordinates
  int nx, ny, nz;

  // Cell index of (x, y, z) - c_i, periodic.
  template <class L>
  __device__ __forceinline__ long long upstream(int i) const {
    const int ux = upstream_coord(comp<L>(i, 0), xm, x, xp);
    const int uy = upstream_coord(comp<L>(i, 1), ym, y, yp);
    const int uz = upstream_coord(comp<L>(i, 2), zm, z, zp);
    return ((long long)ux * ny + uy) * nz + uz;
  }
};

// AA load of one velocity set's populations for this cell.
template <class L, class P, bool EVEN>
__device__ __forceinline__ void aa_load(const typename P::type* __restrict__ f, long long n,
                                        const CellPos& c, typename P::real (&v)[L::Q]) {
  using Real = typename P::real;
#pragma unroll
  for (int i = 0; i < L::Q; ++i) {
    if constexpr (EVEN)
      v[i] = P::load(f + (long long)i * n + c.upstream<L>(i), weight<L, Real>(i));
    else
      v[i] = P::load(f + (long long)opp(i) * n + c.cell, weight<L, Real>(i));
  }
}

// AA store matching aa_load.
template <class L, class P, bool EVEN>
__device__ __forceinline__ void aa_store(typename P::type* __restrict__ f, long long n,
                                         const CellPos& c, const typename P::real (&v)[L::Q]) {
  using Real = typename P::real;
#pragma unroll
  for (int i = 0; i < L::Q; ++i) {
    if constexpr (EVEN)
      P::store(f + (long long)i * n + c.upstream<L>(i), v[opp(i)], weight<L, Real>(i));
    else
      P::store(f + (long long)i * n + c.cell, v[i], weight<L, Real>(i));
  }
}

// BGK or TRT collision against the second-order equilibrium
//   feq_i = w_i r (1 + 3 c_i.u + 4.5 (c_i.u)^2 - 1.5 u.u),
// evaluated per opposite pair (i, i+1): feq = A +- B with A = w r (1 + 4.5 cu^2 - 1.5 uu) and
// B = 3 w r cu. TRT relaxes the symmetric part with om_pos and the antisymmetric part with
// om_neg (src/lib.cl:697-719); BGK relaxes both with om_pos (src/lib.cl:266-274).
template <class L, bool TRT, class Real>
__device__ __forceinline__ void collide(Real (&f)[L::Q], Real r, const Real (&u)[3], Real uu,
                                        Real om_pos, Real om_neg) {
  const Real base = Real(1) - Real(1.5) * uu;
  {
    const Real a0 = weight<L, Real>(0) * r * base;
    f[0] += om_pos * (a0 - f[0]);
  }
#pragma unroll
  for (int i = 1; i < L::Q; i += 2) {
    Real cu = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (comp<L>(i, a) > 0) cu += u[a];
      if (comp<L>(i, a) < 0) cu -= u[a];
    }
    const Real wr = weight<L, Real>(i) * r;
    const Real A = wr * (base + Real(4.5) * cu * cu);
    const Real B = wr * Real(3) * cu;
    if constexpr (TRT) {
      const Real s = Real(0.5) * (f[i] + f[i + 1]);
      const Real d = Real(0.5) * (f[i] - f[i + 1]);
      const Real fp = om_pos * (A - s);
      const Real fn = om_neg * (B - d);
      f[i] += fp + fn;
      f[i + 1] += fp - fn;
    } else {
      f[i] += om_pos * (A + B - f[i]);
      f[i + 1] += om_pos * (A - B - f[i + 1]);
    }
  }
}

template <class L, bool TRT, int K, bool EVEN, bool TRACERS>
__global__ void __launch_bounds__(256)
    aa_step_kernel(const __grid_constant__ StepArgs<typename Pop<K>::real> a) {
  using P = Pop<K>;
  using Real = typename P::real;
  using T = typename P::type;
  using TL = typename TracerLattice<L::D>::type;
  using TP = Pop<(sizeof(Real) == 8 ? kF64 : kF32)>;
  constexpr int Q = L::Q;

  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  if (z >= a.nz) return;

  for (int x = blockIdx.z; x < a.nx; x += gridDim.z) {
    for (int y = blockIdx.y; y < a.ny; y += gridDim.y) {
      CellPos c;
      c.nx = a.nx;
      c.ny = a.ny;
      c.nz = a.nz;
      c.x = x;
      c.y = y;
      c.z = z;
      c.cell = ((long long)x * a.ny + y) * a.nz + z;

      const int flag = a.flags[c.cell];
      if (flag & 1) continue;  // WALL: never updated (src/lib.cl:210-213)

      if constexpr (EVEN) {
        c.xm = x == 0 ? a.nx - 1 : x - 1;
        c.xp = x == a.nx - 1 ? 0 : x + 1;
        c.ym = y == 0 ? a.ny - 1 : y - 1;
        c.yp = y == a.ny - 1 ? 0 : y + 1;
        c.zm = z == 0 ? a.nz - 1 : z - 1;
        c.zp = z == a.nz - 1 ? 0 : z + 1;
      }

      Real f[Q];
      aa_load<L, P, EVEN>(static_cast<const T*>(a.f), a.n, c, f);

      // Moments (src/lib.cl:249-251).
      Real r = 0;
#pragma unroll
      for (int i = 0; i < Q; ++i) r += f[i];
      Real u[3] = {0, 0, 0};
#pragma unroll
      for (int i = 0; i < Q; ++i) {
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
          if (comp<L>(i, ax) > 0) u[ax] += f[i];
          if (comp<L>(i, ax) < 0) u[ax] -= f[i];
        }
      }
#pragma unroll
      for (int ax = 3 - L::D; ax < 3; ++ax) u[ax] = u[ax] / r;

      Real om_pos = a.om_pos, om_neg = a.om_neg;
      // Force as a velocity shift acc / omega (src/lib.cl:253-256; TRT: omega+, 682-685).
      if (a.acc_mode == kAccConstant) {
#pragma unroll
        for (int ax = 3 - L::D; ax < 3; ++ax) u[ax] += a.acc[ax] / om_pos;
      } else if (a.acc_mode == kAccBoussinesq) {
        const Real b = a.alpha * (a.coupled_val[c.cell] - a.c0);
#pragma unroll
        for (int ax = 3 - L::D; ax < 3; ++ax) u[ax] += (a.acc[ax] * b) / om_pos;
      }
      const bool fixed = (flag & 6) != 0;  // FIXED_FLUID_VELOCITY | FIXED_FLUID_DENSITY
      if (fixed) {                         // src/lib.cl:257-262
        om_pos = 1;
        om_neg = 1;
        r = a.rho[c.cell];
#pragma unroll
        for (int ax = 3 - L::D; ax < 3; ++ax) u[ax] = a.vel[c.cell * L::D + ax - (3 - L::D)];
      }
      Real uu = 0;
#pragma unroll
      for (int ax = 3 - L::D; ax < 3; ++ax) uu += u[ax] * u[ax];

      collide<L, TRT>(f, r, u, uu, om_pos, om_neg);
      aa_store<L, P, EVEN>(static_cast<T*>(a.f), a.n, c, f);

      if (a.write_moments && !fixed) {
        a.rho[c.cell] = r;
#pragma unroll
        for (int ax = 3 - L::D; ax < 3; ++ax) a.vel[c.cell * L::D + ax - (3 - L::D)] = u[ax];
        if (!isfinite(r)) atomicOr(a.status, 1);
      }

      if constexpr (TRACERS) {
        // Advection-diffusion tracers in the fluid velocity just computed
        // (src/lib.cl:102-189, 303-405).
        for (int t = 0; t < a.ntracers; ++t) {
          const TracerArgs<Real>& tr = a.tr[t];
          Real g[TL::Q];
          aa_load<TL, TP, EVEN>(tr.g, a.n, c, g);
          Real rt = 0;
#pragma unroll
          for (int i = 0; i < TL::Q; ++i) rt += g[i];
          Real om = tr.omega;
          const bool tfixed = (flag & 8) != 0;  // FIXED_SCALAR_VALUE
          if (tfixed) {
            om = 1;
            rt = tr.val[c.cell];
          }
          collide<TL, false>(g, rt, u, uu, om, om);
          aa_store<TL, TP, EVEN>(tr.g, a.n, c, g);
          const bool keep = a.write_moments || (a.acc_mode == kAccBoussinesq && t == a.coupled);
          if (keep && !tfixed) tr.val[c.cell] = rt;
        }
      }
    }
  }
}

}  // namespace lbm
