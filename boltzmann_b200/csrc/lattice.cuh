// Velocity sets of the lattice-Boltzmann hot path, as compile-time tables.
//
// Slot order is the reference's (djbarker/boltzmann src/velocities.rs:66-191, identical to the
// qs tables of src/lib.cl:105, 195-196, 306-307, 411-417): populations are stored in that order,
// so checkpoints and the AA slot semantics line up with the reference. In every set the rest
// direction is slot 0 and opposite directions sit in adjacent slots (2k-1, 2k).
#pragma once

namespace lbm {

// w(i) / wd(i): the weight in float / double (float is what the reference's host equilibrium
// uses, src/velocities.rs:73-85). wk(i) / kDen: the same weight as an exact integer multiple of
// 1 / kDen, used by the collision so that the weights sum to exactly one in any precision.

struct D1Q3 {
  static constexpr int D = 1, Q = 3, kDen = 6;
  __host__ __device__ static constexpr int c(int i, int a) {
    constexpr int t[3][3] = {{0, 0, 0}, {1, 0, 0}, {-1, 0, 0}};
    return t[i][a];
  }
  __host__ __device__ static constexpr int wk(int i) { return i == 0 ? 4 : 1; }
  __host__ __device__ static constexpr float w(int i) { return i == 0 ? 4.0f / 6.0f : 1.0f / 6.0f; }
  __host__ __device__ static constexpr double wd(int i) { return i == 0 ? 4.0 / 6.0 : 1.0 / 6.0; }
};

struct D2Q9 {
  static constexpr int D = 2, Q = 9, kDen = 36;
  __host__ __device__ static constexpr int wk(int i) { return i == 0 ? 16 : (i < 5 ? 4 : 1); }
  __host__ __device__ static constexpr int c(int i, int a) {
    constexpr int t[9][3] = {{0, 0, 0}, {1, 0, 0},   {-1, 0, 0}, {0, 1, 0}, {0, -1, 0},
                             {1, 1, 0}, {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0}};
    return t[i][a];
  }
  __host__ __device__ static constexpr float w(int i) {
    return i == 0 ? 4.0f / 9.0f : (i < 5 ? 1.0f / 9.0f : 1.0f / 36.0f);
  }
  __host__ __device__ static constexpr double wd(int i) {
    return i == 0 ? 4.0 / 9.0 : (i < 5 ? 1.0 / 9.0 : 1.0 / 36.0);
  }
};

struct D2Q5 {
  static constexpr int D = 2, Q = 5, kDen = 6;
  __host__ __device__ static constexpr int wk(int i) { return i == 0 ? 2 : 1; }
  __host__ __device__ static constexpr int c(int i, int a) {
    constexpr int t[5][3] = {{0, 0, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}};
    return t[i][a];
  }
  __host__ __device__ static constexpr float w(int i) { return i == 0 ? 1.0f / 3.0f : 1.0f / 6.0f; }
  __host__ __device__ static constexpr double wd(int i) { return i == 0 ? 1.0 / 3.0 : 1.0 / 6.0; }
};

struct D3Q7 {
  static constexpr int D = 3, Q = 7, kDen = 120;
  __host__ __device__ static constexpr int wk(int i) { return i == 0 ? 6 : 19; }
  __host__ __device__ static constexpr int c(int i, int a) {
    constexpr int t[7][3] = {{0, 0, 0},  {1, 0, 0}, {-1, 0, 0}, {0, 1, 0},
                             {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    return t[i][a];
  }
  __host__ __device__ static constexpr float w(int i) {
    return i == 0 ? 1.0f / 20.0f : 19.0f / 120.0f;
  }
  __host__ __device__ static constexpr double wd(int i) {
    return i == 0 ? 1.0 / 20.0 : 19.0 / 120.0;
  }
};

struct D3Q27 {
  static constexpr int D = 3, Q = 27, kDen = 216;
  __host__ __device__ static constexpr int wk(int i) {
    return i == 0 ? 64 : (i < 7 ? 16 : (i < 19 ? 4 : 1));
  }
  __host__ __device__ static constexpr int c(int i, int a) {
    constexpr int t[27][3] = {
        {0, 0, 0},   {1, 0, 0},  {-1, 0, 0},  {0, 1, 0},  {0, -1, 0}, {0, 0, 1},   {0, 0, -1},
        {1, 1, 0},   {-1, -1, 0}, {1, -1, 0}, {-1, 1, 0}, {1, 0, 1},  {-1, 0, -1}, {0, 1, 1},
        {0, -1, -1}, {1, 0, -1}, {-1, 0, 1},  {0, 1, -1}, {0, -1, 1}, {1, 1, 1},   {-1, -1, -1},
        {1, -1, 1},  {-1, 1, -1}, {1, 1, -1}, {-1, -1, 1}, {1, -1, -1}, {-1, 1, 1}};
    return t[i][a];
  }
  __host__ __device__ static constexpr float w(int i) {
    return i == 0 ? 8.0f / 27.0f : (i < 7 ? 2.0f / 27.0f : (i < 19 ? 1.0f / 54.0f : 1.0f / 216.0f));
  }
  __host__ __device__ static constexpr double wd(int i) {
    return i == 0 ? 8.0 / 27.0 : (i < 7 ? 2.0 / 27.0 : (i < 19 ? 1.0 / 54.0 : 1.0 / 216.0));
  }
};

// Opposite slot: 0 -> 0, 2k-1 <-> 2k.
__host__ __device__ constexpr int opp(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }

// Tracer velocity set that goes with a fluid dimension (the reference registers D2Q5 and D3Q7
// advection-diffusion kernels only, src/opencl.rs:123-129).
template <int D>
struct TracerLattice;
template <>
struct TracerLattice<2> {
  using type = D2Q5;
};
template <>
struct TracerLattice<3> {
  using type = D3Q7;
};

}  // namespace lbm
