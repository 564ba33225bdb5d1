// Population storage policies.
//
// F32 : populations stored as float, collided in float.
// F16 / BF16 : populations stored as the 16-bit offset f_i - w_i from the lattice weight,
//              widened to float for the collision and rounded to nearest on store; this halves
//              the bytes per cell update.
// F64 : populations and every operation in double (the on-GPU FP64 comparison run).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace lbm {

enum StorageKind : int { kF32 = 0, kF16 = 1, kBF16 = 2, kF64 = 3 };

template <int K>
struct Pop;

template <>
struct Pop<kF32> {
  using type = float;
  using real = float;
  __device__ __forceinline__ static real load(const type* p, real) { return *p; }
  __device__ __forceinline__ static void store(type* p, real v, real) { *p = v; }
};

template <>
struct Pop<kF16> {
  using type = __half;
  using real = float;
  __device__ __forceinline__ static real load(const type* p, real w) {
    return __half2float(*p) + w;
  }
  __device__ __forceinline__ static void store(type* p, real v, real w) {
    *p = __float2half_rn(v - w);
  }
};

template <>
struct Pop<kBF16> {
  using type = __nv_bfloat16;
  using real = float;
  __device__ __forceinline__ static real load(const type* p, real w) {
    return __bfloat162float(*p) + w;
  }
  __device__ __forceinline__ static void store(type* p, real v, real w) {
    *p = __float2bfloat16_rn(v - w);
  }
};

template <>
struct Pop<kF64> {
  using type = double;
  using real = double;
  __device__ __forceinline__ static real load(const type* p, real) { return *p; }
  __device__ __forceinline__ static void store(type* p, real v, real) { *p = v; }
};

// Weight of slot i in the compute precision of the policy.
template <class L, class Real>
__host__ __device__ constexpr Real weight(int i) {
  if constexpr (sizeof(Real) == 8)
    return L::wd(i);
  else
    return L::w(i);
}

}  // namespace lbm
