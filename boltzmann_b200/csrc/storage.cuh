// Population storage policies.
//
// F32 : populations stored as float, collided in float.
// F16 / BF16 : populations stored as the 16-bit offset f_i - w_i from the lattice weight,
//              widened to float for the collision and rounded to nearest on store; this halves
//              the bytes per cell update.
// F64 : populations and every operation in double (the on-GPU FP64 comparison run).
//
// load/store move full population values f_i. load_dev/store_dev move deviations
// d_i = f_i - W_i from the policy's offset W_i (the lattice weight in the compute precision):
// the collision works on deviations, so for F32/F64 storage f_i = W_i + d_i is rounded once on
// store, and for the 16-bit policies the stored value is the deviation itself.
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
  __device__ __forceinline__ static real load_dev(const type* p, real w) { return *p - w; }
  __device__ __forceinline__ static void store_dev(type* p, real d, real w) { *p = w + d; }
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
  __device__ __forceinline__ static real load_dev(const type* p, real) { return __half2float(*p); }
  __device__ __forceinline__ static void store_dev(type* p, real d, real) {
    *p = __float2half_rn(d);
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
  __device__ __forceinline__ static real load_dev(const type* p, real) {
    return __bfloat162float(*p);
  }
  __device__ __forceinline__ static void store_dev(type* p, real d, real) {
    *p = __float2bfloat16_rn(d);
  }
};

template <>
struct Pop<kF64> {
  using type = double;
  using real = double;
  __device__ __forceinline__ static real load(const type* p, real) { return *p; }
  __device__ __forceinline__ static void store(type* p, real v, real) { *p = v; }
  __device__ __forceinline__ static real load_dev(const type* p, real w) { return *p - w; }
  __device__ __forceinline__ static void store_dev(type* p, real d, real w) { *p = w + d; }
};

// Storage of tracer populations: the compute type (float, or double for FP64 runs), or 16-bit
// values stored as they are -- a concentration spans 0 .. 1, so no fixed offset shrinks the stored
// magnitudes -- widened to float for the update and rounded to nearest on store. The weight
// argument is ignored (it is the fluid policies' offset).
template <int KT>
struct TracerPop;
template <>
struct TracerPop<kF32> : Pop<kF32> {};
template <>
struct TracerPop<kF64> : Pop<kF64> {};
template <>
struct TracerPop<kF16> {
  using type = __half;
  using real = float;
  __device__ __forceinline__ static real load(const type* p, real) { return __half2float(*p); }
  __device__ __forceinline__ static void store(type* p, real v, real) { *p = __float2half_rn(v); }
};
template <>
struct TracerPop<kBF16> {
  using type = __nv_bfloat16;
  using real = float;
  __device__ __forceinline__ static real load(const type* p, real) { return __bfloat162float(*p); }
  __device__ __forceinline__ static void store(type* p, real v, real) {
    *p = __float2bfloat16_rn(v);
  }
};

// Tracer storage when none is chosen: the fluid's compute type.
template <int K>
__host__ __device__ constexpr int default_tracer_kind() {
  return K == kF64 ? kF64 : kF32;
}

// 16-bit kinds store deviations f_i - W_i; the update takes them as loaded, without forming the
// full values (their rounding, ~1e-3 relative, dwarfs any FP32 ordering effect). FP32 and FP64
// load full values, whose momentum sum is the reference's.
template <int K>
__host__ __device__ constexpr bool dev_in() {
  return K == kF16 || K == kBF16;
}

// Weight of slot i in the compute precision of the policy.
template <class L, class Real>
__host__ __device__ constexpr Real weight(int i) {
  if constexpr (sizeof(Real) == 8)
    return L::wd(i);
  else
    return L::w(i);
}

// Sum of the offsets minus one (the float weights sum to 1 + O(1e-8)); and the per-slot gap
// between the exact weight wk/kDen and the offset W_i. Both are compile-time constants.
template <class L, class Real>
__host__ __device__ constexpr Real weight_defect() {
  double s = 0;
  for (int i = 0; i < L::Q; ++i) s += (double)weight<L, Real>(i);
  return (Real)(s - 1.0);
}

template <class L, class Real>
__host__ __device__ constexpr Real weight_gap(int i) {
  return (Real)((double)L::wk(i) / (double)L::kDen - (double)weight<L, Real>(i));
}

// 1 / kDen as an unevaluated sum hi + lo of two values of the compute precision. x * (1/kDen)
// evaluated as fma(x, hi, x * lo) is then the correctly rounded quotient up to a few units of
// 2^-48 relative: unbiased like a division, at the cost of two instructions. (A single rounded
// constant would scale every equilibrium weight by the same (1 + eps): a systematic mass drift.)
template <class L, class Real>
__host__ __device__ constexpr Real inv_den_hi() {
  return (Real)(1.0 / (double)L::kDen);
}

template <class L, class Real>
__host__ __device__ constexpr Real inv_den_lo() {
  return (Real)(1.0 / (double)L::kDen - (double)inv_den_hi<L, Real>());
}

template <class L, class Real>
__device__ __forceinline__ Real over_den(Real x) {
  if constexpr (sizeof(Real) == 8)
    return x / Real(L::kDen);
  else
    return fmaf(x, inv_den_hi<L, Real>(), x * inv_den_lo<L, Real>());
}

}  // namespace lbm
