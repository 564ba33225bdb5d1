// Field kernels around the AA step: equilibrium initialisation, checkpoint-layout transposes,
// precision conversions and the FP64 conservation sums.
#include <cstdint>

#include "aa_step.cuh"
#include "sim.h"

namespace lbm {
namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(int64_t n) {
  int64_t b = (n + kThreads - 1) / kThreads;
  return (unsigned)(b < 148 * 64 ? (b > 0 ? b : 1) : 148 * 64);
}

// FP32 equilibrium in the exact operation order of src/velocities.rs:43-52 (no contraction):
//   feq_i = (rho * w_i) * (((1 + 3 vq) + (4.5 vq) vq) - 1.5 vv),
//   vq = (0 + u_0 c_i0) + u_1 c_i1 ..., vv = (0 + u_0 u_0) + u_1 u_1 ...
template <class L>
__device__ __forceinline__ float feq_f32(int i, float rho, const float* u) {
  float vv = 0.0f, vq = 0.0f;
#pragma unroll
  for (int k = 0; k < L::D; ++k) {
    vv = __fadd_rn(vv, __fmul_rn(u[k], u[k]));
    vq = __fadd_rn(vq, __fmul_rn(u[k], (float)L::c(i, k)));
  }
  float poly = __fadd_rn(1.0f, __fmul_rn(3.0f, vq));
  poly = __fadd_rn(poly, __fmul_rn(__fmul_rn(4.5f, vq), vq));
  poly = __fsub_rn(poly, __fmul_rn(1.5f, vv));
  return __fmul_rn(__fmul_rn(rho, L::w(i)), poly);
}

template <class L>
__device__ __forceinline__ double feq_f64(int i, double rho, const double* u) {
  double vv = 0.0, vq = 0.0;
#pragma unroll
  for (int k = 0; k < L::D; ++k) {
    vv += u[k] * u[k];
    vq += u[k] * L::c(i, k);
  }
  return rho * L::wd(i) * (1.0 + 3.0 * vq + 4.5 * vq * vq - 1.5 * vv);
}

// f[i*n + cell] = feq_i(rho[cell], vel[cell]) for one velocity set L and storage K (16-bit
// kinds: the offset f_i - w_i; RAW: the value itself, for 16-bit tracer populations).
template <class L, int K, bool RAW = false>
__global__ void equilibrate_kernel(typename Pop<K>::type* __restrict__ f,
                                   const typename Pop<K>::real* __restrict__ rho,
                                   const typename Pop<K>::real* __restrict__ vel, int64_t n) {
  using P = Pop<K>;
  using Real = typename P::real;
  for (int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; cell < n;
       cell += (int64_t)gridDim.x * blockDim.x) {
    Real u[3];
#pragma unroll
    for (int k = 0; k < L::D; ++k) u[k] = vel[cell * L::D + k];
    const Real r = rho[cell];
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
      Real fe;
      if constexpr (sizeof(Real) == 8)
        fe = feq_f64<L>(i, r, u);
      else
        fe = feq_f32<L>(i, r, u);
      P::store(f + (int64_t)i * n + cell, fe, RAW ? Real(0) : weight<L, Real>(i));
    }
  }
}

template <class L, int K, bool RAW>
cudaError_t equilibrate_set(void* f, const void* rho, const void* vel, int64_t n, cudaStream_t s) {
  using P = Pop<K>;
  equilibrate_kernel<L, K, RAW><<<blocks_for(n), kThreads, 0, s>>>(
      static_cast<typename P::type*>(f), static_cast<const typename P::real*>(rho),
      static_cast<const typename P::real*>(vel), n);
  return cudaGetLastError();
}

template <class L, bool RAW>
cudaError_t equilibrate_storage(int storage, void* f, const void* rho, const void* vel, int64_t n,
                                cudaStream_t s) {
  switch (storage) {
    case kF32: return equilibrate_set<L, kF32, false>(f, rho, vel, n, s);
    case kF16: return equilibrate_set<L, kF16, RAW>(f, rho, vel, n, s);
    case kBF16: return equilibrate_set<L, kBF16, RAW>(f, rho, vel, n, s);
    case kF64: return equilibrate_set<L, kF64, false>(f, rho, vel, n, s);
  }
  return cudaErrorInvalidValue;
}

// `storage` is the storage kind of the buffer f (the fluid's kind, or the tracers'); `raw`: a
// 16-bit buffer holds the values themselves (tracer populations), not offsets from the weights.
cudaError_t equilibrate_any(int d, int q, int storage, void* f, const void* rho, const void* vel,
                            int64_t n, cudaStream_t s, bool raw = false) {
  if (raw) {
    if (d == 2 && q == 5) return equilibrate_storage<D2Q5, true>(storage, f, rho, vel, n, s);
    if (d == 3 && q == 7) return equilibrate_storage<D3Q7, true>(storage, f, rho, vel, n, s);
    return cudaErrorNotSupported;
  }
  if (d == 1 && q == 3) return equilibrate_storage<D1Q3, false>(storage, f, rho, vel, n, s);
  if (d == 2 && q == 9) return equilibrate_storage<D2Q9, false>(storage, f, rho, vel, n, s);
  if (d == 2 && q == 5) return equilibrate_storage<D2Q5, false>(storage, f, rho, vel, n, s);
  if (d == 3 && q == 7) return equilibrate_storage<D3Q7, false>(storage, f, rho, vel, n, s);
  if (d == 3 && q == 27) return equilibrate_storage<D3Q27, false>(storage, f, rho, vel, n, s);
  return cudaErrorNotSupported;
}

inline int tracer_storage(const lbm_sim& sim) { return sim.tracer_kind(); }
// 16-bit tracer populations are stored as values, so their layout transposes and sums take zero
// offsets.
inline bool tracer_raw(const lbm_sim& sim) {
  return sim.tracer_kind() == kF16 || sim.tracer_kind() == kBF16;
}

// Per-slot weights of any velocity set, for the offset encodings of the layout transposes.
struct SlotWeights {
  float w[27];
  int8_t c[27][3];
};

template <class L>
SlotWeights slot_weights() {
  SlotWeights sw{};
  for (int i = 0; i < L::Q; ++i) {
    sw.w[i] = L::w(i);
    for (int k = 0; k < 3; ++k) sw.c[i][k] = (int8_t)(k < L::D ? L::c(i, k) : 0);
  }
  return sw;
}

bool weights_for(int d, int q, SlotWeights& out) {
  if (d == 1 && q == 3) out = slot_weights<D1Q3>();
  else if (d == 2 && q == 9) out = slot_weights<D2Q9>();
  else if (d == 3 && q == 27) out = slot_weights<D3Q27>();
  else if (d == 2 && q == 5) out = slot_weights<D2Q5>();
  else if (d == 3 && q == 7) out = slot_weights<D3Q7>();
  else return false;
  return true;
}

// [n][q] float  <->  [q][n] storage
template <int K, bool TO_SOA>
__global__ void transpose_kernel(typename Pop<K>::type* __restrict__ soa, float* __restrict__ aos,
                                 int64_t n, int q, const SlotWeights sw) {
  using P = Pop<K>;
  using Real = typename P::real;
  for (int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; cell < n;
       cell += (int64_t)gridDim.x * blockDim.x) {
    for (int i = 0; i < q; ++i) {
      if constexpr (TO_SOA)
        P::store(soa + (int64_t)i * n + cell, (Real)aos[cell * q + i], (Real)sw.w[i]);
      else
        aos[cell * q + i] = (float)P::load(soa + (int64_t)i * n + cell, (Real)sw.w[i]);
    }
  }
}

template <bool TO_SOA>
cudaError_t transpose(int storage, void* soa, float* aos, int64_t n, int q, const SlotWeights& sw,
                      cudaStream_t s) {
  const unsigned b = blocks_for(n);
  switch (storage) {
    case kF32:
      transpose_kernel<kF32, TO_SOA><<<b, kThreads, 0, s>>>((float*)soa, aos, n, q, sw);
      break;
    case kF16:
      transpose_kernel<kF16, TO_SOA><<<b, kThreads, 0, s>>>((__half*)soa, aos, n, q, sw);
      break;
    case kBF16:
      transpose_kernel<kBF16, TO_SOA><<<b, kThreads, 0, s>>>((__nv_bfloat16*)soa, aos, n, q, sw);
      break;
    case kF64:
      transpose_kernel<kF64, TO_SOA><<<b, kThreads, 0, s>>>((double*)soa, aos, n, q, sw);
      break;
    default:
      return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

__global__ void narrow_kernel(const double* __restrict__ src, float* __restrict__ dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}

// Low four CellFlags bits of the int32 host layout (WALL, FIXED_FLUID_*, FIXED_SCALAR_VALUE).
__global__ void flags_kernel(const int32_t* __restrict__ src, uint8_t* __restrict__ dst,
                             int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (uint8_t)(src[i] & 0xF);
}

__global__ void widen_kernel(const float* __restrict__ src, double* __restrict__ dst, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}

template <class T>
__global__ void fill_kernel(T* __restrict__ dst, int64_t n, T v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = v;
}

// FP64 sums over all population slots of one set: out[0] += sum f, out[1+k] += sum c_ik f.
// Each warp reduces with shuffles, then lane 0 adds the warp's partials atomically.
template <int K>
__global__ void sums_kernel(const typename Pop<K>::type* __restrict__ f, int64_t n, int q, int d,
                            const SlotWeights sw, double* __restrict__ out, int nout) {
  using P = Pop<K>;
  using Real = typename P::real;
  double acc[4] = {0, 0, 0, 0};
  for (int64_t cell = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; cell < n;
       cell += (int64_t)gridDim.x * blockDim.x) {
    for (int i = 0; i < q; ++i) {
      const double v = (double)P::load(f + (int64_t)i * n + cell, (Real)sw.w[i]);
      acc[0] += v;
      for (int k = 0; k < d; ++k) acc[1 + k] += sw.c[i][k] * v;
    }
  }
  for (int j = 0; j < nout; ++j) {
    double v = acc[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(out + j, v);
  }
}

cudaError_t sums(int storage, const void* f, int64_t n, int q, int d, const SlotWeights& sw,
                 double* out, int nout, cudaStream_t s) {
  const unsigned b = blocks_for(n);
  switch (storage) {
    case kF32: sums_kernel<kF32><<<b, kThreads, 0, s>>>((const float*)f, n, q, d, sw, out, nout); break;
    case kF16: sums_kernel<kF16><<<b, kThreads, 0, s>>>((const __half*)f, n, q, d, sw, out, nout); break;
    case kBF16:
      sums_kernel<kBF16><<<b, kThreads, 0, s>>>((const __nv_bfloat16*)f, n, q, d, sw, out, nout);
      break;
    case kF64: sums_kernel<kF64><<<b, kThreads, 0, s>>>((const double*)f, n, q, d, sw, out, nout); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace

cudaError_t equilibrate(const lbm_sim& sim) {
  cudaError_t e = equilibrate_any(sim.dim, sim.q, sim.storage, sim.f, sim.rho, sim.vel, sim.n,
                                  sim.stream);
  if (e != cudaSuccess) return e;
  for (const lbm_sim::Tracer& t : sim.tracers) {
    e = equilibrate_any(sim.dim, t.q, tracer_storage(sim), t.g, t.val, sim.vel, sim.n, sim.stream,
                        tracer_raw(sim));
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t equilibrate_tracer(const lbm_sim& sim, int tracer) {
  const lbm_sim::Tracer& t = sim.tracers[tracer];
  return equilibrate_any(sim.dim, t.q, tracer_storage(sim), t.g, t.val, sim.vel, sim.n,
                         sim.stream, tracer_raw(sim));
}

cudaError_t populations_from_aos(const lbm_sim& sim, int tracer, const float* d_aos) {
  SlotWeights sw{};
  if (tracer < 0) {
    if (!weights_for(sim.dim, sim.q, sw)) return cudaErrorNotSupported;
    return transpose<true>(sim.storage, sim.f, const_cast<float*>(d_aos), sim.n, sim.q, sw,
                           sim.stream);
  }
  const lbm_sim::Tracer& t = sim.tracers[tracer];
  if (!weights_for(sim.dim, t.q, sw)) return cudaErrorNotSupported;
  if (tracer_raw(sim)) sw = SlotWeights{};
  return transpose<true>(tracer_storage(sim), t.g, const_cast<float*>(d_aos), sim.n,
                         t.q, sw, sim.stream);
}

cudaError_t populations_to_aos(const lbm_sim& sim, int tracer, float* d_aos) {
  SlotWeights sw{};
  if (tracer < 0) {
    if (!weights_for(sim.dim, sim.q, sw)) return cudaErrorNotSupported;
    return transpose<false>(sim.storage, sim.f, d_aos, sim.n, sim.q, sw, sim.stream);
  }
  const lbm_sim::Tracer& t = sim.tracers[tracer];
  if (!weights_for(sim.dim, t.q, sw)) return cudaErrorNotSupported;
  if (tracer_raw(sim)) sw = SlotWeights{};
  return transpose<false>(tracer_storage(sim), t.g, d_aos, sim.n, t.q, sw,
                          sim.stream);
}

cudaError_t narrow_to_float(const double* src, float* dst, int64_t count, cudaStream_t s) {
  narrow_kernel<<<blocks_for(count), kThreads, 0, s>>>(src, dst, count);
  return cudaGetLastError();
}

cudaError_t flags_to_u8(const int32_t* src, uint8_t* dst, int64_t count, cudaStream_t s) {
  flags_kernel<<<blocks_for(count), kThreads, 0, s>>>(src, dst, count);
  return cudaGetLastError();
}

cudaError_t widen_to_double(const float* src, double* dst, int64_t count, cudaStream_t s) {
  widen_kernel<<<blocks_for(count), kThreads, 0, s>>>(src, dst, count);
  return cudaGetLastError();
}

cudaError_t fill_value(void* dst, int64_t count, double value, bool is_double, cudaStream_t s) {
  if (is_double)
    fill_kernel<double><<<blocks_for(count), kThreads, 0, s>>>((double*)dst, count, value);
  else
    fill_kernel<float><<<blocks_for(count), kThreads, 0, s>>>((float*)dst, count, (float)value);
  return cudaGetLastError();
}

cudaError_t conservation_sums(const lbm_sim& sim, double* d_out) {
  SlotWeights sw{};
  if (!weights_for(sim.dim, sim.q, sw)) return cudaErrorNotSupported;
  cudaError_t e = sums(sim.storage, sim.f, sim.n, sim.q, sim.dim, sw, d_out, 1 + sim.dim,
                       sim.stream);
  if (e != cudaSuccess) return e;
  for (size_t t = 0; t < sim.tracers.size(); ++t) {
    const lbm_sim::Tracer& tr = sim.tracers[t];
    if (!weights_for(sim.dim, tr.q, sw)) return cudaErrorNotSupported;
    if (tracer_raw(sim))
      for (int i = 0; i < 27; ++i) sw.w[i] = 0.0f;  // values, not offsets (the c_i stay)
    e = sums(tracer_storage(sim), tr.g, sim.n, tr.q, sim.dim, sw,
             d_out + 1 + sim.dim + t, 1, sim.stream);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace lbm
