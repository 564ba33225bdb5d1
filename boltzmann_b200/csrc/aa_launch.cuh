// Host-side dispatch of the AA kernel family for one fluid lattice. Included by one .cu file per
// lattice so the instantiations compile in parallel.
#pragma once

#include <cudaTypedefs.h>

#include <atomic>
#include <mutex>
#include <type_traits>

#include "aa_tma.cuh"
#include "aa_step.cuh"
#include "sim.h"

namespace lbm {

template <class Real>
StepArgs<Real> make_step_args(const lbm_sim& s, bool write_moments) {
  StepArgs<Real> a{};
  a.f = s.f;
  a.rho = static_cast<Real*>(s.rho);
  a.vel = static_cast<Real*>(s.vel);
  a.flags = s.flags;
  if (s.dim == 3) {
    a.nx = (int)s.counts[0];
    a.ny = (int)s.counts[1];
    a.nz = (int)s.counts[2];
  } else {
    a.nx = 1;
    a.ny = (int)s.counts[0];
    a.nz = (int)s.counts[1];
  }
  a.n = s.n;
  a.om_pos = s.om_pos;
  a.om_neg = s.om_neg;
  const int off = 3 - s.dim;
  // Acceleration source, as src/simulation.rs:326-373 leaves it for the fluid kernel: any
  // Boussinesq coupling overwrites the constant acceleration every step, the last one winning.
  if (!s.couplings.empty()) {
    const lbm_sim::Coupling& c = s.couplings.back();
    a.acc_mode = kAccBoussinesq;
    // (g b) / om_pos in the reference (src/lib.cl:72 then 254); b (g / om_pos) here: the same
    // shift up to one rounding of a term of the size of the buoyancy.
    for (int k = 0; k < s.dim; ++k) a.force[off + k] = (Real)c.g[k] / (Real)s.om_pos;
    a.alpha = c.alpha;
    a.c0 = c.c0;
    a.coupled = c.tracer;
    a.coupled_val = static_cast<const Real*>(s.tracers[c.tracer].val);
  } else if (s.has_gravity) {
    a.acc_mode = kAccConstant;
    // acc / om_pos, the division the reference makes per cell (src/lib.cl:254), made once.
    for (int k = 0; k < s.dim; ++k) a.force[off + k] = (Real)s.gravity[k] / (Real)s.om_pos;
  }
  a.ntracers = (int)s.tracers.size();
  for (int t = 0; t < a.ntracers; ++t) {
    a.tr[t].g = s.tracers[t].g;
    a.tr[t].val = static_cast<Real*>(s.tracers[t].val);
    a.tr[t].omega = s.tracers[t].omega;
    a.tr[t].omega_neg = s.tracers[t].omega_neg;
    a.tr[t].trt = s.tracers[t].collision == 1;
  }
  a.write_moments = write_moments ? 1 : 0;
  a.path = s.kernel_path;
  a.omega_field = s.omega_field;
  a.status = s.status;
  a.spin_limit = s.spin_limit < 0 ? kSpinLimit
                                  : (unsigned)(s.spin_limit < (int64_t)kSpinLimit ? s.spin_limit
                                                                                 : kSpinLimit);
  return a;
}

template <class Real>
void step_geometry(const StepArgs<Real>& a, dim3& grid, dim3& block) {
  const int bx = a.nz >= 256 ? 256 : ((a.nz + 31) / 32) * 32;
  block = dim3(bx, 1, 1);
  grid = dim3((a.nz + bx - 1) / bx, a.ny < 65535 ? a.ny : 65535, a.nx < 65535 ? a.nx : 65535);
}

// Ring depth of the TMA kernel: as many stages as fit in ~50 KB per CTA (2-4), so that three or
// four CTAs (24-32 consumer warps) share an SM and each keeps one or more tiles of copies in
// flight while it computes another.
template <class L, int K, int NT, bool EVEN, bool WR, int KT = default_tracer_kind<K>()>
constexpr int tma_stages() {
  constexpr size_t b = TmaStage<L, K, NT, EVEN, WR, KT>::bytes;
  constexpr int s = (int)((50 * 1024) / b);
  return s < 2 ? 2 : (s > 4 ? 4 : s);
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
inline PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

template <class T>
constexpr CUtensorMapDataType tensor_map_type() {
  if constexpr (sizeof(T) == 8) return CU_TENSOR_MAP_DATA_TYPE_FLOAT64;
  else if constexpr (sizeof(T) == 4) return CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  else if constexpr (std::is_same_v<T, __half>) return CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
  else return CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
}

// A [q slots][n cells] array (slot stride n elements) as a 2D tensor with a box of
// kTmaTile cells by all q slots. False when it cannot be described (the caller then copies row
// segments).
template <class T>
bool encode_slot_map(CUtensorMap* map, const void* base, long long n, int q) {
  auto encode = tensor_map_encoder();
  if (encode == nullptr || n >= (1ll << 31) || q > 256) return false;
  cuuint64_t dims[2] = {(cuuint64_t)n, (cuuint64_t)q};
  cuuint64_t strides[1] = {(cuuint64_t)n * sizeof(T)};
  if (strides[0] % 16 != 0 || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
  cuuint32_t box[2] = {(cuuint32_t)kTmaTile, (cuuint32_t)q};
  cuuint32_t elem[2] = {1, 1};
  return encode(map, tensor_map_type<T>(), 2, const_cast<void*>(base), dims, strides, box, elem,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// The population array as a 2D tensor of rows of nz cells, row (slot, x, y), with a box of one
// row of kTmaTile cells (the four-row copies of even steps of one-tile rows).
template <class T>
bool encode_row_map(CUtensorMap* map, const void* base, long long rows, int nz) {
  auto encode = tensor_map_encoder();
  if (encode == nullptr || rows >= (1ll << 31) || nz != kTmaTile) return false;
  cuuint64_t dims[2] = {(cuuint64_t)nz, (cuuint64_t)rows};
  cuuint64_t strides[1] = {(cuuint64_t)nz * sizeof(T)};
  if (strides[0] % 16 != 0 || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
  cuuint32_t box[2] = {(cuuint32_t)kTmaTile, 1};
  cuuint32_t elem[2] = {1, 1};
  return encode(map, tensor_map_type<T>(), 2, const_cast<void*>(base), dims, strides, box, elem,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <class L, bool TRT, int K, bool EVEN, int NT, bool WR, int KT>
cudaError_t launch_tma(const StepArgs<typename Pop<K>::real>& a, cudaStream_t stream) {
  constexpr int S = tma_stages<L, K, NT, EVEN, WR, KT>();
  constexpr size_t smem = tma_smem_bytes<L, K, NT, EVEN, S, WR, KT>();
  // Two cells a consumer thread with 16-bit populations: D3Q27 BGK without a tracer, on the
  // steps whose results go back through the stage (D3Q27 TRT needs more than the 128 registers
  // three CTAs a SM leave a thread, and spills); D2Q9 BGK / TRT with none or one fused tracer, on
  // every step.
  constexpr bool PAIR = dev_in<K>() && ((L::Q >= 27 && !TRT && NT == 0 && (!EVEN || WR)) ||
                                        (L::D == 2 && NT >= 0 && NT <= 1));
  constexpr int threads = tma_threads<PAIR>();
  auto kern = aa_tma_kernel<L, TRT, K, EVEN, NT, S, WR, PAIR, KT>;
  static std::once_flag once;
  static cudaError_t setup_err = cudaSuccess;
  static int per_sm = 1;
  std::call_once(once, [&] {
    setup_err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (setup_err == cudaSuccess)
      setup_err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (per_sm < 1) per_sm = 1;
  });
  if (setup_err != cudaSuccess) return setup_err;
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const long long tiles = (long long)a.nx * a.ny * (a.nz / kTmaTile);
  long long grid = (long long)sms * per_sm;
  if (grid > tiles) grid = tiles;
  TmaMaps maps{};
  if constexpr (EVEN && WR) {
    using T = typename Pop<K>::type;
    maps.use = encode_row_map<T>(&maps.f, a.f, (long long)L::Q * a.nx * a.ny, a.nz) ? 1 : 0;
  } else if constexpr (!EVEN) {
    using T = typename Pop<K>::type;
    using Real = typename Pop<K>::real;
    bool ok = encode_slot_map<T>(&maps.f, a.f, a.n, L::Q);
    if constexpr (NT == 1)
      ok = ok && encode_slot_map<typename TracerPop<KT>::type>(&maps.g, a.tr[0].g, a.n,
                                                              TracerLattice<L::D>::type::Q);
    maps.use = ok ? 1 : 0;
  }
  kern<<<(unsigned)grid, threads, smem, stream>>>(a, maps);
  return cudaGetLastError();
}

template <class L, bool TRT, int K, bool EVEN, int NT, int KT = default_tracer_kind<K>()>
cudaError_t launch_one(const StepArgs<typename Pop<K>::real>& a, cudaStream_t stream,
                       int64_t* launches) {
  // Rows that split into whole 256-cell tiles go through the TMA-staged kernel (fused tracers:
  // none or one); everything else through the direct kernel.
  // Small domains (under ~8 tiles per SM; they sit in L2 anyway) stay on the direct kernel,
  // whose launch has no ring to fill and drain.
  if constexpr (NT >= 0) {
    const long long tiles = (long long)a.nx * a.ny * (a.nz / kTmaTile);
    const bool fits = a.nz % kTmaTile == 0;
    const bool staged = a.path == 2 || (a.path == 0 && tiles >= 8LL * 148);
    if (fits && staged) {
      cudaError_t e;
      if (EVEN && a.nz == kTmaTile)
        e = launch_tma<L, TRT, K, EVEN, NT, EVEN, KT>(a, stream);
      else
        e = launch_tma<L, TRT, K, EVEN, NT, false, KT>(a, stream);
      if (e == cudaSuccess) ++launches[1];
      return e;
    }
  }
  dim3 grid, block;
  step_geometry(a, grid, block);
  aa_step_kernel<L, TRT, K, EVEN, NT, KT><<<grid, block, 0, stream>>>(a);
  const cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) ++launches[0];
  return e;
}

template <class L, bool TRT, int K>
cudaError_t launch_typed(const lbm_sim& s, bool even, bool write_moments) {
  using Real = typename Pop<K>::real;
  const StepArgs<Real> a = make_step_args<Real>(s, write_moments);
  // Fused tracers: none, exactly one (loads hoisted with the fluid's), or a runtime count.
  // 16-bit tracer populations (the fluid's own 16-bit kind) take the one-tracer path only.
  const int nt = a.ntracers;
  const bool t16 = s.tracer_storage == K && dev_in<K>();
  if (t16 && nt > 1) return cudaErrorNotSupported;
  if (even) {
    if (nt == 0) return launch_one<L, TRT, K, true, 0>(a, s.stream, s.launches);
    if (nt == 1) {
      if constexpr (dev_in<K>())
        if (t16) return launch_one<L, TRT, K, true, 1, K>(a, s.stream, s.launches);
      return launch_one<L, TRT, K, true, 1>(a, s.stream, s.launches);
    }
    return launch_one<L, TRT, K, true, -1>(a, s.stream, s.launches);
  }
  if (nt == 0) return launch_one<L, TRT, K, false, 0>(a, s.stream, s.launches);
  if (nt == 1) {
    if constexpr (dev_in<K>())
      if (t16) return launch_one<L, TRT, K, false, 1, K>(a, s.stream, s.launches);
    return launch_one<L, TRT, K, false, 1>(a, s.stream, s.launches);
  }
  return launch_one<L, TRT, K, false, -1>(a, s.stream, s.launches);
}

template <class L>
cudaError_t launch_lattice(const lbm_sim& s, bool even, bool write_moments) {
  const bool trt = s.collision == 1;
  switch (s.storage) {
    case kF32:
      return trt ? launch_typed<L, true, kF32>(s, even, write_moments)
                 : launch_typed<L, false, kF32>(s, even, write_moments);
    case kF16:
      return trt ? launch_typed<L, true, kF16>(s, even, write_moments)
                 : launch_typed<L, false, kF16>(s, even, write_moments);
    case kBF16:
      return trt ? launch_typed<L, true, kBF16>(s, even, write_moments)
                 : launch_typed<L, false, kBF16>(s, even, write_moments);
    case kF64:
      return trt ? launch_typed<L, true, kF64>(s, even, write_moments)
                 : launch_typed<L, false, kF64>(s, even, write_moments);
  }
  return cudaErrorInvalidValue;
}

}  // namespace lbm
