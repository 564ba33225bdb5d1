// lbm_population_sums_noalloc: the FP64 conservation sums of a caller-owned population array,
// with no device allocation at all.
//
// Why: some callers cannot allocate device memory -- code running inside another framework's
// memory arena, under an allocator that forbids extra cudaMalloc calls, or in a process whose
// memory budget is fixed before the solver is loaded. lbm_conservation() needs a simulation
// handle (whose creation allocates); this entry point only reads the caller's populations and
// writes the caller's output buffer.
//
// Scratch: the per-block partial sums live in the file-scope array `g_partials` below, a fixed
// kMaxBlocks x 4 doubles (64 KiB) that every GPU which loads this library holds until the process
// exits. One block reduces kCellsPerBlock cells, so one call handles at most
// kMaxBlocks * kCellsPerBlock = 134,217,728 cells; larger inputs are rejected.
//
// In host code `g_partials` names a host-side stand-in, not device memory: handing it to a kernel
// would fault, or, where the GPU can reach host memory, silently use the wrong memory. The device
// address is obtained once per device with cudaGetSymbolAddress (with that device current) on the
// first call there; make that first call before any stream capture begins. The address belongs to
// the device's context: when that context is destroyed and created again (cudaDeviceReset), the
// next call notices the new context (its unique id, cuCtxGetId) and looks the address up again.
//
// Every call on a device shares g_partials and it keeps the last call's contents. Each call
// overwrites every slot it later reads (nothing needs to start at zero), but two calls whose
// kernels overlap on the GPU (different streams, no ordering between them) race on the array.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>
#include <utility>

#include "../../include/lbm_cuda.h"
#include "lattice.cuh"
#include "sim.h"
#include "storage.cuh"

namespace {

constexpr int kMaxBlocks = 2048;
constexpr int64_t kCellsPerBlock = 65536;
constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_partials[kMaxBlocks][4];

struct SetWeights {
  float w[27];
  int8_t c[27][3];
  int q, d;
};

template <class L>
SetWeights make_weights() {
  SetWeights s{};
  s.q = L::Q;
  s.d = L::D;
  for (int i = 0; i < L::Q; ++i) {
    s.w[i] = L::w(i);
    for (int k = 0; k < 3; ++k) s.c[i][k] = (int8_t)(k < L::D ? L::c(i, k) : 0);
  }
  return s;
}

bool weights_of(int d, int q, SetWeights& out) {
  using namespace lbm;
  if (d == 1 && q == 3) out = make_weights<D1Q3>();
  else if (d == 2 && q == 9) out = make_weights<D2Q9>();
  else if (d == 2 && q == 5) out = make_weights<D2Q5>();
  else if (d == 3 && q == 7) out = make_weights<D3Q7>();
  else if (d == 3 && q == 27) out = make_weights<D3Q27>();
  else return false;
  return true;
}

// Pass 1: block b sums cells [b * kCellsPerBlock, (b + 1) * kCellsPerBlock) and overwrites
// partials[b][0..3] with (sum f, sum c_x f, sum c_y f, sum c_z f).
template <int K>
__global__ void __launch_bounds__(kThreads)
    block_sums(const typename lbm::Pop<K>::type* __restrict__ f, int64_t n, const SetWeights sw,
               double (*partials)[4]) {
  using P = lbm::Pop<K>;
  using Real = typename P::real;
  const int64_t begin = (int64_t)blockIdx.x * kCellsPerBlock;
  const int64_t end = begin + kCellsPerBlock < n ? begin + kCellsPerBlock : n;
  double acc[4] = {0, 0, 0, 0};
  for (int64_t cell = begin + threadIdx.x; cell < end; cell += kThreads) {
    for (int i = 0; i < sw.q; ++i) {
      const double v = (double)P::load(f + (int64_t)i * n + cell, (Real)sw.w[i]);
      acc[0] += v;
      for (int k = 0; k < sw.d; ++k) acc[1 + k] += sw.c[i][k] * v;
    }
  }
  __shared__ double warp_sums[kThreads / 32][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    double v = acc[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) warp_sums[warp][j] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0;
    for (int w = 0; w < kThreads / 32; ++w) v += warp_sums[w][threadIdx.x];
    partials[blockIdx.x][threadIdx.x] = v;
  }
}

// Pass 2: one block adds the first `blocks` partials in a fixed order and writes 1 + d outputs.
__global__ void __launch_bounds__(kThreads)
    final_sums(double (*partials)[4], int blocks, int d, double* __restrict__ out) {
  __shared__ double part[kThreads][4];
  double acc[4] = {0, 0, 0, 0};
  for (int b = threadIdx.x; b < blocks; b += kThreads)
    for (int j = 0; j < 4; ++j) acc[j] += partials[b][j];
  for (int j = 0; j < 4; ++j) part[threadIdx.x][j] = acc[j];
  __syncthreads();
  for (int stride = kThreads / 2; stride > 0; stride >>= 1) {
    if (threadIdx.x < stride)
      for (int j = 0; j < 4; ++j) part[threadIdx.x][j] += part[threadIdx.x + stride][j];
    __syncthreads();
  }
  if (threadIdx.x <= d) out[threadIdx.x] = part[0][threadIdx.x];
}

std::mutex g_setup_mutex;
void* g_scratch_address[kMaxDevices] = {};
unsigned long long g_scratch_context[kMaxDevices] = {};

// Unique id of the calling thread's current context (cuCtxGetId, through the runtime's driver
// entry points: no link against libcuda), or 0 when it cannot be read.
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static const auto fns = [] {
    void *cur = nullptr, *id = nullptr;
    cudaDriverEntryPointQueryResult q1{}, q2{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &cur, cudaEnableDefault, &q1) != cudaSuccess ||
        q1 != cudaDriverEntryPointSuccess)
      cur = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &id, cudaEnableDefault, &q2) != cudaSuccess ||
        q2 != cudaDriverEntryPointSuccess)
      id = nullptr;
    return std::make_pair(reinterpret_cast<GetCurrent>(cur), reinterpret_cast<GetId>(id));
  }();
  if (fns.first == nullptr || fns.second == nullptr) return 0;
  CUcontext ctx = nullptr;
  unsigned long long ident = 0;
  if (fns.first(&ctx) != CUDA_SUCCESS || ctx == nullptr) return 0;
  if (fns.second(ctx, &ident) != CUDA_SUCCESS) return 0;
  return ident;
}

// Device address of g_partials for the current device: looked up once per device, and again
// when the device's context has been re-created since.
int scratch_address(double (**out)[4]) {
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) {
    lbm::set_last_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    return LBM_ERR_CUDA;
  }
  if (device < 0 || device >= kMaxDevices) {
    lbm::set_last_error("device index out of range");
    return LBM_ERR_ARGUMENT;
  }
  // 0 when this thread has no current context yet (the look-up below binds the primary one).
  const unsigned long long ctx = current_context_id();
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (g_scratch_address[device] == nullptr || ctx == 0 || g_scratch_context[device] != ctx) {
    void* ptr = nullptr;
    e = cudaGetSymbolAddress(&ptr, g_partials);
    if (e != cudaSuccess || ptr == nullptr) {
      lbm::set_last_error(std::string("cudaGetSymbolAddress(g_partials): ") + cudaGetErrorString(e));
      return LBM_ERR_CUDA;
    }
    g_scratch_address[device] = ptr;
    g_scratch_context[device] = current_context_id();
  }
  *out = static_cast<double (*)[4]>(g_scratch_address[device]);
  return LBM_OK;
}

template <int K>
cudaError_t launch(const void* f, int64_t n, const SetWeights& sw, double (*scratch)[4],
                   int blocks, double* out, cudaStream_t stream) {
  block_sums<K><<<blocks, kThreads, 0, stream>>>(
      static_cast<const typename lbm::Pop<K>::type*>(f), n, sw, scratch);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  final_sums<<<1, kThreads, 0, stream>>>(scratch, blocks, sw.d, out);
  return cudaGetLastError();
}

}  // namespace

extern "C" {

int lbm_population_sums_noalloc(int dim, int q, int storage, const void* f, int64_t n,
                                double* out, void* stream) {
  SetWeights sw;
  if (!weights_of(dim, q, sw)) {
    lbm::set_last_error("Unknown model: D" + std::to_string(dim) + "Q" + std::to_string(q));
    return LBM_ERR_ARGUMENT;
  }
  if (storage < LBM_STORAGE_F32 || storage > LBM_STORAGE_F64) {
    lbm::set_last_error("unknown storage kind");
    return LBM_ERR_ARGUMENT;
  }
  if (f == nullptr || out == nullptr || n <= 0) {
    lbm::set_last_error("populations and output must be device pointers and n > 0");
    return LBM_ERR_ARGUMENT;
  }
  const int64_t blocks = (n + kCellsPerBlock - 1) / kCellsPerBlock;
  if (blocks > kMaxBlocks) {
    lbm::set_last_error("n = " + std::to_string(n) + " cells exceeds the maximum of " +
                      std::to_string((int64_t)kMaxBlocks * kCellsPerBlock) +
                      " for lbm_population_sums_noalloc (fixed scratch of " +
                      std::to_string(kMaxBlocks) + " partial sums)");
    return LBM_ERR_ARGUMENT;
  }
  double (*scratch)[4] = nullptr;
  if (int rc = scratch_address(&scratch)) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaSuccess;
  switch (storage) {
    case LBM_STORAGE_F32: e = launch<lbm::kF32>(f, n, sw, scratch, (int)blocks, out, s); break;
    case LBM_STORAGE_F16: e = launch<lbm::kF16>(f, n, sw, scratch, (int)blocks, out, s); break;
    case LBM_STORAGE_BF16: e = launch<lbm::kBF16>(f, n, sw, scratch, (int)blocks, out, s); break;
    case LBM_STORAGE_F64: e = launch<lbm::kF64>(f, n, sw, scratch, (int)blocks, out, s); break;
  }
  if (e != cudaSuccess) {
    lbm::set_last_error(std::string("kernel launch: ") + cudaGetErrorString(e));
    return LBM_ERR_CUDA;
  }
  return LBM_OK;
}

}  // extern "C"
