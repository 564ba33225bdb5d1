// C ABI of include/lbm_cuda.h: simulation lifetime, transfers and the per-step launch loop.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "../../include/lbm_cuda.h"
#include "aa_step.cuh"
#include "sim.h"

namespace {

thread_local std::string g_error;

int fail(int code, const std::string& msg) {
  g_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  return fail(LBM_ERR_CUDA, std::string("CUDA error in ") + where + ": " + cudaGetErrorName(e) +
                                " (" + cudaGetErrorString(e) + ")");
}

#define LBM_CUDA(call)                                \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

// Velocity sets known to the reference (src/velocities.rs:55-64).
bool known_set(int d, int q) {
  return (d == 1 && q == 3) || (d == 2 && (q == 9 || q == 5)) || (d == 3 && (q == 7 || q == 27));
}

// Sets that have a fluid update kernel (src/opencl.rs:123-129, plus D3Q27 TRT).
bool fluid_kernel(int d, int q) { return (d == 2 && q == 9) || (d == 3 && q == 27); }

// Sets that have a tracer update kernel: D2Q5 / D3Q7 with BGK (src/opencl.rs:123-129) or TRT
// (the kernels python/boltzmann/kernel_gen.py:250-462 generates, which the reference never
// registers).
bool tracer_kernel(int d, int q, int collision) {
  return (collision == LBM_BGK || collision == LBM_TRT) && ((d == 2 && q == 5) || (d == 3 && q == 7));
}

int activate(lbm_sim* s) {
  if (s == nullptr) return fail(LBM_ERR_ARGUMENT, "null simulation handle");
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return cuda_fail(e, "cudaSetDevice");
  return LBM_OK;
}

int check_tracer(lbm_sim* s, int t) {
  if (t < 0 || t >= (int)s->tracers.size()) return fail(LBM_ERR_ARGUMENT, "no such tracer index");
  return LBM_OK;
}

// Host float -> device real (float, or double through a temporary for F64).
int upload_reals(lbm_sim* s, void* dst, const float* src, int64_t count) {
  if (s->storage != LBM_STORAGE_F64) {
    LBM_CUDA(cudaMemcpyAsync(dst, src, count * sizeof(float), cudaMemcpyHostToDevice, s->stream));
    return LBM_OK;
  }
  float* tmp = nullptr;
  LBM_CUDA(cudaMallocAsync((void**)&tmp, count * sizeof(float), s->stream));
  LBM_CUDA(cudaMemcpyAsync(tmp, src, count * sizeof(float), cudaMemcpyHostToDevice, s->stream));
  LBM_CUDA(lbm::widen_to_double(tmp, static_cast<double*>(dst), count, s->stream));
  LBM_CUDA(cudaFreeAsync(tmp, s->stream));
  return LBM_OK;
}

// Device real -> host float.
int download_reals(lbm_sim* s, float* dst, const void* src, int64_t count) {
  if (s->storage != LBM_STORAGE_F64) {
    LBM_CUDA(cudaMemcpyAsync(dst, src, count * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
    return LBM_OK;
  }
  float* tmp = nullptr;
  LBM_CUDA(cudaMallocAsync((void**)&tmp, count * sizeof(float), s->stream));
  LBM_CUDA(lbm::narrow_to_float(static_cast<const double*>(src), tmp, count, s->stream));
  LBM_CUDA(cudaMemcpyAsync(dst, tmp, count * sizeof(float), cudaMemcpyDeviceToHost, s->stream));
  LBM_CUDA(cudaFreeAsync(tmp, s->stream));
  return LBM_OK;
}

// Reads the device status word after a synchronisation: bit 1 means a kernel gave up waiting for
// its own asynchronous copies (it then stopped early and the state is not valid).
int check_status(lbm_sim* s) {
  int word = 0;
  LBM_CUDA(cudaMemcpyAsync(&word, s->status, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  LBM_CUDA(cudaStreamSynchronize(s->stream));
  if (word & 2) {
    // Reported once: the bit is cleared so that the simulation can be restored and run again.
    const int rest = word & ~2;
    LBM_CUDA(cudaMemcpyAsync(s->status, &rest, sizeof(int), cudaMemcpyHostToDevice, s->stream));
    LBM_CUDA(cudaStreamSynchronize(s->stream));
    return fail(LBM_ERR_CUDA, "an AA step gave up waiting for its staged copies (status bit 1)");
  }
  return LBM_OK;
}

// The captured step graphs no longer match the simulation's state.
void drop_graph(lbm_sim* s) {
  for (const lbm_sim::StepGraph& g : s->graphs) cudaGraphExecDestroy(g.exec);
  s->graphs.clear();
  s->graph_warm = false;
  s->graph_failed = false;
}

void release(lbm_sim* s) {
  drop_graph(s);
  for (lbm_sim::Tracer& t : s->tracers) {
    cudaFree(t.g);
    cudaFree(t.val);
  }
  cudaFree(s->f);
  cudaFree(s->rho);
  cudaFree(s->vel);
  cudaFree(s->flags);
  cudaFree(s->status);
  if (s->stream) cudaStreamDestroy(s->stream);
}

}  // namespace

namespace {

// Step pairs in one captured graph: at most kGraphPairs, at least kMinGraphPairs. Small domains
// take a few microseconds a step, as long as a launch takes on the host, and a replayed graph
// issues its launches back to back; but a replay has a start-up latency of its own on the GPU,
// which shorter graphs do not repay (a learned closure's loop of 10-step calls between its own
// kernels measured 5% slower with graphs of 4 pairs).
constexpr int64_t kGraphPairs = 16, kMinGraphPairs = 8;

// One AA step pair (even, odd); the odd step writes rho / vel when `last`
// (src/simulation.rs:350: even steps are the iteration counter's even values).
cudaError_t launch_pair(lbm_sim* s, bool last) {
  for (int k = 0; k < 2; ++k) {
    const bool even = k == 0, moments = last && !even;
    const cudaError_t e = s->dim == 2 ? lbm::launch_step_d2q9(*s, even, moments)
                                      : lbm::launch_step_d3q27(*s, even, moments);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// The graph of `pairs` step pairs (no moments written), captured from the simulation's stream if
// it is not cached yet; null when the capture fails. The launch counters the capture advanced are
// put back and kept per replay.
const lbm_sim::StepGraph* step_graph(lbm_sim* s, int64_t pairs) {
  for (const lbm_sim::StepGraph& g : s->graphs)
    if (g.pairs == pairs) return &g;
  if (s->graphs.size() >= 4) {
    cudaGraphExecDestroy(s->graphs.front().exec);
    s->graphs.erase(s->graphs.begin());
  }
  lbm_sim::StepGraph g{pairs, nullptr, {0, 0}};
  const int64_t before[2] = {s->launches[0], s->launches[1]};
  cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return nullptr;
  cudaError_t le = cudaSuccess;
  for (int64_t p = 0; p < pairs && le == cudaSuccess; ++p) le = launch_pair(s, false);
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(s->stream, &graph);
  for (int k = 0; k < 2; ++k) {
    g.launches[k] = s->launches[k] - before[k];
    s->launches[k] = before[k];
  }
  if (le == cudaSuccess && e == cudaSuccess) e = cudaGraphInstantiate(&g.exec, graph, 0);
  if (graph) cudaGraphDestroy(graph);
  if (le != cudaSuccess || e != cudaSuccess) return nullptr;
  s->graphs.push_back(g);
  return &s->graphs.back();
}

int step_launch_fail(cudaError_t e) {
  if (e == cudaErrorNotSupported)
    return fail(LBM_ERR_UNSUPPORTED, "16-bit tracer storage takes one tracer");
  return cuda_fail(e, "AA step launch");
}

}  // namespace

void lbm::set_last_error(const std::string& msg) { g_error = msg; }

extern "C" {

const char* lbm_last_error(void) { return g_error.c_str(); }

int lbm_abi_version(void) { return 1; }

int lbm_create(int dim, const int64_t* counts, int q, int collision, float omega_pos,
               float omega_neg, int storage, lbm_sim** out) {
  if (out == nullptr || counts == nullptr) return fail(LBM_ERR_ARGUMENT, "null argument");
  *out = nullptr;
  if (dim < 1 || dim > 3)
    return fail(LBM_ERR_ARGUMENT, "Invalid number of dimensions. Expected either 1, 2 or 3.");
  if (!known_set(dim, q))
    return fail(LBM_ERR_ARGUMENT,
                "Unknown model: D" + std::to_string(dim) + "Q" + std::to_string(q));
  if (collision != LBM_BGK && collision != LBM_TRT)
    return fail(LBM_ERR_ARGUMENT, "unknown collision operator");
  if (storage < LBM_STORAGE_F32 || storage > LBM_STORAGE_F64)
    return fail(LBM_ERR_ARGUMENT, "unknown storage kind");
  int64_t n = 1;
  for (int k = 0; k < dim; ++k) {
    if (counts[k] <= 0 || counts[k] > (1 << 30))
      return fail(LBM_ERR_ARGUMENT, "cell counts must be positive");
    n *= counts[k];
  }
  // Kernels index cells with 32-bit offsets (populations are addressed per direction).
  if (n >= ((int64_t)1 << 32)) return fail(LBM_ERR_ARGUMENT, "domain too large (2^32 cells)");

  lbm_sim* s = new (std::nothrow) lbm_sim();
  if (s == nullptr) return fail(LBM_ERR_ARGUMENT, "out of host memory");
  s->dim = dim;
  s->q = q;
  s->collision = collision;
  s->storage = storage;
  for (int k = 0; k < dim; ++k) s->counts[k] = counts[k];
  s->n = n;
  s->om_pos = omega_pos;
  s->om_neg = omega_neg;

  auto bail = [&](cudaError_t e, const char* where) {
    release(s);
    delete s;
    return cuda_fail(e, where);
  };
  cudaError_t e = cudaGetDevice(&s->device);
  if (e != cudaSuccess) return bail(e, "cudaGetDevice");
  e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return bail(e, "cudaStreamCreate");
  const size_t rb = s->real_bytes();
  if ((e = cudaMalloc(&s->f, (size_t)n * q * lbm::pop_bytes(storage))) != cudaSuccess)
    return bail(e, "cudaMalloc(f)");
  if ((e = cudaMalloc(&s->rho, (size_t)n * rb)) != cudaSuccess) return bail(e, "cudaMalloc(rho)");
  if ((e = cudaMalloc(&s->vel, (size_t)n * dim * rb)) != cudaSuccess)
    return bail(e, "cudaMalloc(vel)");
  // Flags are padded to whole 256-byte blocks: kernels read them as aligned 4-byte words.
  const size_t flag_bytes = ((size_t)n + 255) / 256 * 256;
  if ((e = cudaMalloc((void**)&s->flags, flag_bytes)) != cudaSuccess)
    return bail(e, "cudaMalloc(flags)");
  if ((e = cudaMalloc((void**)&s->status, 64 * sizeof(double))) != cudaSuccess)
    return bail(e, "cudaMalloc(status)");
  s->sums = reinterpret_cast<double*>(s->status) + 1;  // 63 doubles after the status word
  s->sums_len = 63;
  // Reference defaults (src/fields.rs:75-77, src/simulation.rs:35): f = 0, rho = 1, vel = 0,
  // flags = 0.
  if ((e = cudaMemsetAsync(s->f, 0, (size_t)n * q * lbm::pop_bytes(storage), s->stream)) ||
      (e = lbm::fill_value(s->rho, n, 1.0, storage == LBM_STORAGE_F64, s->stream)) ||
      (e = cudaMemsetAsync(s->vel, 0, (size_t)n * dim * rb, s->stream)) ||
      (e = cudaMemsetAsync(s->flags, 0, flag_bytes, s->stream)) ||
      (e = cudaMemsetAsync(s->status, 0, 64 * sizeof(double), s->stream)) ||
      (e = cudaStreamSynchronize(s->stream)))
    return bail(e, "initialise fields");
  *out = s;
  return LBM_OK;
}

int lbm_destroy(lbm_sim* sim) {
  if (sim == nullptr) return LBM_OK;
  cudaSetDevice(sim->device);
  cudaStreamSynchronize(sim->stream);
  release(sim);
  delete sim;
  return LBM_OK;
}

int lbm_device_info(lbm_sim* sim, char* buf, int len) {
  if (int rc = activate(sim)) return rc;
  cudaDeviceProp p;
  LBM_CUDA(cudaGetDeviceProperties(&p, sim->device));
  if (buf && len > 0) std::snprintf(buf, (size_t)len, "NVIDIA %s GPU", p.name);
  return LBM_OK;
}

int lbm_device_bytes(lbm_sim* sim, int64_t* out) {
  if (int rc = activate(sim)) return rc;
  const int64_t n = sim->n, rb = (int64_t)sim->real_bytes();
  int64_t b = n * sim->q * (int64_t)lbm::pop_bytes(sim->storage) + n * rb * (1 + sim->dim) + n;
  for (const lbm_sim::Tracer& t : sim->tracers)
    b += n * (int64_t)sim->tracer_pop_bytes() * t.q + n * rb;
  *out = b;
  return LBM_OK;
}

int lbm_add_tracer(lbm_sim* sim, int q, int collision, float omega_pos, float omega_neg,
                   int* out_index) {
  if (int rc = activate(sim)) return rc;
  if (!known_set(sim->dim, q))
    return fail(LBM_ERR_ARGUMENT,
                "Unknown model: D" + std::to_string(sim->dim) + "Q" + std::to_string(q));
  if ((int)sim->tracers.size() >= lbm::kMaxTracers)
    return fail(LBM_ERR_UNSUPPORTED, "at most " + std::to_string(lbm::kMaxTracers) +
                                         " tracers per simulation");
  lbm_sim::Tracer t;
  t.q = q;
  t.collision = collision;
  t.omega = omega_pos;
  t.omega_neg = omega_neg;
  if (sim->tracer_storage >= 0 && !sim->tracers.empty())
    return fail(LBM_ERR_UNSUPPORTED, "16-bit tracer storage takes one tracer");
  const size_t rb = sim->real_bytes(), gb = sim->tracer_pop_bytes();
  LBM_CUDA(cudaMalloc(&t.g, (size_t)sim->n * q * gb));
  cudaError_t e = cudaMalloc(&t.val, (size_t)sim->n * rb);
  if (e != cudaSuccess) {
    cudaFree(t.g);
    return cuda_fail(e, "cudaMalloc(tracer val)");
  }
  LBM_CUDA(cudaMemsetAsync(t.g, 0, (size_t)sim->n * q * gb, sim->stream));
  LBM_CUDA(cudaMemsetAsync(t.val, 0, (size_t)sim->n * rb, sim->stream));
  sim->tracers.push_back(t);
  drop_graph(sim);
  if (out_index) *out_index = (int)sim->tracers.size() - 1;
  return LBM_OK;
}

int lbm_set_tracer_storage(lbm_sim* sim, int storage) {
  if (int rc = activate(sim)) return rc;
  if (!sim->tracers.empty())
    return fail(LBM_ERR_STATE, "the tracer storage is chosen before the first tracer is added");
  if (storage == LBM_STORAGE_F32 && sim->storage != LBM_STORAGE_F64) {
    sim->tracer_storage = -1;
    drop_graph(sim);
    return LBM_OK;
  }
  if ((storage == LBM_STORAGE_F16 || storage == LBM_STORAGE_BF16) && storage == sim->storage) {
    sim->tracer_storage = storage;
    drop_graph(sim);
    return LBM_OK;
  }
  return fail(LBM_ERR_UNSUPPORTED,
              "tracer populations are stored as float, or in the fluid's own 16-bit kind");
}

int lbm_set_gravity(lbm_sim* sim, const float* g) {
  if (int rc = activate(sim)) return rc;
  if (g == nullptr) return fail(LBM_ERR_ARGUMENT, "null gravity");
  sim->has_gravity = true;
  drop_graph(sim);
  for (int k = 0; k < sim->dim; ++k) sim->gravity[k] = g[k];
  return LBM_OK;
}

int lbm_add_coupling(lbm_sim* sim, int tracer, float alpha, float c0, const float* g) {
  if (int rc = activate(sim)) return rc;
  if (int rc = check_tracer(sim, tracer)) return rc;
  if (g == nullptr) return fail(LBM_ERR_ARGUMENT, "null gravity");
  lbm_sim::Coupling c;
  c.tracer = tracer;
  c.alpha = alpha;
  c.c0 = c0;
  for (int k = 0; k < sim->dim; ++k) c.g[k] = g[k];
  sim->couplings.push_back(c);
  drop_graph(sim);
  return LBM_OK;
}

int lbm_upload_flags(lbm_sim* sim, const int32_t* flags) {
  if (int rc = activate(sim)) return rc;
  if (flags == nullptr) return fail(LBM_ERR_ARGUMENT, "null flags");
  // Only bits 0-3 are read by the kernels (WALL, FIXED_FLUID_*, FIXED_SCALAR_VALUE): the int32
  // array goes over as it is (one DMA from the caller's buffer) and is narrowed on the device.
  int32_t* tmp = nullptr;
  LBM_CUDA(cudaMallocAsync((void**)&tmp, (size_t)sim->n * sizeof(int32_t), sim->stream));
  LBM_CUDA(cudaMemcpyAsync(tmp, flags, (size_t)sim->n * sizeof(int32_t), cudaMemcpyHostToDevice,
                           sim->stream));
  LBM_CUDA(lbm::flags_to_u8(tmp, static_cast<uint8_t*>(sim->flags), sim->n, sim->stream));
  LBM_CUDA(cudaFreeAsync(tmp, sim->stream));
  LBM_CUDA(cudaStreamSynchronize(sim->stream));
  return LBM_OK;
}

int lbm_upload_fluid(lbm_sim* sim, const float* rho, const float* vel) {
  if (int rc = activate(sim)) return rc;
  if (rho) {
    if (int rc = upload_reals(sim, sim->rho, rho, sim->n)) return rc;
  }
  if (vel) {
    if (int rc = upload_reals(sim, sim->vel, vel, sim->n * sim->dim)) return rc;
  }
  LBM_CUDA(cudaStreamSynchronize(sim->stream));
  return LBM_OK;
}

int lbm_upload_tracer(lbm_sim* sim, int tracer, const float* val) {
  if (int rc = activate(sim)) return rc;
  if (int rc = check_tracer(sim, tracer)) return rc;
  if (int rc = upload_reals(sim, sim->tracers[tracer].val, val, sim->n)) return rc;
  LBM_CUDA(cudaStreamSynchronize(sim->stream));
  return LBM_OK;
}

int lbm_equilibrate(lbm_sim* sim) {
  if (int rc = activate(sim)) return rc;
  cudaError_t e = lbm::equilibrate(*sim);
  if (e == cudaErrorNotSupported) return fail(LBM_ERR_UNSUPPORTED, "no equilibrium for this set");
  if (e != cudaSuccess) return cuda_fail(e, "equilibrate");
  return LBM_OK;
}

int lbm_equilibrate_tracer(lbm_sim* sim, int tracer) {
  if (int rc = activate(sim)) return rc;
  if (int rc = check_tracer(sim, tracer)) return rc;
  cudaError_t e = lbm::equilibrate_tracer(*sim, tracer);
  if (e == cudaErrorNotSupported) return fail(LBM_ERR_UNSUPPORTED, "no equilibrium for this set");
  if (e != cudaSuccess) return cuda_fail(e, "equilibrate_tracer");
  return LBM_OK;
}

static int transfer_populations(lbm_sim* sim, int tracer, float* host, bool to_device) {
  if (int rc = activate(sim)) return rc;
  if (tracer >= 0) {
    if (int rc = check_tracer(sim, tracer)) return rc;
  }
  const int q = tracer < 0 ? sim->q : sim->tracers[tracer].q;
  const size_t bytes = (size_t)sim->n * q * sizeof(float);
  float* tmp = nullptr;
  LBM_CUDA(cudaMallocAsync((void**)&tmp, bytes, sim->stream));
  cudaError_t e;
  if (to_device) {
    e = cudaMemcpyAsync(tmp, host, bytes, cudaMemcpyHostToDevice, sim->stream);
    if (e == cudaSuccess) e = lbm::populations_from_aos(*sim, tracer, tmp);
  } else {
    e = lbm::populations_to_aos(*sim, tracer, tmp);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, tmp, bytes, cudaMemcpyDeviceToHost, sim->stream);
  }
  cudaFreeAsync(tmp, sim->stream);
  if (e == cudaErrorNotSupported) return fail(LBM_ERR_UNSUPPORTED, "no layout for this set");
  if (e != cudaSuccess) return cuda_fail(e, "populations transfer");
  LBM_CUDA(cudaStreamSynchronize(sim->stream));
  return LBM_OK;
}

int lbm_upload_f(lbm_sim* sim, const float* f) {
  return transfer_populations(sim, -1, const_cast<float*>(f), true);
}
int lbm_download_f(lbm_sim* sim, float* f) { return transfer_populations(sim, -1, f, false); }
int lbm_upload_g(lbm_sim* sim, int tracer, const float* g) {
  return transfer_populations(sim, tracer < 0 ? -2 : tracer, const_cast<float*>(g), true);
}
int lbm_download_g(lbm_sim* sim, int tracer, float* g) {
  return transfer_populations(sim, tracer < 0 ? -2 : tracer, g, false);
}

int lbm_iterate(lbm_sim* sim, int64_t iters) {
  if (int rc = activate(sim)) return rc;
  if (iters < 0 || iters % 2 != 0) return fail(LBM_ERR_ARGUMENT, "iters must be even");
  if (iters == 0) return LBM_OK;  // no kernel is looked up when no step runs
  if (!fluid_kernel(sim->dim, sim->q))
    return fail(LBM_ERR_UNSUPPORTED, "Kernel not found: D" + std::to_string(sim->dim) + "Q" +
                                         std::to_string(sim->q) + " NavierStokes");
  for (const lbm_sim::Tracer& t : sim->tracers)
    if (!tracer_kernel(sim->dim, t.q, t.collision))
      return fail(LBM_ERR_UNSUPPORTED, "Kernel not found: D" + std::to_string(sim->dim) + "Q" +
                                           std::to_string(t.q) + " AdvectionDiffusion");
  int64_t left = iters / 2;  // step pairs
  // The pairs before the last one (which writes the moments) go out as replays of captured
  // graphs of kMinGraphPairs..kGraphPairs pairs while that many are left; the rest are launched
  // directly, and so is the first pair after creation or a change of state (outside any capture,
  // so each kernel's one-time set-up has run). Not while the caller is capturing the simulation's
  // stream into a graph of its own.
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  const bool outer = cudaStreamIsCapturing(sim->stream, &cs) == cudaSuccess &&
                     cs != cudaStreamCaptureStatusNone;
  if (!outer && !sim->graph_failed && left >= kMinGraphPairs + 2) {
    if (!sim->graph_warm) {
      if (cudaError_t e = launch_pair(sim, false)) return step_launch_fail(e);
      --left;
      sim->graph_warm = true;
    }
    while (left - 1 >= kMinGraphPairs) {
      const int64_t pairs = left - 1 < kGraphPairs ? left - 1 : kGraphPairs;
      const lbm_sim::StepGraph* g = step_graph(sim, pairs);
      if (g == nullptr) {  // launched one at a time from now on, until the state changes
        cudaGetLastError();
        sim->graph_failed = true;
        break;
      }
      LBM_CUDA(cudaGraphLaunch(g->exec, sim->stream));
      sim->launches[0] += g->launches[0];
      sim->launches[1] += g->launches[1];
      left -= pairs;
    }
  }
  for (; left > 0; --left)
    if (cudaError_t e = launch_pair(sim, left == 1)) return step_launch_fail(e);
  return LBM_OK;
}

int lbm_download_fluid(lbm_sim* sim, float* rho, float* vel) {
  if (int rc = activate(sim)) return rc;
  if (rho) {
    if (int rc = download_reals(sim, rho, sim->rho, sim->n)) return rc;
  }
  if (vel) {
    if (int rc = download_reals(sim, vel, sim->vel, sim->n * sim->dim)) return rc;
  }
  LBM_CUDA(cudaStreamSynchronize(sim->stream));
  return check_status(sim);
}

int lbm_download_tracer(lbm_sim* sim, int tracer, float* val) {
  if (int rc = activate(sim)) return rc;
  if (int rc = check_tracer(sim, tracer)) return rc;
  if (int rc = download_reals(sim, val, sim->tracers[tracer].val, sim->n)) return rc;
  LBM_CUDA(cudaStreamSynchronize(sim->stream));
  return LBM_OK;
}

int lbm_download_fluid_f64(lbm_sim* sim, double* rho, double* vel) {
  if (int rc = activate(sim)) return rc;
  if (sim->storage != LBM_STORAGE_F64)
    return fail(LBM_ERR_STATE, "lbm_download_fluid_f64 needs LBM_STORAGE_F64");
  if (rho)
    LBM_CUDA(cudaMemcpyAsync(rho, sim->rho, sim->n * sizeof(double), cudaMemcpyDeviceToHost,
                             sim->stream));
  if (vel)
    LBM_CUDA(cudaMemcpyAsync(vel, sim->vel, sim->n * sim->dim * sizeof(double),
                             cudaMemcpyDeviceToHost, sim->stream));
  LBM_CUDA(cudaStreamSynchronize(sim->stream));
  return LBM_OK;
}

int lbm_conservation(lbm_sim* sim, double* out, int len) {
  if (int rc = activate(sim)) return rc;
  const int need = 1 + sim->dim + (int)sim->tracers.size();
  if (out == nullptr || len < need)
    return fail(LBM_ERR_ARGUMENT, "output needs 1 + dim + ntracers doubles");
  LBM_CUDA(cudaMemsetAsync(sim->sums, 0, need * sizeof(double), sim->stream));
  cudaError_t e = lbm::conservation_sums(*sim, sim->sums);
  if (e == cudaErrorNotSupported) return fail(LBM_ERR_UNSUPPORTED, "no sums for this set");
  if (e != cudaSuccess) return cuda_fail(e, "conservation sums");
  LBM_CUDA(cudaMemcpyAsync(out, sim->sums, need * sizeof(double), cudaMemcpyDeviceToHost,
                           sim->stream));
  LBM_CUDA(cudaStreamSynchronize(sim->stream));
  return LBM_OK;
}

int lbm_nonfinite(lbm_sim* sim, int* out) {
  if (int rc = activate(sim)) return rc;
  int word = 0;
  LBM_CUDA(cudaMemcpyAsync(&word, sim->status, sizeof(int), cudaMemcpyDeviceToHost, sim->stream));
  LBM_CUDA(cudaMemsetAsync(sim->status, 0, sizeof(int), sim->stream));
  LBM_CUDA(cudaStreamSynchronize(sim->stream));
  if (out) *out = word & 1;
  return LBM_OK;
}

int lbm_set_kernel_path(lbm_sim* sim, int path) {
  if (int rc = activate(sim)) return rc;
  if (path < LBM_PATH_AUTO || path > LBM_PATH_STAGED)
    return fail(LBM_ERR_ARGUMENT, "unknown kernel path");
  if (sim->kernel_path != path) drop_graph(sim);
  sim->kernel_path = path;
  return LBM_OK;
}

int lbm_set_spin_limit(lbm_sim* sim, int64_t polls) {
  if (int rc = activate(sim)) return rc;
  if (sim->spin_limit != (polls < 0 ? -1 : polls)) drop_graph(sim);
  sim->spin_limit = polls < 0 ? -1 : polls;
  return LBM_OK;
}

int lbm_launch_counts(lbm_sim* sim, int64_t* direct, int64_t* staged) {
  if (int rc = activate(sim)) return rc;
  if (direct) *direct = sim->launches[0];
  if (staged) *staged = sim->launches[1];
  return LBM_OK;
}

int lbm_set_omega_field(lbm_sim* sim, const float* field) {
  if (int rc = activate(sim)) return rc;
  if (field != nullptr && sim->storage == LBM_STORAGE_F64)
    return fail(LBM_ERR_UNSUPPORTED, "per-cell relaxation needs a float storage kind");
  if (sim->omega_field != field) drop_graph(sim);
  sim->omega_field = field;
  return LBM_OK;
}

int lbm_fluid_device(lbm_sim* sim, void** rho, void** vel) {
  if (int rc = activate(sim)) return rc;
  if (rho) *rho = sim->rho;
  if (vel) *vel = sim->vel;
  return LBM_OK;
}

int lbm_synchronize(lbm_sim* sim) {
  if (int rc = activate(sim)) return rc;
  LBM_CUDA(cudaStreamSynchronize(sim->stream));
  return check_status(sim);
}

int lbm_stream(lbm_sim* sim, void** stream) {
  if (int rc = activate(sim)) return rc;
  if (stream) *stream = (void*)sim->stream;
  return LBM_OK;
}

void* lbm_host_alloc(size_t bytes) {
  void* p = nullptr;
  if (cudaMallocHost(&p, bytes ? bytes : 1) != cudaSuccess) {
    g_error = "cudaMallocHost failed";
    return nullptr;
  }
  return p;
}

void lbm_host_free(void* ptr) {
  if (ptr) cudaFreeHost(ptr);
}

}  // extern "C"
