// Internal state behind the lbm_sim handle of include/lbm_cuda.h.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

struct lbm_sim {
  struct Tracer {
    int q = 0;
    int collision = 0;
    float omega = 0;      // omega (BGK) or omega+ (TRT)
    float omega_neg = 0;  // omega- (TRT)
    void* g = nullptr;    // [q][N], float (double for F64 storage)
    void* val = nullptr;  // [N]
  };
  struct Coupling {
    int tracer = 0;
    float alpha = 0, c0 = 0;
    float g[3] = {0, 0, 0};
  };

  int dim = 0, q = 0, collision = 0, storage = 0;
  // Storage kind of the tracers' populations: -1 for the fluid's compute type (float, double
  // for FP64 runs), or the fluid's 16-bit kind (lbm_set_tracer_storage).
  int tracer_storage = -1;
  int64_t counts[3] = {1, 1, 1};
  int64_t n = 0;  // cell count
  float om_pos = 0, om_neg = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  int kernel_path = 0;  // LBM_PATH_AUTO / _DIRECT / _STAGED
  int64_t spin_limit = -1;  // polls of the staged kernel's pipeline waits; < 0: the default
  // AA step launches since creation, per kernel variant: [0] direct, [1] TMA-staged.
  mutable int64_t launches[2] = {0, 0};
  // Step pairs captured as CUDA graphs and replayed by lbm_iterate, one per pair count (at most
  // four), dropped whenever a setter changes what a step launches; `warm` once a pair has run
  // outside any capture in the current state (each kernel's one-time launch set-up done).
  struct StepGraph {
    int64_t pairs;
    cudaGraphExec_t exec;
    int64_t launches[2];  // what one replay adds to `launches`
  };
  std::vector<StepGraph> graphs;
  bool graph_warm = false, graph_failed = false;
  const float* omega_field = nullptr;  // caller-owned per-cell om_pos, or null

  void* f = nullptr;    // [q][N] populations in the storage type
  void* rho = nullptr;  // [N], float (double for F64)
  void* vel = nullptr;  // [N][dim]
  uint8_t* flags = nullptr;
  int* status = nullptr;      // device word: bit 0 = non-finite density seen
  double* sums = nullptr;     // device scratch of the conservation reduction
  int sums_len = 0;

  std::vector<Tracer> tracers;
  bool has_gravity = false;
  float gravity[3] = {0, 0, 0};
  std::vector<Coupling> couplings;

  size_t real_bytes() const { return storage == 3 ? 8 : 4; }
  // Storage kind and element bytes of tracer populations.
  int tracer_kind() const { return tracer_storage >= 0 ? tracer_storage : (storage == 3 ? 3 : 0); }
  size_t tracer_pop_bytes() const { return tracer_kind() == 3 ? 8 : (tracer_kind() == 0 ? 4 : 2); }
};

namespace lbm {

// Sets the thread-local message returned by lbm_last_error().
void set_last_error(const std::string& msg);

// Bytes of one stored population for a storage kind.
inline size_t pop_bytes(int storage) { return storage == 3 ? 8 : (storage == 0 ? 4 : 2); }

// Enqueues one AA step of the whole simulation (fluid, tracers, sources) on sim.stream.
cudaError_t launch_step_d2q9(const lbm_sim& sim, bool even, bool write_moments);
cudaError_t launch_step_d3q27(const lbm_sim& sim, bool even, bool write_moments);

// Field kernels (fields.cu), all on sim.stream.
cudaError_t equilibrate(const lbm_sim& sim);
cudaError_t equilibrate_tracer(const lbm_sim& sim, int tracer);
cudaError_t populations_from_aos(const lbm_sim& sim, int tracer, const float* d_aos);
cudaError_t populations_to_aos(const lbm_sim& sim, int tracer, float* d_aos);
cudaError_t narrow_to_float(const double* src, float* dst, int64_t count, cudaStream_t s);
cudaError_t widen_to_double(const float* src, double* dst, int64_t count, cudaStream_t s);
cudaError_t flags_to_u8(const int32_t* src, uint8_t* dst, int64_t count, cudaStream_t s);
cudaError_t fill_value(void* dst, int64_t count, double value, bool is_double, cudaStream_t s);
cudaError_t conservation_sums(const lbm_sim& sim, double* d_out);

}  // namespace lbm
