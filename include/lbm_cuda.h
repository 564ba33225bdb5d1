/*
 * lbm_cuda.h -- C ABI of the CUDA (sm_100a) lattice-Boltzmann backend.
 *
 * This is the device layer that replaces the OpenCL backend of djbarker/boltzmann
 * (src/opencl.rs, plus the enqueue calls of src/simulation.rs and src/fields.rs). A host layer
 * (the Python extension boltzmann_b200.boltzmann here; pyo3 bindings wherever Rust is available)
 * owns the host arrays, keeps the reference's semantics (upload at the first iterate call,
 * read-back after every call) and calls these functions.
 *
 * Conventions
 *   - Every function returns LBM_OK (0) or an lbm_status; lbm_last_error() then describes the
 *     failure (thread-local). No C++ exception crosses this boundary.
 *   - Host arrays use the reference's host layouts (row-major, x slowest):
 *       flags int32 [N], rho float [N], vel float [N, dim], tracer val float [N],
 *       populations float [N, q] (checkpoint layout, src/fields.rs:71-75),
 *     where N = counts[0] * ... * counts[dim-1].
 *   - All device work of one simulation runs on its own CUDA stream; functions that return
 *     host data synchronise that stream first.
 *   - The device layout is internal: populations structure-of-arrays, optionally stored as
 *     16-bit offsets from the lattice weights (LBM_STORAGE_F16 / _BF16).
 */
#ifndef LBM_CUDA_H
#define LBM_CUDA_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define LBM_API __attribute__((visibility("default")))
#else
#define LBM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct lbm_sim lbm_sim;

enum lbm_status {
  LBM_OK = 0,
  LBM_ERR_ARGUMENT = 1,    /* bad argument (odd iters, unknown model, wrong index, ...) */
  LBM_ERR_UNSUPPORTED = 2, /* no kernel for this combination ("Kernel not found") */
  LBM_ERR_CUDA = 3,        /* a CUDA runtime call failed */
  LBM_ERR_STATE = 4        /* call not valid in the current state */
};

enum lbm_collision { LBM_BGK = 0, LBM_TRT = 1 };

enum lbm_storage {
  LBM_STORAGE_F32 = 0,  /* float populations (the reference's precision) */
  LBM_STORAGE_F16 = 1,  /* half offsets f_i - w_i, collision in float */
  LBM_STORAGE_BF16 = 2, /* bfloat16 offsets f_i - w_i, collision in float */
  LBM_STORAGE_F64 = 3   /* double populations and arithmetic (the FP64 comparison run) */
};

enum lbm_kernel_path {
  LBM_PATH_AUTO = 0,   /* staged for large domains whose rows split into 256-cell tiles */
  LBM_PATH_DIRECT = 1, /* one cell per thread, loads straight into registers */
  LBM_PATH_STAGED = 2  /* TMA bulk copies into a shared-memory ring (rows of 256k cells only) */
};

/* Thread-local description of the last failure. */
LBM_API const char* lbm_last_error(void);

/* ABI version of this header (bumped on any signature change). */
LBM_API int lbm_abi_version(void);

/* Creates a simulation on the current CUDA device: flags = 0, rho = 1, vel = 0, populations 0.
 * Replaces OpenCLCtx::new + Simulation::new + Fluid::new
 * (src/opencl.rs:102-171, src/simulation.rs:179-192, src/fields.rs:68-82).
 * dim in {1,2,3}; q must name a velocity set of src/velocities.rs:55-64 (else
 * LBM_ERR_ARGUMENT, "Unknown model"); a set without an update kernel is accepted here and
 * rejected by lbm_iterate, as in the reference. */
LBM_API int lbm_create(int dim, const int64_t* counts, int q, int collision, float omega_pos,
               float omega_neg, int storage, lbm_sim** out);

/* Releases all device memory of the simulation. */
LBM_API int lbm_destroy(lbm_sim* sim);

/* "<device name> GPU", the analogue of Simulation.device_info (src/lib.rs:205-215). */
LBM_API int lbm_device_info(lbm_sim* sim, char* buf, int len);

/* Device bytes held by populations, rho, vel and tracers (src/lib.rs:228-236 counts host
 * mirrors of the same arrays). */
LBM_API int lbm_device_bytes(lbm_sim* sim, int64_t* out);

/* Adds an advection-diffusion tracer (g = 0, val = 0) and returns its index.
 * Replaces Scalar::new + Simulation::add_tracer (src/fields.rs:152-163,
 * src/simulation.rs:221-229). collision LBM_BGK (omega_pos) or LBM_TRT (omega_pos, omega_neg):
 * the reference registers BGK tracer kernels only (src/opencl.rs:123-129); TRT follows the
 * D2Q5 / D3Q7 kernels its generator writes (python/boltzmann/kernel_gen.py:250-462). */
LBM_API int lbm_add_tracer(lbm_sim* sim, int q, int collision, float omega_pos, float omega_neg,
                   int* out_index);

/* Storage of the tracers' populations, chosen before the first tracer is added: LBM_STORAGE_F32
 * (the default; double for an LBM_STORAGE_F64 simulation) or the fluid's own 16-bit kind
 * (LBM_STORAGE_F16 / _BF16 for a simulation created with it), which halves the tracer's bytes per
 * cell update; 16-bit tracer populations hold the values themselves (not offsets) and take one
 * tracer per simulation (LBM_ERR_UNSUPPORTED otherwise). The tracer values (val) stay float. No
 * reference counterpart (the reference stores float). */
LBM_API int lbm_set_tracer_storage(lbm_sim* sim, int storage);

/* Constant body force, dim floats (src/simulation.rs:194-196). */
LBM_API int lbm_set_gravity(lbm_sim* sim, const float* g);

/* Boussinesq coupling acc = g * alpha * (C - c0) to tracer `tracer`, dim floats of g
 * (src/simulation.rs:201-216). With several couplings the last one added sets the
 * acceleration, and any coupling overrides the constant body force, as in
 * src/simulation.rs:326-373. */
LBM_API int lbm_add_coupling(lbm_sim* sim, int tracer, float alpha, float c0, const float* g);

/* Host -> device copies of the macroscopic fields (Data::enqueue_write, src/opencl.rs:253-265,
 * as called by Simulation::finalize, src/simulation.rs:254-275). */
LBM_API int lbm_upload_flags(lbm_sim* sim, const int32_t* flags);
LBM_API int lbm_upload_fluid(lbm_sim* sim, const float* rho, const float* vel);
LBM_API int lbm_upload_tracer(lbm_sim* sim, int tracer, const float* val);

/* f = feq(rho, vel) and every tracer's g = feq(val, vel) on the device, bit-identical in FP32 to
 * Fluid::equilibrate / Scalar::equilibrate (src/fields.rs:106-114, 185-193,
 * src/velocities.rs:43-52). */
LBM_API int lbm_equilibrate(lbm_sim* sim);

/* Same for one tracer only, against the fluid velocity currently on the device. Used for a
 * tracer added after the first iterate call, whose device buffers the reference leaves
 * unwritten (src/simulation.rs:221-229 allocates, only finalize() at iteration 0 uploads). */
LBM_API int lbm_equilibrate_tracer(lbm_sim* sim, int tracer);

/* Populations in the checkpoint layout float [N, q] (src/simulation.rs:448-479). */
LBM_API int lbm_upload_f(lbm_sim* sim, const float* f);
LBM_API int lbm_download_f(lbm_sim* sim, float* f);
LBM_API int lbm_upload_g(lbm_sim* sim, int tracer, const float* g);
LBM_API int lbm_download_g(lbm_sim* sim, int tracer, float* g);

/* Advances `iters` AA steps (the per-step loop of Simulation::iterate,
 * src/simulation.rs:288-433). iters must be even (src/simulation.rs:279-281). Asynchronous:
 * returns once the steps are enqueued on the simulation's stream. The step pairs before the
 * last go out as replays of CUDA graphs of 8 to 16 pairs while that many are left, each graph
 * captured once per simulation state; the rest, and the first pair after creation or after a
 * setter changed the state, are launched directly, as is every step of a call made while the
 * caller captures the simulation's stream. */
LBM_API int lbm_iterate(lbm_sim* sim, int64_t iters);

/* Device -> host copies after an iterate call (Fluid/Scalar::read_to_host,
 * src/fields.rs:97-104, 177-183). Synchronous. */
LBM_API int lbm_download_fluid(lbm_sim* sim, float* rho, float* vel);
LBM_API int lbm_download_tracer(lbm_sim* sim, int tracer, float* val);

/* Same for an LBM_STORAGE_F64 simulation, in double. */
LBM_API int lbm_download_fluid_f64(lbm_sim* sim, double* rho, double* vel);

/* FP64 sums over every population slot: out[0] = sum f, out[1..dim] = sum c_i f_i, then one
 * sum of g per tracer. No reference counterpart (conservation diagnostics). Synchronous. */
LBM_API int lbm_conservation(lbm_sim* sim, double* out, int len);

/* Sets *out to 1 when a non-finite density or velocity was produced by a step that ended an
 * iterate call since the last query, else 0; clears the flag. The device-side analogue of run_sim's NaN check
 * (python/boltzmann/simulation.py:241-242). Synchronous. */
LBM_API int lbm_nonfinite(lbm_sim* sim, int* out);

/* Chooses the AA kernel variant (enum lbm_kernel_path). A tuning and testing knob: results are
 * identical up to floating-point rounding order; LBM_PATH_STAGED falls back to the direct kernel
 * where the row length is not a multiple of 256 or more than one tracer is fused. No reference
 * counterpart. */
LBM_API int lbm_set_kernel_path(lbm_sim* sim, int path);

/* Polls that each pipeline wait of the TMA-staged kernel makes before it gives up (the copies of
 * a stage, or its release by the consumer warps); polls < 0 restores the default (2^22). A kernel
 * that gives up sets bit 1 of the status word, still waits (with the default bound) for the
 * copies it issued, and returns; the next synchronising call (lbm_download_fluid,
 * lbm_synchronize) then fails with LBM_ERR_CUDA, once, and the populations are not valid until
 * they are uploaded again. 0 makes every pipeline wait give up at once: a way to exercise that
 * path. No reference counterpart. */
LBM_API int lbm_set_spin_limit(lbm_sim* sim, int64_t polls);

/* AA step launches since lbm_create, per kernel variant: the direct kernel (aa_step_kernel) and
 * the TMA-staged one (aa_tma_kernel). Host-side counters, no synchronisation. No reference
 * counterpart (instrumentation: which kernel a workload actually ran). */
LBM_API int lbm_launch_counts(lbm_sim* sim, int64_t* direct, int64_t* staged);

/* Per-cell relaxation rate: `field` is a device array of N floats (omega+ of every cell) that
 * the caller owns and keeps alive, written on the simulation's stream (a learned closure's output);
 * NULL returns to the uniform rate. Fixed cells still relax with 1; the force shift keeps the
 * uniform rate. Float storage kinds only. No reference counterpart. */
LBM_API int lbm_set_omega_field(lbm_sim* sim, const float* field);

/* Device pointers of rho [N] and vel [N, dim] (valid until lbm_destroy; written on the step that
 * ends each lbm_iterate call), for device-side consumers on the simulation's stream. */
LBM_API int lbm_fluid_device(lbm_sim* sim, void** rho, void** vel);

/* Blocks until all work of the simulation is done. */
LBM_API int lbm_synchronize(lbm_sim* sim);

/* The simulation's cudaStream_t, for callers that time or order work around it. */
LBM_API int lbm_stream(lbm_sim* sim, void** stream);

/* The FP64 sums of lbm_conservation (sum f, then sum c_i f per axis) for a population array the
 * caller owns, allocating no device memory: for callers that cannot allocate -- solvers embedded
 * in another framework's memory arena or under an allocator that forbids extra cudaMalloc calls.
 * No counterpart in the reference.
 *   f      device pointer, layout [q][n] in the storage encoding of `storage` (the 16-bit kinds
 *          hold f_i - w_i);
 *   out    device pointer to 1 + dim doubles, all written;
 *   stream cudaStream_t to run on (NULL: the default stream). Asynchronous.
 * Scratch is a fixed 64 KiB per device inside this library, held until the process exits, so n is
 * limited to 134,217,728 cells (LBM_ERR_ARGUMENT beyond). The first call on a device looks up that
 * scratch's address; make it before any stream capture. After the device's context is created
 * again (cudaDeviceReset) the next call looks the address up again, so make that call outside
 * stream capture too. All calls share the scratch: calls that may overlap on the GPU (unordered
 * streams) race. */
LBM_API int lbm_population_sums_noalloc(int dim, int q, int storage, const void* f, int64_t n,
                                        double* out, void* stream);

/* ---- Batched ensembles of independent 2D D2Q9 domains (no reference counterpart: the reference
 * runs one domain per Simulation). All domains advance together, one launch per step. ---- */
typedef struct lbm_ensemble lbm_ensemble;

enum lbm_ensemble_mode {
  LBM_ENSEMBLE_PERSISTENT = 0, /* one persistent launch per step over the tile table */
  LBM_ENSEMBLE_GRAPH = 1,      /* the same launches replayed from a captured CUDA graph */
  LBM_ENSEMBLE_PER_DOMAIN = 2  /* one launch per domain per step (the unbatched baseline) */
};

/* counts: [ndomains][2] (nx, ny of each domain, the reference's 2D counts); omega_pos/omega_neg:
 * per-domain BGK rate (or TRT rates; omega_neg may be NULL for BGK). Host arrays of an ensemble
 * are the per-domain arrays concatenated in domain order (flags int32, rho, vel [.., 2]).
 * Populations f32, f16 or bf16 (offsets). Each domain is periodic in itself. */
LBM_API int lbm_ensemble_create(int ndomains, const int64_t* counts, int collision,
                                const float* omega_pos, const float* omega_neg, int storage,
                                lbm_ensemble** out);
LBM_API int lbm_ensemble_destroy(lbm_ensemble* ens);
LBM_API int lbm_ensemble_cells(lbm_ensemble* ens, int64_t* total);
/* Launch shape of the persistent kernel. tile_cells 0 selects the row-staged kernel (the default
 * when every domain row has at most 512 cells; LBM_ERR_UNSUPPORTED otherwise): one domain row
 * per work item, loaded by TMA bulk copies into a shared-memory ring. A multiple of 32 in
 * [32, 512] selects the tile kernel with that many cells per tile (two per thread), loads straight
 * into registers. blocks_per_sm: CTAs per SM of the persistent grid (0 = as many as fit).
 * Chosen by the autotuner (boltzmann_b200.autotune); every shape gives the same bits. */
LBM_API int lbm_ensemble_set_shape(lbm_ensemble* ens, int tile_cells, int blocks_per_sm);
LBM_API int lbm_ensemble_upload(lbm_ensemble* ens, const int32_t* flags, const float* rho,
                                const float* vel);
LBM_API int lbm_ensemble_equilibrate(lbm_ensemble* ens);
/* iters even; mode: enum lbm_ensemble_mode. Asynchronous on the ensemble's stream. */
LBM_API int lbm_ensemble_iterate(lbm_ensemble* ens, int64_t iters, int mode);
LBM_API int lbm_ensemble_download(lbm_ensemble* ens, float* rho, float* vel);
LBM_API int lbm_ensemble_upload_f(lbm_ensemble* ens, const float* f);
LBM_API int lbm_ensemble_download_f(lbm_ensemble* ens, float* f);
LBM_API int lbm_ensemble_stream(lbm_ensemble* ens, void** stream);
LBM_API int lbm_ensemble_synchronize(lbm_ensemble* ens);

/* Page-locked host memory for host arrays (fast transfers); NULL on failure. */
LBM_API void* lbm_host_alloc(size_t bytes);
LBM_API void lbm_host_free(void* ptr);

#ifdef __cplusplus
}
#endif

#endif /* LBM_CUDA_H */
