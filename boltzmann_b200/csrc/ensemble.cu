// Batched ensembles: many independent 2D D2Q9 domains of uneven sizes (parameter sweeps)
// advanced together.
//
// All domains' cells are concatenated into one structure-of-arrays population array
// (domain d owns cells [base_d, base_d + nx_d * ny_d), each domain in the reference's row-major
// order), with one flags/rho/vel array, so one kernel launch advances every domain by one AA step.
// A host-built tile table splits every domain row into segments of `tile` cells; a persistent
// grid (a fixed number of CTAs per SM) walks the table, two cells of a tile per thread (tile / 2
// threads a CTA), with the domain's sizes and relaxation rates read from a domain table. Each
// domain is periodic in itself (its own rows wrap), exactly as a separate simulation of that size
// would be, and the cell update is the same device function the single-domain kernels use.
//
// Modes of lbm_ensemble_iterate:
//   persistent        one launch per step;
//   persistent+graph  the same launches captured once into a CUDA graph of `chunk` step pairs and
//                     replayed (no per-launch host overhead);
//   per-domain        one launch per domain per step: the baseline the batched launch replaces.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/lbm_cuda.h"
#include "aa_step.cuh"
#include "sim.h"

namespace {

struct DomainDesc {
  long long base;   // first cell
  int nx, ny;       // the reference's counts: rows x, cells per row y
  float om_pos, om_neg;
};

struct TileDesc {
  int domain;
  int x;       // row of the domain
  int z0;      // first cell of the row in this tile
  int len;     // cells in this tile
};

struct EnsembleArgs {
  const DomainDesc* domains;
  const TileDesc* tiles;
  long long ntiles;
};

template <bool TRT, int K, bool EVEN>
__global__ void __launch_bounds__(512)
    ensemble_step_kernel(const __grid_constant__ lbm::StepArgs<typename lbm::Pop<K>::real> a,
                         const EnsembleArgs e) {
  using namespace lbm;
  using P = Pop<K>;
  using Real = typename P::real;
  using T = typename P::type;
  // Two cells a thread (t and t + half of the tile): both cells' loads are issued before either
  // update, twice the loads in flight a thread.
  for (long long t = blockIdx.x; t < e.ntiles; t += gridDim.x) {
    const TileDesc tile = e.tiles[t];
    const int half = (tile.len + 1) / 2;
    if ((int)threadIdx.x >= half) continue;
    const DomainDesc dom = e.domains[tile.domain];
    const int x = tile.x;
    const bool hasB = (int)threadIdx.x + half < tile.len;
    CellPos c[2];
    const unsigned base = (unsigned)dom.base, ny = (unsigned)dom.ny;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int z = tile.z0 + threadIdx.x + k * half;
      c[k].ox[0] = c[k].ox[1] = c[k].ox[2] = base;
      c[k].oy[1] = (unsigned)x * ny;
      c[k].oz[1] = (unsigned)z;
      c[k].cell = base + c[k].oy[1] + c[k].oz[1];
      if (EVEN) {
        c[k].oy[0] = (unsigned)(x == 0 ? dom.nx - 1 : x - 1) * ny;
        c[k].oy[2] = (unsigned)(x == dom.nx - 1 ? 0 : x + 1) * ny;
        c[k].oz[0] = (unsigned)(z == 0 ? dom.ny - 1 : z - 1);
        c[k].oz[2] = (unsigned)(z == dom.ny - 1 ? 0 : z + 1);
      }
    }
    const int flagA = a.flags[c[0].cell];
    const int flagB = hasB ? a.flags[c[1].cell] : 1;  // a missing cell acts as a wall
    Real fa[D2Q9::Q], fb[D2Q9::Q];
    aa_load<D2Q9, P, EVEN, lbm::dev_in<K>()>(static_cast<const T*>(a.f), a.n, c[0], fa);
    if (hasB) aa_load<D2Q9, P, EVEN, lbm::dev_in<K>()>(static_cast<const T*>(a.f), a.n, c[1], fb);
    Real g[1];
    update_cell<D2Q9, TRT, K, EVEN, 0>(a, c[0], flagA, fa, g, Real(0), (Real)dom.om_pos,
                                       (Real)dom.om_neg);
    if (hasB)
      update_cell<D2Q9, TRT, K, EVEN, 0>(a, c[1], flagB, fb, g, Real(0), (Real)dom.om_pos,
                                         (Real)dom.om_neg);
  }
}

}  // namespace

struct lbm_ensemble {
  int ndomains = 0, collision = 0, storage = 0;
  std::vector<DomainDesc> domains;
  long long n = 0;                 // total cells
  int tile = 256;                  // cells per tile (tile / 2 threads)
  int blocks_per_sm = 0;           // 0: occupancy limit
  int device = 0;
  cudaStream_t stream = nullptr;
  lbm_sim shell;                   // describes the concatenated arrays for the field kernels
  DomainDesc* d_domains = nullptr;
  TileDesc* d_tiles = nullptr;
  long long ntiles = 0;
  int tiles_for = 0;               // tile width the table was built for
  // Captured graph of `graph_pairs` step pairs in persistent mode.
  cudaGraphExec_t graph = nullptr;
  int graph_pairs = 0, graph_tile = 0, graph_blocks = 0;
};

namespace {

int efail(int code, const std::string& msg) {
  lbm::set_last_error(msg);
  return code;
}

int ecuda(cudaError_t e, const char* where) {
  return efail(LBM_ERR_CUDA, std::string("CUDA error in ") + where + ": " + cudaGetErrorName(e) +
                                 " (" + cudaGetErrorString(e) + ")");
}

#define ENS_CUDA(call)                                  \
  do {                                                  \
    cudaError_t e_ = (call);                            \
    if (e_ != cudaSuccess) return ecuda(e_, #call);     \
  } while (0)

int activate(lbm_ensemble* e) {
  if (e == nullptr) return efail(LBM_ERR_ARGUMENT, "null ensemble handle");
  cudaError_t r = cudaSetDevice(e->device);
  if (r != cudaSuccess) return ecuda(r, "cudaSetDevice");
  return LBM_OK;
}

void drop_graph(lbm_ensemble* e) {
  if (e->graph) cudaGraphExecDestroy(e->graph);
  e->graph = nullptr;
  e->graph_pairs = 0;
}

// (Re)builds the tile table for the current tile width.
int build_tiles(lbm_ensemble* e) {
  if (e->d_tiles && e->tiles_for == e->tile) return LBM_OK;
  std::vector<TileDesc> tiles;
  for (int d = 0; d < e->ndomains; ++d) {
    const DomainDesc& dom = e->domains[d];
    for (int x = 0; x < dom.nx; ++x)
      for (int z0 = 0; z0 < dom.ny; z0 += e->tile)
        tiles.push_back(TileDesc{d, x, z0, std::min(e->tile, dom.ny - z0)});
  }
  if (e->d_tiles) cudaFree(e->d_tiles);
  e->d_tiles = nullptr;
  ENS_CUDA(cudaMalloc((void**)&e->d_tiles, tiles.size() * sizeof(TileDesc)));
  ENS_CUDA(cudaMemcpyAsync(e->d_tiles, tiles.data(), tiles.size() * sizeof(TileDesc),
                           cudaMemcpyHostToDevice, e->stream));
  ENS_CUDA(cudaStreamSynchronize(e->stream));
  e->ntiles = (long long)tiles.size();
  e->tiles_for = e->tile;
  drop_graph(e);
  return LBM_OK;
}

template <class Real>
lbm::StepArgs<Real> base_args(const lbm_ensemble* e, bool write_moments) {
  lbm::StepArgs<Real> a{};
  a.f = e->shell.f;
  a.rho = static_cast<Real*>(e->shell.rho);
  a.vel = static_cast<Real*>(e->shell.vel);
  a.flags = e->shell.flags;
  a.n = e->n;
  a.acc_mode = lbm::kAccNone;
  a.write_moments = write_moments ? 1 : 0;
  a.status = e->shell.status;
  return a;
}

template <bool TRT, int K>
cudaError_t launch_persistent(lbm_ensemble* e, bool even, bool write_moments) {
  using Real = typename lbm::Pop<K>::real;
  const lbm::StepArgs<Real> a = base_args<Real>(e, write_moments);
  const EnsembleArgs args{e->d_domains, e->d_tiles, e->ntiles};
  auto kern = even ? ensemble_step_kernel<TRT, K, true> : ensemble_step_kernel<TRT, K, false>;
  int per_sm = e->blocks_per_sm;
  if (per_sm <= 0) {
    cudaError_t r = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, e->tile / 2, 0);
    if (r != cudaSuccess) return r;
    if (per_sm < 1) per_sm = 1;
  }
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
  long long grid = (long long)sms * per_sm;
  if (grid > e->ntiles) grid = e->ntiles;
  kern<<<(unsigned)grid, e->tile / 2, 0, e->stream>>>(a, args);
  return cudaGetLastError();
}

template <bool TRT, int K>
cudaError_t launch_per_domain(lbm_ensemble* e, bool even, bool write_moments) {
  using Real = typename lbm::Pop<K>::real;
  using T = typename lbm::Pop<K>::type;
  for (int d = 0; d < e->ndomains; ++d) {
    const DomainDesc& dom = e->domains[d];
    lbm::StepArgs<Real> a = base_args<Real>(e, write_moments);
    a.f = static_cast<T*>(e->shell.f) + dom.base;  // stride stays the ensemble's n
    a.rho = static_cast<Real*>(e->shell.rho) + dom.base;
    a.vel = static_cast<Real*>(e->shell.vel) + 2 * dom.base;
    a.flags = e->shell.flags + dom.base;
    a.nx = 1;
    a.ny = dom.nx;
    a.nz = dom.ny;
    a.om_pos = dom.om_pos;
    a.om_neg = dom.om_neg;
    const int bx = a.nz >= 256 ? 256 : ((a.nz + 31) / 32) * 32;
    const dim3 grid((a.nz + bx - 1) / bx, a.ny, 1);
    if (even)
      lbm::aa_step_kernel<lbm::D2Q9, TRT, K, true, 0><<<grid, bx, 0, e->stream>>>(a);
    else
      lbm::aa_step_kernel<lbm::D2Q9, TRT, K, false, 0><<<grid, bx, 0, e->stream>>>(a);
    cudaError_t r = cudaGetLastError();
    if (r != cudaSuccess) return r;
  }
  return cudaSuccess;
}

template <bool TRT, int K>
cudaError_t launch_step(lbm_ensemble* e, bool even, bool write_moments, int mode) {
  if (mode == 2) return launch_per_domain<TRT, K>(e, even, write_moments);
  return launch_persistent<TRT, K>(e, even, write_moments);
}

cudaError_t step(lbm_ensemble* e, bool even, bool write_moments, int mode) {
  const bool trt = e->collision == LBM_TRT;
  switch (e->storage) {
    case LBM_STORAGE_F32:
      return trt ? launch_step<true, lbm::kF32>(e, even, write_moments, mode)
                 : launch_step<false, lbm::kF32>(e, even, write_moments, mode);
    case LBM_STORAGE_F16:
      return trt ? launch_step<true, lbm::kF16>(e, even, write_moments, mode)
                 : launch_step<false, lbm::kF16>(e, even, write_moments, mode);
    case LBM_STORAGE_BF16:
      return trt ? launch_step<true, lbm::kBF16>(e, even, write_moments, mode)
                 : launch_step<false, lbm::kBF16>(e, even, write_moments, mode);
  }
  return cudaErrorInvalidValue;
}

// A graph of `pairs` AA step pairs (no moment writes) in persistent mode, captured once.
int ensure_graph(lbm_ensemble* e, int pairs) {
  if (e->graph && e->graph_pairs == pairs && e->graph_tile == e->tile &&
      e->graph_blocks == e->blocks_per_sm)
    return LBM_OK;
  drop_graph(e);
  cudaGraph_t g = nullptr;
  ENS_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
  cudaError_t r = cudaSuccess;
  for (int p = 0; p < pairs && r == cudaSuccess; ++p) {
    r = step(e, true, false, 0);
    if (r == cudaSuccess) r = step(e, false, false, 0);
  }
  cudaError_t end = cudaStreamEndCapture(e->stream, &g);
  if (r != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return ecuda(r, "graph capture");
  }
  if (end != cudaSuccess) return ecuda(end, "cudaStreamEndCapture");
  r = cudaGraphInstantiate(&e->graph, g, 0);
  cudaGraphDestroy(g);
  if (r != cudaSuccess) return ecuda(r, "cudaGraphInstantiate");
  e->graph_pairs = pairs;
  e->graph_tile = e->tile;
  e->graph_blocks = e->blocks_per_sm;
  return LBM_OK;
}

void release(lbm_ensemble* e) {
  drop_graph(e);
  cudaFree(e->shell.f);
  cudaFree(e->shell.rho);
  cudaFree(e->shell.vel);
  cudaFree(e->shell.flags);
  cudaFree(e->shell.status);
  cudaFree(e->d_domains);
  cudaFree(e->d_tiles);
  if (e->stream) cudaStreamDestroy(e->stream);
}

}  // namespace

extern "C" {

int lbm_ensemble_create(int ndomains, const int64_t* counts, int collision,
                        const float* omega_pos, const float* omega_neg, int storage,
                        lbm_ensemble** out) {
  if (out == nullptr || counts == nullptr || omega_pos == nullptr)
    return efail(LBM_ERR_ARGUMENT, "null argument");
  *out = nullptr;
  if (ndomains <= 0) return efail(LBM_ERR_ARGUMENT, "an ensemble needs at least one domain");
  if (collision != LBM_BGK && collision != LBM_TRT)
    return efail(LBM_ERR_ARGUMENT, "unknown collision operator");
  if (storage != LBM_STORAGE_F32 && storage != LBM_STORAGE_F16 && storage != LBM_STORAGE_BF16)
    return efail(LBM_ERR_UNSUPPORTED, "ensembles store populations as f32, f16 or bf16");
  lbm_ensemble* e = new (std::nothrow) lbm_ensemble();
  if (e == nullptr) return efail(LBM_ERR_ARGUMENT, "out of host memory");
  e->ndomains = ndomains;
  e->collision = collision;
  e->storage = storage;
  long long n = 0;
  for (int d = 0; d < ndomains; ++d) {
    const int64_t nx = counts[2 * d], ny = counts[2 * d + 1];
    if (nx <= 0 || ny <= 0) {
      delete e;
      return efail(LBM_ERR_ARGUMENT, "domain counts must be positive");
    }
    DomainDesc dom{n, (int)nx, (int)ny, omega_pos[d], omega_neg ? omega_neg[d] : 0.0f};
    e->domains.push_back(dom);
    n += nx * ny;
  }
  if (n >= ((long long)1 << 32)) {
    delete e;
    return efail(LBM_ERR_ARGUMENT, "ensemble too large (2^32 cells)");
  }
  e->n = n;
  auto bail = [&](cudaError_t r, const char* where) {
    release(e);
    delete e;
    return ecuda(r, where);
  };
  cudaError_t r;
  if ((r = cudaGetDevice(&e->device)) != cudaSuccess) return bail(r, "cudaGetDevice");
  if ((r = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return bail(r, "cudaStreamCreate");
  lbm_sim& s = e->shell;
  s.dim = 2;
  s.q = 9;
  s.collision = collision;
  s.storage = storage;
  s.counts[0] = 1;
  s.counts[1] = n;
  s.n = n;
  s.device = e->device;
  s.stream = e->stream;
  const size_t flag_bytes = ((size_t)n + 255) / 256 * 256;
  if ((r = cudaMalloc(&s.f, (size_t)n * 9 * lbm::pop_bytes(storage))) != cudaSuccess ||
      (r = cudaMalloc(&s.rho, (size_t)n * sizeof(float))) != cudaSuccess ||
      (r = cudaMalloc(&s.vel, (size_t)n * 2 * sizeof(float))) != cudaSuccess ||
      (r = cudaMalloc((void**)&s.flags, flag_bytes)) != cudaSuccess ||
      (r = cudaMalloc((void**)&s.status, 64 * sizeof(double))) != cudaSuccess ||
      (r = cudaMalloc((void**)&e->d_domains, ndomains * sizeof(DomainDesc))) != cudaSuccess)
    return bail(r, "cudaMalloc");
  s.sums = reinterpret_cast<double*>(s.status) + 1;
  if ((r = cudaMemsetAsync(s.flags, 0, flag_bytes, e->stream)) != cudaSuccess ||
      (r = cudaMemsetAsync(s.status, 0, 64 * sizeof(double), e->stream)) != cudaSuccess ||
      (r = cudaMemcpyAsync(e->d_domains, e->domains.data(), ndomains * sizeof(DomainDesc),
                           cudaMemcpyHostToDevice, e->stream)) != cudaSuccess ||
      (r = cudaStreamSynchronize(e->stream)) != cudaSuccess)
    return bail(r, "initialise ensemble");
  if (int rc = build_tiles(e)) {
    release(e);
    delete e;
    return rc;
  }
  *out = e;
  return LBM_OK;
}

int lbm_ensemble_destroy(lbm_ensemble* e) {
  if (e == nullptr) return LBM_OK;
  cudaSetDevice(e->device);
  cudaStreamSynchronize(e->stream);
  release(e);
  delete e;
  return LBM_OK;
}

int lbm_ensemble_cells(lbm_ensemble* e, int64_t* total) {
  if (int rc = activate(e)) return rc;
  if (total) *total = e->n;
  return LBM_OK;
}

int lbm_ensemble_set_shape(lbm_ensemble* e, int tile_cells, int blocks_per_sm) {
  if (int rc = activate(e)) return rc;
  if (tile_cells < 32 || tile_cells > 512 || tile_cells % 32 != 0)
    return efail(LBM_ERR_ARGUMENT, "tile_cells must be a multiple of 32 in [32, 512]");
  if (blocks_per_sm < 0 || blocks_per_sm > 64)
    return efail(LBM_ERR_ARGUMENT, "blocks_per_sm must be in [0, 64]");
  e->tile = tile_cells;
  e->blocks_per_sm = blocks_per_sm;
  return build_tiles(e);
}

int lbm_ensemble_upload(lbm_ensemble* e, const int32_t* flags, const float* rho,
                        const float* vel) {
  if (int rc = activate(e)) return rc;
  if (flags) {
    if (int rc = lbm_upload_flags(&e->shell, flags)) return rc;
  }
  if (rho || vel) {
    if (int rc = lbm_upload_fluid(&e->shell, rho, vel)) return rc;
  }
  return LBM_OK;
}

int lbm_ensemble_equilibrate(lbm_ensemble* e) {
  if (int rc = activate(e)) return rc;
  return lbm_equilibrate(&e->shell);
}

int lbm_ensemble_iterate(lbm_ensemble* e, int64_t iters, int mode) {
  if (int rc = activate(e)) return rc;
  if (iters < 0 || iters % 2 != 0) return efail(LBM_ERR_ARGUMENT, "iters must be even");
  if (mode < 0 || mode > 2) return efail(LBM_ERR_ARGUMENT, "unknown ensemble mode");
  if (iters == 0) return LBM_OK;
  int64_t pairs = iters / 2 - 1;  // the last pair ends with the moment write
  if (mode == 1 && pairs > 0) {
    const int chunk = (int)std::min<int64_t>(pairs, 50);
    if (int rc = ensure_graph(e, chunk)) return rc;
    while (pairs >= chunk) {
      ENS_CUDA(cudaGraphLaunch(e->graph, e->stream));
      pairs -= chunk;
    }
  }
  for (int64_t p = 0; p < pairs; ++p) {
    cudaError_t r = step(e, true, false, mode == 2 ? 2 : 0);
    if (r == cudaSuccess) r = step(e, false, false, mode == 2 ? 2 : 0);
    if (r != cudaSuccess) return ecuda(r, "ensemble step");
  }
  cudaError_t r = step(e, true, false, mode == 2 ? 2 : 0);
  if (r == cudaSuccess) r = step(e, false, true, mode == 2 ? 2 : 0);
  if (r != cudaSuccess) return ecuda(r, "ensemble step");
  return LBM_OK;
}

int lbm_ensemble_download(lbm_ensemble* e, float* rho, float* vel) {
  if (int rc = activate(e)) return rc;
  return lbm_download_fluid(&e->shell, rho, vel);
}

int lbm_ensemble_upload_f(lbm_ensemble* e, const float* f) {
  if (int rc = activate(e)) return rc;
  return lbm_upload_f(&e->shell, f);
}

int lbm_ensemble_download_f(lbm_ensemble* e, float* f) {
  if (int rc = activate(e)) return rc;
  return lbm_download_f(&e->shell, f);
}

int lbm_ensemble_stream(lbm_ensemble* e, void** stream) {
  if (int rc = activate(e)) return rc;
  if (stream) *stream = (void*)e->stream;
  return LBM_OK;
}

int lbm_ensemble_synchronize(lbm_ensemble* e) {
  if (int rc = activate(e)) return rc;
  return lbm_synchronize(&e->shell);
}

}  // extern "C"
