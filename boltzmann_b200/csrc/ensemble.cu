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
// Two kernels walk the domains:
//   rows (default whenever every row has at most 512 cells): one domain row per work item. A
//     producer warp copies, with one TMA bulk copy per population slot, the 16-byte-aligned
//     superset of the row that slot is read from (on even steps rows x-1, x, x+1 of the domain,
//     wrapped; on odd steps row x) plus the row's flags into a ring of shared-memory stages,
//     completing on the stage's mbarrier; four consumer warps collide from shared memory (the
//     periodic z-wrap is an index wrap in the stage) and store the results with coalesced
//     per-thread stores. The loads of several rows stay in flight while others are computed, so
//     no thread waits on HBM latency.
//   tiles: row segments of `tile` cells, two cells per thread, loads straight into registers
//     (lbm_ensemble_set_shape with a tile width; the only kernel for rows over 512 cells).
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
#include "aa_tma.cuh"
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

// ---- The row-staged kernel.

constexpr int kRowMax = 512;               // longest domain row the staged kernel takes
constexpr int kRowConsumerWarps = 4;       // 128 threads: up to four cells each per row
constexpr int kRowThreads = 32 * kRowConsumerWarps + 32;  // + the producer warp

struct RowDesc {
  int domain;
  int x;  // row of the domain (the reference's x)
};

struct RowArgs {
  const DomainDesc* domains;
  const RowDesc* rows;
  long long nrows;
};

// Written by the producer into each stage next to the copies: where the row's cells are and
// where each copied segment starts inside its stage slot.
struct RowHead {
  unsigned row[3];        // first cell of rows x-1, x, x+1 of the domain (wrapped)
  int ny;                 // cells in the row
  float om_pos, om_neg;   // the domain's relaxation rates
  unsigned char off[10];  // slots 0-8 and the flags: element offset of the row in its segment
};

template <int K>
struct RowStage {
  using T = typename lbm::Pop<K>::type;
  static constexpr int kSlack = 16 / (int)sizeof(T);  // elements before a 16-byte boundary
  static constexpr int SEG = kRowMax + kSlack;         // elements per slot segment
  static constexpr size_t seg_bytes = (size_t)SEG * sizeof(T);
  static_assert(seg_bytes % 16 == 0, "slot segments start on 16-byte boundaries");
  static constexpr size_t off_flags = 9 * seg_bytes;
  static constexpr size_t off_head = off_flags + kRowMax + 16;
  static constexpr size_t bytes = (off_head + sizeof(RowHead) + 127) / 128 * 128;
  // Ring depth: two stages (38 KB) a CTA for 32-bit populations and three (30 KB) for 16-bit
  // ones, so that five to seven CTAs share an SM: the consumers' cell updates, not the loads,
  // need the warps.
  static constexpr int stages = sizeof(T) == 4 ? 2 : 3;
};

// Slots whose velocity has a positive / negative component along internal axis 1 (the
// reference's x), as bit masks: a runtime slot index then needs no table in local memory.
__host__ __device__ constexpr unsigned row_shift_mask(int sign) {
  unsigned m = 0;
  for (int i = 0; i < lbm::D2Q9::Q; ++i)
    if (lbm::comp<lbm::D2Q9>(i, 1) * sign > 0) m |= 1u << i;
  return m;
}

template <int K>
constexpr size_t row_smem_bytes() {
  return RowStage<K>::stages * RowStage<K>::bytes + 2 * RowStage<K>::stages * sizeof(uint64_t);
}

// update_cell's AA store for a row work item with 32-bit populations: slot i of each result goes
// to its row (the row upstream of c_i on even steps, the row itself on odd steps), whose first
// element the consumer addresses once per row, so a store is one add to a pointer held in
// registers (+1.3% on the 512-cavity FP32 ensemble; the 16-bit kernel, short of registers,
// measured 1.8% slower with it and keeps update_cell's own store).
template <int K>
struct RowStoreSink {
  using T = typename lbm::Pop<K>::type;
  using Real = typename lbm::Pop<K>::real;
  T* const* rows;  // slot i's row, at its position 0

  template <class L, class P, bool EVEN, bool DEV>
  __device__ __forceinline__ void fluid(T*, long long, const lbm::CellPos& c,
                                        const Real (&v)[L::Q]) const {
#pragma unroll
    for (int i = 0; i < L::Q; ++i) {
      const int cz = lbm::comp<L>(i, 2);
      const unsigned zi = !EVEN ? c.oz[1] : (cz > 0 ? c.oz[0] : (cz < 0 ? c.oz[2] : c.oz[1]));
      const Real val = EVEN ? v[lbm::opp(i)] : v[i];
      if constexpr (DEV)
        P::store_dev(rows[i] + zi, val, lbm::weight<L, Real>(i));
      else
        P::store(rows[i] + zi, val, lbm::weight<L, Real>(i));
    }
  }
  template <class TL, class TP, bool EVEN>
  __device__ __forceinline__ void tracer(typename TP::type*, long long, const lbm::CellPos&,
                                         const typename TP::real (&)[TL::Q]) const {}
};

template <bool TRT, int K, bool EVEN>
__global__ void __launch_bounds__(kRowThreads)
    ensemble_rows_kernel(const __grid_constant__ lbm::StepArgs<typename lbm::Pop<K>::real> a,
                         const RowArgs e) {
  using namespace lbm;
  using P = Pop<K>;
  using Real = typename P::real;
  using T = typename P::type;
  using St = RowStage<K>;
  constexpr int S = St::stages;
  constexpr int CW = kRowConsumerWarps;

  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)S * St::bytes);
  uint64_t* empty = full + S;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // This CTA's rows: blockIdx.x + j * gridDim.x, j = 0 .. count-1.
  const int count =
      (long long)blockIdx.x < e.nrows ? (int)((e.nrows - 1 - blockIdx.x) / gridDim.x + 1) : 0;
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, CW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  if (warp == CW) {
    // ---- producer warp: lane k < 9 copies slot k, lane 9 the flags.
    // Row descriptors are loaded two rows ahead and domain descriptors one row ahead, so that
    // the dependent table loads never hold up the copies of the next row.
    const long long r0 = blockIdx.x, dr = gridDim.x;
    RowDesc rd_next{0, 0}, rd_after{0, 0};
    DomainDesc dom_next{0, 1, 1, 0.0f, 0.0f};
    if (count > 0) rd_next = e.rows[r0];
    if (count > 1) rd_after = e.rows[r0 + dr];
    if (count > 0) dom_next = e.domains[rd_next.domain];
    bool ok = true;
    int produced = 0;
    for (int j = 0; j < count && ok; ++j) {
      const int s = j % S;
      const RowDesc rd = rd_next;
      const DomainDesc dom = dom_next;
      rd_next = rd_after;
      if (j + 2 < count) rd_after = e.rows[r0 + (long long)(j + 2) * dr];
      if (j + 1 < count) dom_next = e.domains[rd_next.domain];
      if (j >= S) ok = mbar_wait(empty + s, (unsigned)(((j / S) - 1) & 1), a.spin_limit);
      if (!__all_sync(0xffffffffu, ok)) {
        ok = false;
        break;
      }
      const unsigned ny = (unsigned)dom.ny;
      const unsigned rowx = (unsigned)dom.base + (unsigned)rd.x * ny;
      const unsigned rowm = (unsigned)dom.base + (unsigned)(rd.x == 0 ? dom.nx - 1 : rd.x - 1) * ny;
      const unsigned rowp = (unsigned)dom.base + (unsigned)(rd.x == dom.nx - 1 ? 0 : rd.x + 1) * ny;
      unsigned char* st = smem + (size_t)s * St::bytes;
      uintptr_t lo = 0, addr = 0;
      unsigned bytes = 0, dst = 0;
      int es = 1;
      if (lane < 9) {
        // Even steps read slot i of the row upstream of c_i (internal axis 1: the reference's
        // x); odd steps read the row itself.
        constexpr unsigned kPlus = row_shift_mask(1), kMinus = row_shift_mask(-1);
        const unsigned row = !EVEN ? rowx
                                   : (((kPlus >> lane) & 1u) ? rowm
                                                             : (((kMinus >> lane) & 1u) ? rowp : rowx));
        addr = reinterpret_cast<uintptr_t>(static_cast<const T*>(a.f) + (size_t)lane * a.n + row);
        es = (int)sizeof(T);
        dst = (unsigned)(lane * St::seg_bytes);
      } else if (lane == 9) {
        addr = reinterpret_cast<uintptr_t>(a.flags + rowx);
        dst = (unsigned)St::off_flags;
      }
      if (lane < 10) {
        // The 16-byte-aligned superset of the row's ny elements (at most ny + 16 bytes: it fits
        // the segment, and the arrays are padded so that it stays inside their allocations).
        lo = addr & ~(uintptr_t)15;
        const uintptr_t hi = (addr + (uintptr_t)ny * es + 15) & ~(uintptr_t)15;
        bytes = (unsigned)(hi - lo);
      }
      const unsigned expect = __reduce_add_sync(0xffffffffu, bytes);
      RowHead* h = reinterpret_cast<RowHead*>(st + St::off_head);
      if (lane < 10) h->off[lane] = (unsigned char)((addr - lo) / (uintptr_t)es);
      if (lane == 0) {
        h->row[0] = rowm;
        h->row[1] = rowx;
        h->row[2] = rowp;
        h->ny = (int)ny;
        h->om_pos = dom.om_pos;
        h->om_neg = dom.om_neg;
      }
      __syncwarp();
      if (lane == 0) mbar_expect_tx(full + s, expect);  // releases the header writes too
      __syncwarp();
      if (bytes) bulk_copy(st + dst, reinterpret_cast<const void*>(lo), bytes, full + s);
      produced = j + 1;
    }
    if (!ok && lane == 0) atomicOr(a.status, 2);
    // Leave only once the copies of the last stages have landed (bounded), so that no copy
    // writes into shared memory after the CTA is gone.
    if (lane == 0)
      for (int j = produced - S > 0 ? produced - S : 0; j < produced; ++j)
        mbar_wait(full + j % S, (unsigned)((j / S) & 1));
    return;
  }

  // ---- consumer warps: thread tid updates cells tid, tid + 128, ... of every row.
  for (int j = 0; j < count; ++j) {
    const int s = j % S;
    const bool ok =
        __all_sync(0xffffffffu, mbar_wait(full + s, (unsigned)((j / S) & 1), a.spin_limit));
    if (!ok) {
      if (lane == 0) atomicOr(a.status, 2);
      break;  // the producer's own waits are bounded too
    }
    const unsigned char* st = smem + (size_t)s * St::bytes;
    // The row's header into registers once (the cell loop's global stores could otherwise alias
    // it, as far as the compiler knows, and force a reload per cell).
    const RowHead& h = *reinterpret_cast<const RowHead*>(st + St::off_head);
    const int ny = h.ny;
    const unsigned row0 = h.row[0], row1 = h.row[1], row2 = h.row[2];
    const Real om_p = (Real)h.om_pos, om_n = (Real)h.om_neg;
    const T* seg[D2Q9::Q];
#pragma unroll
    for (int i = 0; i < D2Q9::Q; ++i)
      seg[i] = reinterpret_cast<const T*>(st + (size_t)i * St::seg_bytes) + h.off[i];
    const unsigned char* fl = st + St::off_flags + h.off[9];
    T* out_rows[D2Q9::Q];
    if constexpr (sizeof(T) == 4) {
      constexpr unsigned kPlus = row_shift_mask(1), kMinus = row_shift_mask(-1);
#pragma unroll
      for (int i = 0; i < D2Q9::Q; ++i) {
        const unsigned row =
            !EVEN ? row1 : (((kPlus >> i) & 1u) ? row0 : (((kMinus >> i) & 1u) ? row2 : row1));
        out_rows[i] = static_cast<T*>(a.f) + (size_t)i * a.n + row;
      }
    }
    for (int z = tid; z < ny; z += 32 * CW) {
      CellPos c;
      c.ox[0] = c.ox[1] = c.ox[2] = 0u;
      c.oy[0] = row0;
      c.oy[1] = row1;
      c.oy[2] = row2;
      c.oz[0] = (unsigned)(z == 0 ? ny - 1 : z - 1);
      c.oz[1] = (unsigned)z;
      c.oz[2] = (unsigned)(z == ny - 1 ? 0 : z + 1);
      c.cell = row1 + (unsigned)z;
      const int flag = fl[z];
      Real fv[D2Q9::Q];
#pragma unroll
      for (int i = 0; i < D2Q9::Q; ++i) {
        const int slot = EVEN ? i : opp(i);
        // even: the upstream cell's z is z - c_iz, wrapped
        const int cz = comp<D2Q9>(i, 2);
        const unsigned zi = !EVEN ? (unsigned)z : (cz > 0 ? c.oz[0] : (cz < 0 ? c.oz[2] : c.oz[1]));
        if constexpr (dev_in<K>())
          fv[i] = P::load_dev(seg[slot] + zi, weight<D2Q9, Real>(i));
        else
          fv[i] = P::load(seg[slot] + zi, weight<D2Q9, Real>(i));
      }
      Real g[1];
      // (ensembles carry no body force, coupling or relaxation field)
      if constexpr (sizeof(T) == 4)
        update_cell<D2Q9, TRT, K, EVEN, 0, RowStoreSink<K>, default_tracer_kind<K>(), true>(
            a, c, flag, fv, g, Real(0), om_p, om_n, RowStoreSink<K>{out_rows});
      else
        update_cell<D2Q9, TRT, K, EVEN, 0, GlobalSink, default_tracer_kind<K>(), true>(
            a, c, flag, fv, g, Real(0), om_p, om_n);
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(empty + s);  // this warp is done with stage s
  }
}

}  // namespace

struct lbm_ensemble {
  int ndomains = 0, collision = 0, storage = 0;
  std::vector<DomainDesc> domains;
  long long n = 0;                 // total cells
  int tile = 0;                    // cells per tile (tile / 2 threads); 0: the row-staged kernel
  int blocks_per_sm = 0;           // 0: occupancy limit
  int device = 0;
  cudaStream_t stream = nullptr;
  lbm_sim shell;                   // describes the concatenated arrays for the field kernels
  DomainDesc* d_domains = nullptr;
  TileDesc* d_tiles = nullptr;
  long long ntiles = 0;
  int tiles_for = -1;              // tile width the table was built for
  RowDesc* d_rows = nullptr;       // the row table of the row-staged kernel (tile == 0)
  long long nrows = 0;
  int max_row = 0;                 // longest row (cells)
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

// (Re)builds the tile table for the current tile width, or the row table (tile == 0).
int build_tiles(lbm_ensemble* e) {
  if (e->tiles_for == e->tile) return LBM_OK;
  if (e->tile == 0) {
    if (e->d_rows == nullptr) {
      std::vector<RowDesc> rows;
      for (int d = 0; d < e->ndomains; ++d)
        for (int x = 0; x < e->domains[d].nx; ++x) rows.push_back(RowDesc{d, x});
      ENS_CUDA(cudaMalloc((void**)&e->d_rows, rows.size() * sizeof(RowDesc)));
      ENS_CUDA(cudaMemcpyAsync(e->d_rows, rows.data(), rows.size() * sizeof(RowDesc),
                               cudaMemcpyHostToDevice, e->stream));
      ENS_CUDA(cudaStreamSynchronize(e->stream));
      e->nrows = (long long)rows.size();
    }
    e->tiles_for = 0;
    drop_graph(e);
    return LBM_OK;
  }
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

template <bool TRT, int K, bool EVEN>
cudaError_t launch_rows_parity(lbm_ensemble* e, bool write_moments) {
  using Real = typename lbm::Pop<K>::real;
  auto kern = ensemble_rows_kernel<TRT, K, EVEN>;
  constexpr size_t smem = row_smem_bytes<K>();
  static std::once_flag once;
  static cudaError_t setup_err = cudaSuccess;
  static int occupancy = 1;
  std::call_once(once, [&] {
    setup_err = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (setup_err == cudaSuccess)
      setup_err =
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occupancy, kern, kRowThreads, smem);
    if (occupancy < 1) occupancy = 1;
  });
  if (setup_err != cudaSuccess) return setup_err;
  const int per_sm = e->blocks_per_sm > 0 ? std::min(e->blocks_per_sm, occupancy) : occupancy;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, e->device);
  long long grid = (long long)sms * per_sm;
  if (grid > e->nrows) grid = e->nrows;
  lbm::StepArgs<Real> a = base_args<Real>(e, write_moments);
  a.spin_limit = lbm::kSpinLimit;
  kern<<<(unsigned)grid, kRowThreads, smem, e->stream>>>(a, RowArgs{e->d_domains, e->d_rows,
                                                                    e->nrows});
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
  if (e->tile == 0)
    return even ? launch_rows_parity<TRT, K, true>(e, write_moments)
                : launch_rows_parity<TRT, K, false>(e, write_moments);
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
  cudaFree(e->d_rows);
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
    e->max_row = std::max(e->max_row, (int)ny);
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
  // Rows longer than the staged kernel's stages go through the tile kernel.
  e->tile = e->max_row <= kRowMax ? 0 : 256;
  const size_t flag_bytes = ((size_t)n + 255) / 256 * 256;
  // 256 bytes of padding after the populations: the staged kernel's aligned row copies may
  // reach up to 15 bytes past the last slot's last row.
  if ((r = cudaMalloc(&s.f, (size_t)n * 9 * lbm::pop_bytes(storage) + 256)) != cudaSuccess ||
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
  if (tile_cells != 0 && (tile_cells < 32 || tile_cells > 512 || tile_cells % 32 != 0))
    return efail(LBM_ERR_ARGUMENT, "tile_cells must be 0 or a multiple of 32 in [32, 512]");
  if (tile_cells == 0 && e->max_row > kRowMax)
    return efail(LBM_ERR_UNSUPPORTED, "the row-staged kernel takes rows of at most 512 cells");
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
