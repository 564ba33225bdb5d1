// TMA-staged variant of the AA step: the main kernel for domains whose contiguous axis is a
// multiple of 256 cells (kTmaTile).
//
// Work unit: a tile of T consecutive cells of one grid row (T threads, one cell each). A
// persistent CTA walks its tiles with an S-stage ring in shared memory. For every tile, the
// producer warp moves each operand row segment with a single bulk copy (cp.async.bulk, the TMA
// engine, completion counted on the stage's mbarrier): per direction i the T populations the
// tile needs -- on even steps slot i of the upstream row segment, which is shifted by -c_iz, so
// the copy takes a 16-byte-aligned superset with H = 16 / sizeof(T) extra elements on the side
// the shift reaches (pieces past the row ends come from the other end: the domain is periodic;
// when a row is a single tile the plain row is copied and the index wraps in shared memory) --
// plus the fused tracer's populations, the coupled tracer value and the flag bytes.
// Threads read their operands from shared memory (consecutive threads, consecutive words: no
// bank conflicts), collide, and write their results back into the stage at the positions they
// read; the producer warp writes the stage back with one bulk store per row segment
// (cp.async.bulk shared -> global) before refilling it. Even steps on rows longer than one tile
// have shifted segments: there the bulk store takes the segment's 16-byte chunks and the cells
// at the tile's ends store the few results outside them (edge_range).
// 16-bit populations: two cells a consumer thread on packed FP32 instructions (aa_pair.cuh) for
// D3Q27 BGK without a tracer and for D2Q9.
//
// In-flight data is bounded by shared memory, not by registers, and the copy engine issues one
// instruction per row segment instead of one per element. Odd steps, which read their own row of
// every slot, take all slots of an array in one tensor-map copy (cp.async.bulk.tensor, a box of
// 256 cells by Q slots) when the launcher provides the maps.
//
// Synchronisation: stage s has a `full` mbarrier (the producer's expect_tx plus the copies'
// bytes) and an `empty` one (one arrival per consumer warp, once its results are in the stage).
// Before refilling stage s the producer waits on `empty`, issues the stage's bulk stores and
// waits until they have read it. There is no CTA-wide barrier in the loop. Every wait is
// bounded: on timeout the kernel sets bit 1 (value 2) of the status word and leaves.
// Every population slot is still read and written by exactly one thread per step, and no tile
// writes what another tile of the same step reads, so stores need no ordering with the copies.
#pragma once

#include <cuda.h>

#include <cstdint>

#include "aa_step.cuh"

namespace lbm {

constexpr int kTmaTile = 256;       // threads and cells per tile
constexpr unsigned kSpinLimit = 1u << 22;  // mbarrier try_wait polls before giving up

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Bounded wait for the phase with the given parity; false after `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity,
                                          unsigned limit = kSpinLimit) {
  const unsigned addr = smem_u32(bar);
  for (unsigned i = 0; i < limit; ++i) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// One bulk copy global -> shared, completing on `bar`. Addresses 16-byte aligned, size a
// multiple of 16.
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, unsigned bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::
          "r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Tensor-map copies of the odd step: the population (or tracer) array seen as a [slots][cells]
// matrix, one {256 cells x all slots} box per tile, landing as [slot][256] in the stage.
struct TmaMaps {
  CUtensorMap f;  // odd steps: populations, box {256, Q}; even steps of one-tile rows: the
                  // population array as rows of 256 cells, row (slot, x, y), box {256, 1}
  CUtensorMap g;  // odd steps: fused tracer populations, box {256, Qt}
  int use;        // 1 when the maps this launch needs are valid
};

__device__ __forceinline__ void tensor_copy_2d(void* dst, const CUtensorMap* map, int c0, int c1,
                                               uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, "
      "{%2, %3}], [%4];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
      : "memory");
}

// The reverse: one box from shared memory back to the tensor (completion tracked by the bulk
// group, like bulk_store). The coordinates are non-negative and the inner one a multiple of 256.
__device__ __forceinline__ void tensor_store_2d(const CUtensorMap* map, int c0, int c1,
                                                const void* src) {
  asm volatile(
      "cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(
          reinterpret_cast<uint64_t>(map)),
      "r"(c0), "r"(c1), "r"(smem_u32(src))
      : "memory");
}

// Four rows of a 2D tensor (x from 0, rows r0..r3; a box one row high) into four consecutive
// rows of shared memory, and the reverse.
__device__ __forceinline__ void tensor_gather4(void* dst, const CUtensorMap* map, int r0, int r1,
                                               int r2, int r3, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes "
      "[%0], [%1, {%2, %3, %4, %5, %6}], [%7];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(r0), "r"(r1), "r"(r2), "r"(r3),
      "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void tensor_scatter4(const CUtensorMap* map, int r0, int r1, int r2,
                                                int r3, const void* src) {
  asm volatile(
      "cp.async.bulk.tensor.2d.global.shared::cta.tile::scatter4.bulk_group "
      "[%0, {%1, %2, %3, %4, %5}], [%6];\n" ::"l"(reinterpret_cast<uint64_t>(map)),
      "r"(0), "r"(r0), "r"(r1), "r"(r2), "r"(r3), "r"(smem_u32(src))
      : "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}

// One bulk copy shared -> global (16-byte aligned addresses, size a multiple of 16).
__device__ __forceinline__ void bulk_store(void* dst, const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(dst),
               "r"(smem_u32(src)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() {
  asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
}
// This thread's bulk stores have read their shared-memory source (the stage may be refilled).
__device__ __forceinline__ void bulk_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
}
// This thread's bulk stores have completed.
__device__ __forceinline__ void bulk_wait_all() {
  asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
}

// Shared-memory layout of one stage, in elements of each operand's type.
// WR: rows of one tile (even steps then copy whole rows and need no halo).
template <class L, int K, int NT, bool EVEN, bool WR = false, int KT = default_tracer_kind<K>()>
struct TmaStage {
  using T = typename Pop<K>::type;
  using Real = typename Pop<K>::real;
  using TP = TracerPop<KT>;       // the fused tracer's population storage
  using TT = typename TP::type;
  using TL = typename TracerLattice<L::D>::type;
  static constexpr int Q = L::Q;
  static constexpr bool kWR = WR;
  static constexpr int NG = NT == 1 ? TL::Q : 0;
  static constexpr int H = EVEN && !WR ? 16 / (int)sizeof(T) : 0;      // population halo
  static constexpr int HG = EVEN && !WR ? 16 / (int)sizeof(TT) : 0;    // tracer halo
  static constexpr int SEG = kTmaTile + 2 * H;                   // populations per direction
  static constexpr int SEGG = kTmaTile + 2 * HG;
  // Even steps of one-tile rows move slots four rows at a time; the last group is padded with
  // repeats of slot Q - 1 into rows Q .. QP - 1 of the stage.
  static constexpr int QP = EVEN && WR ? 4 * ((Q + 3) / 4) : Q;
  static constexpr size_t pop_bytes = (size_t)QP * SEG * sizeof(T);
  static constexpr size_t trc_bytes = ((size_t)NG * SEGG * sizeof(TT) + 15) / 16 * 16;
  static constexpr size_t val_bytes = (size_t)kTmaTile * sizeof(Real);
  static constexpr size_t flag_bytes = kTmaTile;
  // offsets (bytes) inside a stage; every part 16-byte aligned, stages 128-byte aligned (the
  // tensor copies' shared-memory boxes start on 128 bytes)
  static constexpr size_t off_trc = pop_bytes;
  static constexpr size_t off_val = off_trc + trc_bytes;
  static constexpr size_t off_flag = off_val + val_bytes;
  static constexpr size_t bytes = (off_flag + flag_bytes + 127) / 128 * 128;
};

template <class L, int K, int NT, bool EVEN, int S, bool WR = false,
          int KT = default_tracer_kind<K>()>
__host__ __device__ constexpr size_t tma_smem_bytes() {
  return (size_t)S * TmaStage<L, K, NT, EVEN, WR, KT>::bytes + 16 * S;  // + full/empty mbarriers
}

// Bulk-copies the row segment [z0 - hl, z0 + T + hr) of one operand row (elements of `es` bytes)
// into dst, taking the parts left of 0 / right of nz from the other end of the row.
__device__ __forceinline__ void copy_row_segment(unsigned char* dst, const unsigned char* row,
                                                 int z0, int hl, int hr, int nz, int es,
                                                 uint64_t* bar) {
  const int lo = z0 - hl, hi = z0 + kTmaTile + hr;
  if (lo < 0)  // wrapped left halo: [nz + lo, nz)
    bulk_copy(dst, row + (size_t)(nz + lo) * es, (unsigned)(-lo * es), bar);
  const int a = lo < 0 ? 0 : lo, b = hi > nz ? nz : hi;
  bulk_copy(dst + (size_t)(a - lo) * es, row + (size_t)a * es, (unsigned)((b - a) * es), bar);
  if (hi > nz)  // wrapped right halo: [0, hi - nz)
    bulk_copy(dst + (size_t)(nz - lo) * es, row, (unsigned)((hi - nz) * es), bar);
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

// Index, inside its stage segment, of the population column `tid` reads and writes: its own
// column on odd steps; on even steps the upstream column tid - cz behind the segment's halo h,
// wrapped instead when rows are one tile (WR, no halo).
template <bool WR, bool EVEN>
__device__ __forceinline__ int stage_pos(int h, int tid, int cz) {
  if constexpr (!EVEN) return tid;
  if constexpr (WR) return (tid - cz) & (kTmaTile - 1);
  return h + tid - cz;
}

// Even steps of rows longer than one tile read slot i of their tile's cells from the row
// segment [z0 - c_iz, z0 - c_iz + 256) of the row upstream of c_i and write the results back to
// the same positions. The stage holds element z0 - h + k of the segment at index k (h = 16 bytes
// of elements, the halo), so the results are indices [h - c_iz, h - c_iz + 256): the producer
// stores the 16-byte chunks wholly inside that range with one bulk store, and the h elements
// left at its two ends (1 and h - 1, for c_iz != 0) come from the cells at the tile's ends.
struct EdgeRange {
  int first, last1;  // chunks [first, last1) of h elements lie wholly inside the result range
};
__host__ __device__ constexpr EdgeRange edge_range(int h, int cz) {
  return EdgeRange{(h - cz + h - 1) / h, (h - cz + kTmaTile) / h};
}

// Whether column tid's result for a slot with z-component cz falls outside the bulk-stored chunks.
__device__ __forceinline__ bool is_edge(int h, int tid, int cz) {
  const EdgeRange r = edge_range(h, cz);
  const int k = h + tid - cz;
  return k < r.first * h || k >= r.last1 * h;
}

// The results of one cell at a tile's end (column col, neighbourhood e) that fall outside the
// bulk-stored chunks, straight from its registers: fval(i) / gval(i) are its post-collision
// populations and first tracer's (stored as in the stage: deviations for the populations).
template <class St, class L, class P, class TP, int NT, class FV, class GV>
__device__ __forceinline__ void edge_stores(const StepArgs<typename P::real>& a, const CellPos& e,
                                            int col, FV fval, GV gval) {
  using Real = typename P::real;
  using TL = typename TracerLattice<L::D>::type;
  auto* f = static_cast<typename P::type*>(a.f);
#pragma unroll
  for (int i = 0; i < L::Q; ++i) {
    const int cz = comp<L>(i, 2);
    if (cz == 0 || !is_edge(St::H, col, cz)) continue;
    P::store_dev(f + (size_t)i * a.n + e.upstream<L>(i), fval(opp(i)), weight<L, Real>(i));
  }
  if constexpr (NT == 1) {
    auto* g = static_cast<typename TP::type*>(a.tr[0].g);
#pragma unroll
    for (int i = 0; i < TL::Q; ++i) {
      const int cz = comp<TL>(i, 2);
      if (cz == 0 || !is_edge(St::HG, col, cz)) continue;
      TP::store(g + (size_t)i * a.n + e.upstream<TL>(i), gval(opp(i)), 0.0f);
    }
  }
}

}  // namespace lbm

// The two-cells-a-thread update, which writes through stage_pos.
#include "aa_pair.cuh"

namespace lbm {

// update_cell's output into the stage it read from: slot i of the thread's cell on odd steps
// (position i, column tid), slot i of the upstream cell on even steps (the very position the
// thread read: shifted, and wrapped when a row is one tile). The producer then writes the stage
// back as row segments.
template <class St, class L, class TL>
struct StageSink {
  using Real = typename St::Real;
  unsigned char* st;
  int tid;

  template <class LL, class P, bool EVEN, bool DEV>
  __device__ __forceinline__ void fluid(typename P::type*, long long, const CellPos&,
                                        const typename P::real (&v)[LL::Q]) const {
    using T = typename P::type;
    T* base = reinterpret_cast<T*>(st);
#pragma unroll
    for (int i = 0; i < LL::Q; ++i) {
      T* p = base + i * St::SEG + stage_pos<St::kWR, EVEN>(St::H, tid, comp<LL>(i, 2));
      const Real val = EVEN ? v[opp(i)] : v[i];
      if constexpr (DEV)
        P::store_dev(p, val, weight<LL, Real>(i));
      else
        P::store(p, val, weight<LL, Real>(i));
    }
    if constexpr (EVEN && St::QP > LL::Q) {
      // The padding rows of the last four-row group repeat slot Q - 1 (the store writes them
      // to the same row again).
      constexpr int i = LL::Q - 1;
      const int pos = St::H + ((tid - comp<LL>(i, 2)) & (kTmaTile - 1));
      const T w = base[i * St::SEG + pos];
#pragma unroll
      for (int r = LL::Q; r < St::QP; ++r) base[r * St::SEG + pos] = w;
    }
  }
  template <class TLL, class TP, bool EVEN>
  __device__ __forceinline__ void tracer(typename TP::type*, long long, const CellPos&,
                                         const typename TP::real (&v)[TLL::Q]) const {
    using TT = typename TP::type;
    TT* base = reinterpret_cast<TT*>(st + St::off_trc);
#pragma unroll
    for (int i = 0; i < TLL::Q; ++i) {
      TT* p = base + i * St::SEGG + stage_pos<St::kWR, EVEN>(St::HG, tid, comp<TLL>(i, 2));
      TP::store(p, EVEN ? v[opp(i)] : v[i], 0.0f);
    }
  }
};

constexpr int kConsumerWarps = kTmaTile / 32;
constexpr int kTmaThreads = kTmaTile + 32;  // + one producer warp
// PAIR: each consumer thread updates two cells of the tile (tid and tid + 128), with half the
// consumer warps.
template <bool PAIR>
__host__ __device__ constexpr int tma_consumer_warps() {
  return PAIR ? kConsumerWarps / 2 : kConsumerWarps;
}
template <bool PAIR>
__host__ __device__ constexpr int tma_threads() {
  return 32 * tma_consumer_warps<PAIR>() + 32;
}

// CTAs per SM the register allocation is asked to allow. 32- and 64-bit populations: one, so
// the compiler keeps more of each cell in registers (~90 for FP32 D3Q27, ~80 for the fused
// D2Q9 + tracer even step) and two CTAs share an SM; measured 3-5% faster than three leaner CTAs.
// 16-bit populations move half the bytes and need the occupancy instead: three CTAs for D3Q27,
// four for D2Q9 (one CTA a SM cost them 15%). Two cells a thread: three CTAs for D3Q27, four for
// D2Q9 (~95 registers; five or six CTAs cap them at 81 / 68 and measured 9% / 32% slower on the
// FP16 channel).
template <class L, int K, bool PAIR = false>
constexpr int tma_min_blocks() {
  if constexpr (PAIR) return L::Q >= 27 ? 3 : 4;
  return (K == kF16 || K == kBF16) ? (L::Q >= 27 ? 3 : 4) : 1;
}

// Warp-specialised: warps 0..7 consume (one cell per thread), warp 8 loads and stores stages.
template <class L, bool TRT, int K, bool EVEN, int NT, int S, bool WR, bool PAIR = false,
          int KT = default_tracer_kind<K>()>
__global__ void __launch_bounds__(tma_threads<PAIR>(), tma_min_blocks<L, K, PAIR>())
    aa_tma_kernel(const __grid_constant__ StepArgs<typename Pop<K>::real> a,
                  const __grid_constant__ TmaMaps maps) {
  using P = Pop<K>;
  using Real = typename P::real;
  using T = typename P::type;
  using TL = typename TracerLattice<L::D>::type;
  using St = TmaStage<L, K, NT, EVEN, WR, KT>;
  using TP = TracerPop<KT>;
  using TT = typename TP::type;
  constexpr int Q = L::Q;

  extern __shared__ __align__(128) unsigned char smem[];
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + (size_t)S * St::bytes);
  uint64_t* empty = full + S;
  auto stage_ptr = [&](int s) { return smem + (size_t)s * St::bytes; };

  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int tiles_per_row = a.nz / kTmaTile;
  const long long ntiles = (long long)a.nx * a.ny * tiles_per_row;
  // This CTA's tiles: blockIdx.x + j * gridDim.x, j = 0 .. count-1.
  const int count =
      (long long)blockIdx.x < ntiles ? (int)((ntiles - 1 - blockIdx.x) / gridDim.x + 1) : 0;

  // This CTA's tiles in order, t = blockIdx.x + j * gridDim.x, as (x, y, tile within the row),
  // advanced by a fixed stride with carries: no division per tile (every thread walks the
  // tiles, so a division here would cost every cell).
  struct TileWalker {
    int x, y, zt, dx, dy, dz, ny, tpr;
    __device__ void init(long long t0, long long stride, int ny_, int tpr_) {
      ny = ny_;
      tpr = tpr_;
      const long long row = t0 / tpr, drow = stride / tpr;
      zt = (int)(t0 - row * tpr);
      dz = (int)(stride - drow * tpr);
      y = (int)(row % ny);
      x = (int)(row / ny);
      dy = (int)(drow % ny);
      dx = (int)(drow / ny);
    }
    __device__ void next() {
      zt += dz;
      const int carry = zt >= tpr ? 1 : 0;
      zt -= carry * tpr;
      y += dy + carry;
      const int cy = y >= ny ? 1 : 0;
      y -= cy * ny;
      x += dx + cy;
    }
  };

  // WR: every row is one tile (nz == T; even steps only). Every step leaves its results in the
  // stage, and the producer writes the stage back as row segments before refilling it (bulk
  // stores): whole segments on odd steps and on even steps of one-tile rows; on other even
  // steps, whose segments are shifted by c_iz, the 16-byte chunks wholly inside each segment,
  // while the cells at the tile's ends store the few results outside them from their registers
  // once their warp has released the stage (edge_range, edge_stores). (Per-thread stores of
  // every result straight from registers cost ~100 integer instructions per cell for their
  // addresses and made the 16-bit even step issue-bound; the producer storing the ragged ends
  // made it the limit; the end cells storing them before the release held back every stage.)
  constexpr bool whole_row = WR;
  constexpr int CW = tma_consumer_warps<PAIR>();
  static_assert(!PAIR || L::D == 2 || NT == 0, "two cells a thread in 3D: no tracer");
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, CW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  if (warp == CW) {
    // ---- producer warp. Each lane owns up to two copy jobs (job = lane, lane + 32), fixed for
    // the whole kernel and described once here: source array, row shift (even steps read slot i
    // of the row upstream of c_i), halo, element size, destination inside a stage.
    // A segment always lands so that its element z0 sits at index H of its slot in the stage.
    // Even steps read z0 + t - c_iz: a direction with c_iz = +1 needs the left halo only, -1 the
    // right one, 0 none. When a row is one tile (nz == T) the whole row is copied and consumers
    // wrap the index instead, so no segment needs a halo or a wrapped piece.
    struct Job {
      const unsigned char* base;  // first element of the operand array (slot array for populations)
      int cx, cy;                 // row shift: source row = (x - cx, y - cy)
      int hl, hr, es;             // left / right halo (elements), element size (bytes)
      unsigned dst;               // byte offset inside a stage of element z0 - hl
      int kind;                   // 0 none, 1 row segment with halo, 2 own tile (no halo)
      bool gathered;              // moved by the four-row tensor copies instead (see below)
      int so;                     // results: row elements [z0 + so, z0 + so + sbytes / es)
      unsigned sdst, sbytes;      // from this stage byte offset
    };
    // The bulk-stored part of a row segment's results: the whole tile, or on even steps of rows
    // longer than one tile the chunks of edge_range (the stage holds element z0 - h + k at
    // index k, h = 16 / es).
    auto set_store = [&](Job& jb, int cz) {
      jb.so = 0;
      jb.sdst = jb.dst;
      jb.sbytes = (unsigned)(kTmaTile * jb.es);
      if (EVEN && !whole_row) {
        const int h = 16 / jb.es;
        const EdgeRange r = edge_range(h, cz);
        jb.so = (r.first - 1) * h;
        jb.sdst = jb.dst + (unsigned)((r.first * h - (h - jb.hl)) * jb.es);
        jb.sbytes = (unsigned)((r.last1 - r.first) * h * jb.es);
      }
    };
    // Even steps of one-tile rows: the population slots travel four rows at a time
    // (tile::gather4 / scatter4 over the population array seen as rows of 256 cells, row
    // (slot, x, y)); lane k < NG4 moves slots 4k .. 4k + 3, the last group padded with repeats
    // of slot Q - 1.
    constexpr int NG4 = EVEN && WR ? St::QP / 4 : 0;
    const bool by_rows = NG4 > 0 && maps.use;
    Job jobs[2];
    unsigned lane_bytes = 0;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int op = lane + 32 * k;
      Job jb{nullptr, 0, 0, 0, 0, 1, 0u, 0, false, 0, 0u, 0u};
      if (op < Q) {
        const int slot = op;  // stage position op holds slot op (odd steps read opp(i) from it)
        const int cz = EVEN && !whole_row ? comp_rt<L, 2>(op) : 0;
        jb.base = reinterpret_cast<const unsigned char*>(static_cast<const T*>(a.f) +
                                                         (size_t)slot * a.n);
        jb.cx = EVEN ? comp_rt<L, 0>(op) : 0;
        jb.cy = EVEN ? comp_rt<L, 1>(op) : 0;
        jb.hl = cz > 0 ? St::H : 0;
        jb.hr = cz < 0 ? St::H : 0;
        jb.es = sizeof(T);
        jb.dst = (unsigned)(((size_t)op * St::SEG + St::H - jb.hl) * sizeof(T));
        jb.kind = 1;
        jb.gathered = by_rows;
        set_store(jb, cz);
      } else if (op < Q + St::NG) {
        if constexpr (NT == 1) {
          const int i = op - Q;
          const int slot = i;
          const int cz = EVEN && !whole_row ? comp_rt<TL, 2>(i) : 0;
          jb.base = static_cast<const unsigned char*>(a.tr[0].g) + (size_t)slot * a.n * sizeof(TT);
          jb.cx = EVEN ? comp_rt<TL, 0>(i) : 0;
          jb.cy = EVEN ? comp_rt<TL, 1>(i) : 0;
          jb.hl = cz > 0 ? St::HG : 0;
          jb.hr = cz < 0 ? St::HG : 0;
          jb.es = sizeof(TT);
          jb.dst = (unsigned)(St::off_trc + ((size_t)i * St::SEGG + St::HG - jb.hl) * sizeof(TT));
          jb.kind = 1;
          set_store(jb, cz);
        }
      } else if (op == Q + St::NG) {
        if (a.acc_mode == kAccBoussinesq) {
          jb.base = reinterpret_cast<const unsigned char*>(a.coupled_val);
          jb.es = sizeof(Real);
          jb.dst = (unsigned)St::off_val;
          jb.kind = 2;
        }
      } else if (op == Q + St::NG + 1) {
        jb.base = a.flags;
        jb.es = 1;
        jb.dst = (unsigned)St::off_flag;
        jb.kind = 2;
      }
      jobs[k] = jb;
      if (jb.kind != 0 && !jb.gathered)
        lane_bytes += (unsigned)((kTmaTile + jb.hl + jb.hr) * jb.es);
    }
    if (by_rows && lane < NG4) lane_bytes += 4u * kTmaTile * (unsigned)sizeof(T);
    const unsigned expect = __reduce_add_sync(0xffffffffu, lane_bytes);
    const long long plane = (long long)a.ny * a.nz;
    // First byte of the row a job's segment of tile (x, y) comes from: the tile's own row, or
    // the row upstream of the job's direction on even steps.
    auto job_row = [&](const Job& jb, int x, int y) {
      const int ux = jb.cx > 0 ? (x == 0 ? a.nx - 1 : x - 1) : (jb.cx < 0 ? (x == a.nx - 1 ? 0 : x + 1) : x);
      const int uy = jb.cy > 0 ? (y == 0 ? a.ny - 1 : y - 1) : (jb.cy < 0 ? (y == a.ny - 1 ? 0 : y + 1) : y);
      return jb.base + (size_t)(ux * plane + (long long)uy * a.nz) * jb.es;
    };
    // The rows of lane k's four gathered slots for tile (x, y).
    int gcx[4] = {0, 0, 0, 0}, gcy[4] = {0, 0, 0, 0};
    if (lane < NG4) {
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int slot = 4 * lane + m < Q ? 4 * lane + m : Q - 1;
        gcx[m] = comp_rt<L, 0>(slot);
        gcy[m] = comp_rt<L, 1>(slot);
      }
    }
    auto group_rows = [&](int x, int y, int (&r)[4]) {
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int ux = gcx[m] > 0 ? (x == 0 ? a.nx - 1 : x - 1) : (gcx[m] < 0 ? (x == a.nx - 1 ? 0 : x + 1) : x);
        const int uy = gcy[m] > 0 ? (y == 0 ? a.ny - 1 : y - 1) : (gcy[m] < 0 ? (y == a.ny - 1 ? 0 : y + 1) : y);
        const int slot = 4 * lane + m < Q ? 4 * lane + m : Q - 1;
        r[m] = slot * a.nx * a.ny + ux * a.ny + uy;
      }
    };
    // The consumers leave a tile's results in its stage: each population and tracer segment
    // goes back to the row it came from (set_store's part of it), and the stage is refilled once
    // the stores have read it.
    TileWalker tws;
    tws.init(blockIdx.x, gridDim.x, a.ny, tiles_per_row);
    auto store_stage = [&](int s) {
      const unsigned char* st = stage_ptr(s);
      if (!EVEN && maps.use) {
        // Odd steps: the tile's own row of every slot, the box the tensor-map load brought in.
        if (lane == 0) {
          const int cell0 = (int)((long long)tws.x * plane + (long long)tws.y * a.nz +
                                  (long long)tws.zt * kTmaTile);
          tensor_store_2d(&maps.f, cell0, 0, st);
          if constexpr (NT == 1) tensor_store_2d(&maps.g, cell0, 0, st + St::off_trc);
        }
      } else {
        if (by_rows && lane < NG4) {
          int r[4];
          group_rows(tws.x, tws.y, r);
          tensor_scatter4(&maps.f, r[0], r[1], r[2], r[3],
                          st + (size_t)4 * lane * St::SEG * sizeof(T));
        }
#pragma unroll
        for (int k = 0; k < 2; ++k) {
          const Job& jb = jobs[k];
          if (jb.kind == 1 && !jb.gathered) {
            unsigned char* row = const_cast<unsigned char*>(job_row(jb, tws.x, tws.y));
            bulk_store(row + ((size_t)tws.zt * kTmaTile + jb.so) * jb.es, st + jb.sdst,
                       jb.sbytes);
          }
        }
      }
      bulk_commit();
      bulk_wait_read();
      __syncwarp();
      tws.next();
    };
    bool ok = true;
    int produced = 0;
    TileWalker tw;
    tw.init(blockIdx.x, gridDim.x, a.ny, tiles_per_row);
    for (int j = 0; j < count && ok; ++j, tw.next()) {
      const int s = j % S;
      if (j >= S) ok = mbar_wait(empty + s, (unsigned)(((j / S) - 1) & 1), a.spin_limit);
      if (!__all_sync(0xffffffffu, ok)) break;
      if (j >= S) store_stage(s);
      const int x = tw.x, y = tw.y, z0 = tw.zt * kTmaTile;
      unsigned char* st = stage_ptr(s);
      if (lane == 0) mbar_expect_tx(full + s, expect);
      __syncwarp();
      const bool by_map = !EVEN && maps.use;
      if (by_map && lane == 0) {
        // All slots of the tile's cells in one box per array (the row's first cell is a
        // multiple of 256, so the inner coordinate is 16-byte aligned).
        const int cell0 = (int)((long long)x * plane + (long long)y * a.nz + z0);
        tensor_copy_2d(st, &maps.f, cell0, 0, full + s);
        if constexpr (NT == 1) tensor_copy_2d(st + St::off_trc, &maps.g, cell0, 0, full + s);
      }
      if (by_rows && lane < NG4) {
        int r[4];
        group_rows(x, y, r);
        tensor_gather4(st + (size_t)4 * lane * St::SEG * sizeof(T), &maps.f, r[0], r[1], r[2],
                       r[3], full + s);
      }
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const Job& jb = jobs[k];
        if (jb.kind == 1 && !by_map && !jb.gathered) {
          copy_row_segment(st + jb.dst, job_row(jb, x, y), z0, jb.hl, jb.hr, a.nz, jb.es,
                           full + s);
        } else if (jb.kind == 2) {
          const long long first = (long long)x * plane + (long long)y * a.nz + z0;
          bulk_copy(st + jb.dst, jb.base + (size_t)first * jb.es, (unsigned)(kTmaTile * jb.es),
                    full + s);
        }
      }
      produced = j + 1;
    }
    // The last tiles' results (bounded waits for the consumers), then every store complete.
    if (ok) {
      for (int j = produced - S > 0 ? produced - S : 0; j < produced && ok; ++j) {
        ok = __all_sync(0xffffffffu, mbar_wait(empty + j % S, (unsigned)((j / S) & 1), a.spin_limit));
        if (ok) store_stage(j % S);
      }
    }
    bulk_wait_all();
    if (!ok && lane == 0) atomicOr(a.status, 2);
    // Leave only once the copies of the last stages have landed (bounded), so that no copy
    // writes into shared memory after the CTA is gone.
    if (lane == 0)
      for (int j = produced - S > 0 ? produced - S : 0; j < produced; ++j)
        mbar_wait(full + j % S, (unsigned)((j / S) & 1));
    return;
  }

  if constexpr (PAIR) {
    // ---- consumer warps, two cells a thread: cells z0 + col and z0 + col + T/2 of every tile.
    constexpr int HALF = kTmaTile / 2;
    constexpr int QT = NT == 1 ? TL::Q : 1;
    TileWalker tw;
    tw.init(blockIdx.x, gridDim.x, a.ny, tiles_per_row);
    for (int j = 0; j < count; ++j, tw.next()) {
      const int s = j % S;
      const bool ok =
        __all_sync(0xffffffffu, mbar_wait(full + s, (unsigned)((j / S) & 1), a.spin_limit));
      if (!ok) {
        if (lane == 0) atomicOr(a.status, 2);
        break;
      }
      const int x = tw.x, y = tw.y, z0 = tw.zt * kTmaTile;
      unsigned char* st = stage_ptr(s);
      const int col = tid;  // this thread's columns: col and col + T/2
      float2 fv[Q];
#pragma unroll
      for (int i = 0; i < Q; ++i) {
        const T* seg =
            reinterpret_cast<const T*>(st + (size_t)(EVEN ? i : opp(i)) * St::SEG * sizeof(T));
        const int cz = comp<L>(i, 2);
        const T va = seg[stage_pos<whole_row, EVEN>(St::H, col, cz)];
        const T vb = seg[stage_pos<whole_row, EVEN>(St::H, col + HALF, cz)];
        fv[i] = make_float2(P::load_dev(&va, 0.0f), P::load_dev(&vb, 0.0f));
      }
      float2 gv[QT];
      if constexpr (NT == 1) {
#pragma unroll
        for (int i = 0; i < St::NG; ++i) {
          const TT* seg = reinterpret_cast<const TT*>(
              st + St::off_trc + (size_t)(EVEN ? i : opp(i)) * St::SEGG * sizeof(TT));
          const int cz = comp<TL>(i, 2);
          gv[i] = make_float2(TP::load(seg + stage_pos<whole_row, EVEN>(St::HG, col, cz), 0.0f),
                              TP::load(seg + stage_pos<whole_row, EVEN>(St::HG, col + HALF, cz),
                                       0.0f));
        }
      }
      const float2 cval =
          a.acc_mode == kAccBoussinesq
              ? make_float2(reinterpret_cast<const Real*>(st + St::off_val)[col],
                            reinterpret_cast<const Real*>(st + St::off_val)[col + HALF])
              : make_float2(0.0f, 0.0f);
      const int flagA = st[St::off_flag + col], flagB = st[St::off_flag + col + HALF];
      const CellPos cA = make_cellpos(a, x, y, z0 + col, false);
      const CellPos cB = make_cellpos(a, x, y, z0 + col + HALF, false);
      // fv / gv hold the results afterwards (walls: untouched)
      update_cell2<L, TRT, K, EVEN, NT, KT>(a, PairSink<St, kTmaTile>{st, col}, cA, cB, flagA,
                                            flagB, fv, gv, cval);
      fence_proxy_async();  // this thread's stage writes, visible to the bulk stores
      __syncwarp();
      if (lane == 0) mbar_arrive(empty + s);
      if constexpr (EVEN && !whole_row) {
        // Cell A can only be at the tile's left end, cell B only at its right end.
        constexpr int HE = St::H > St::HG ? St::H : St::HG;
        const bool ea = col < HE && !(flagA & 1), eb = col + HALF >= kTmaTile - HE && !(flagB & 1);
        if (ea || eb) {
          const int ec = ea ? col : col + HALF;
          const CellPos e = make_cellpos(a, x, y, z0 + ec, true);
          edge_stores<St, L, P, TP, NT>(
              a, e, ec, [&](int i) { return ea ? fv[i].x : fv[i].y; },
              [&](int i) { return ea ? gv[i].x : gv[i].y; });
        }
      }
    }
    return;
  }

  // ---- consumer warps: thread tid owns cell z0 + col of every tile.
  TileWalker tw;
  tw.init(blockIdx.x, gridDim.x, a.ny, tiles_per_row);
  for (int j = 0; j < count; ++j, tw.next()) {
    const int s = j % S;
    const bool ok =
        __all_sync(0xffffffffu, mbar_wait(full + s, (unsigned)((j / S) & 1), a.spin_limit));
    if (!ok) {
      if (lane == 0) atomicOr(a.status, 2);
      break;  // the producer's own waits are bounded too
    }
    const int x = tw.x, y = tw.y, z0 = tw.zt * kTmaTile;
    unsigned char* st = stage_ptr(s);
    const int col = tid;  // this thread's column
    Real fv[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const T* seg =
          reinterpret_cast<const T*>(st + (size_t)(EVEN ? i : opp(i)) * St::SEG * sizeof(T));
      const T v = seg[stage_pos<whole_row, EVEN>(St::H, col, comp<L>(i, 2))];
      if constexpr (dev_in<K>())
        fv[i] = P::load_dev(&v, weight<L, Real>(i));
      else
        fv[i] = P::load(&v, weight<L, Real>(i));
    }
    Real g[NT == 1 ? TL::Q : 1];
    if constexpr (NT == 1) {
#pragma unroll
      for (int i = 0; i < St::NG; ++i) {
        const TT* seg = reinterpret_cast<const TT*>(
            st + St::off_trc + (size_t)(EVEN ? i : opp(i)) * St::SEGG * sizeof(TT));
        g[i] = TP::load(seg + stage_pos<whole_row, EVEN>(St::HG, col, comp<TL>(i, 2)), 0.0f);
      }
    }
    const Real cval = a.acc_mode == kAccBoussinesq
                          ? reinterpret_cast<const Real*>(st + St::off_val)[col]
                          : Real(0);
    const int flag = st[St::off_flag + col];
    const CellPos c = make_cellpos(a, x, y, z0 + col, false);
    // Results into the stage, where the producer picks them up as row segments (fv / g hold
    // them afterwards; walls: untouched).
    const StageSink<St, L, TL> sink{st, col};
    update_cell<L, TRT, K, EVEN, NT, StageSink<St, L, TL>, KT>(a, c, flag, fv, g, cval, a.om_pos,
                                                              a.om_neg, sink);
    fence_proxy_async();  // this thread's stage writes, visible to the bulk stores
    __syncwarp();
    if (lane == 0) mbar_arrive(empty + s);
    if constexpr (EVEN && !whole_row) {
      constexpr int HE = St::H > St::HG ? St::H : St::HG;
      if ((col < HE || col >= kTmaTile - HE) && !(flag & 1)) {
        const CellPos e = make_cellpos(a, x, y, z0 + col, true);
        edge_stores<St, L, P, TP, NT>(
            a, e, col, [&](int i) { return fv[i]; }, [&](int i) { return g[i]; });
      }
    }
  }
}

}  // namespace lbm
