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
// bank conflicts), collide, and store straight to HBM with coalesced stores.
//
// In-flight data is bounded by shared memory, not by registers, and the copy engine issues one
// instruction per row segment instead of one per element. Odd steps, which read their own row of
// every slot, take all slots of an array in one tensor-map copy (cp.async.bulk.tensor, a box of
// 256 cells by Q slots) when the launcher provides the maps.
//
// Synchronisation: a producer warp fills stage s once every consumer warp has arrived on the
// stage's `empty` barrier; consumers wait on its `full` barrier (expected bytes), read their
// operands into registers, arrive on `empty`, then compute and store. There is no CTA-wide
// barrier in the loop. Every wait is bounded: on timeout the kernel sets bit 1 (value 2) of the
// status word and leaves.
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

// Bounded wait for the phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
  const unsigned addr = smem_u32(bar);
  for (unsigned i = 0; i < kSpinLimit; ++i) {
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
  CUtensorMap f;  // populations, box {256, Q}
  CUtensorMap g;  // fused tracer populations, box {256, Qt}
  int use;        // 1 when both maps are valid for this launch
};

__device__ __forceinline__ void tensor_copy_2d(void* dst, const CUtensorMap* map, int c0, int c1,
                                               uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, "
      "{%2, %3}], [%4];\n" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
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

// Named barrier 1 over the 256 consumer threads (the producer warp never takes part).
__device__ __forceinline__ void consumers_sync() {
  asm volatile("bar.sync 1, 256;\n" ::: "memory");
}
// The same barrier, returning whether `ok` held in every consumer thread.
__device__ __forceinline__ bool consumers_all(bool ok) {
  unsigned r;
  asm volatile(
      "{\n .reg .pred q, p;\n setp.ne.u32 q, %1, 0;\n bar.red.and.pred p, 1, 256, q;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(r)
      : "r"(ok ? 1u : 0u)
      : "memory");
  return r != 0;
}

// Shared-memory layout of one stage, in elements of each operand's type.
template <class L, int K, int NT, bool EVEN>
struct TmaStage {
  using T = typename Pop<K>::type;
  using Real = typename Pop<K>::real;
  using TL = typename TracerLattice<L::D>::type;
  static constexpr int Q = L::Q;
  static constexpr int NG = NT == 1 ? TL::Q : 0;
  static constexpr int H = EVEN ? 16 / (int)sizeof(T) : 0;       // population halo
  static constexpr int HG = EVEN ? 16 / (int)sizeof(Real) : 0;   // tracer halo
  static constexpr int SEG = kTmaTile + 2 * H;                   // populations per direction
  static constexpr int SEGG = kTmaTile + 2 * HG;
  static constexpr size_t pop_bytes = (size_t)Q * SEG * sizeof(T);
  static constexpr size_t trc_bytes = (size_t)NG * SEGG * sizeof(Real);
  static constexpr size_t val_bytes = (size_t)kTmaTile * sizeof(Real);
  static constexpr size_t flag_bytes = kTmaTile;
  // offsets (bytes) inside a stage; every part 16-byte aligned
  static constexpr size_t off_trc = pop_bytes;
  static constexpr size_t off_val = off_trc + trc_bytes;
  static constexpr size_t off_flag = off_val + val_bytes;
  static constexpr size_t bytes = off_flag + flag_bytes;
};

template <class L, int K, int NT, bool EVEN, int S>
__host__ __device__ constexpr size_t tma_smem_bytes() {
  return (size_t)S * TmaStage<L, K, NT, EVEN>::bytes + 16 * S;  // + full/empty mbarriers
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

// update_cell's output into the stage it read from: slot i of the thread's cell on odd steps
// (position i, column tid), slot i of the upstream cell on even steps of whole rows (the very
// position the thread read, shifted and wrapped). A tile's slots then leave as whole row segments.
template <class St, class L, class TL>
struct StageSink {
  unsigned char* st;
  int tid;
  template <class LL, class P, bool EVEN, bool DEV>
  __device__ __forceinline__ void fluid(typename P::type*, long long, const CellPos&,
                                        const typename P::real (&v)[LL::Q]) const {
    using T = typename P::type;
    using Real = typename P::real;
    T* base = reinterpret_cast<T*>(st);
#pragma unroll
    for (int i = 0; i < LL::Q; ++i) {
      T* p = base + i * St::SEG +
             (EVEN ? St::H + ((tid - comp<LL>(i, 2)) & (kTmaTile - 1)) : tid);
      const Real val = EVEN ? v[opp(i)] : v[i];
      if constexpr (DEV)
        P::store_dev(p, val, weight<LL, Real>(i));
      else
        P::store(p, val, weight<LL, Real>(i));
    }
  }
  template <class TT, class TP, bool EVEN>
  __device__ __forceinline__ void tracer(typename TP::type*, long long, const CellPos&,
                                         const typename TP::real (&v)[TT::Q]) const {
    using Real = typename TP::real;
    Real* base = reinterpret_cast<Real*>(st + St::off_trc);
#pragma unroll
    for (int i = 0; i < TT::Q; ++i) {
      Real* p = base + i * St::SEGG +
                (EVEN ? St::HG + ((tid - comp<TT>(i, 2)) & (kTmaTile - 1)) : tid);
      *p = EVEN ? v[opp(i)] : v[i];
    }
  }
};

constexpr int kConsumerWarps = kTmaTile / 32;
constexpr int kTmaThreads = kTmaTile + 32;  // + one producer warp

// Warp-specialised: warps 0..7 consume (one cell per thread), warp 8 produces. Stage s has a
// `full` barrier (one arrival: the producer's expect_tx, plus the copies' bytes) and an `empty`
// barrier (one arrival per consumer warp once it has its operands in registers).
template <class L, bool TRT, int K, bool EVEN, int NT, int S>
__global__ void __launch_bounds__(kTmaThreads)
    aa_tma_kernel(const __grid_constant__ StepArgs<typename Pop<K>::real> a,
                  const __grid_constant__ TmaMaps maps) {
  using P = Pop<K>;
  using Real = typename P::real;
  using T = typename P::type;
  using TL = typename TracerLattice<L::D>::type;
  using St = TmaStage<L, K, NT, EVEN>;
  constexpr int Q = L::Q;
  constexpr int NOPS = Q + St::NG + 2;  // copy jobs per tile: populations, tracer, value, flags

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

  // Odd steps write their populations back through the stage (bulk stores of the tile's own row
  // segments, one arrival on `empty` once they have read it); even steps store from registers
  // and release the stage warp by warp as soon as the operands are read. (Bulk stores on even
  // steps of one-tile rows were correct but measured 15% slower with FP16 populations: the stage
  // stays busy through the collision, and the ring runs dry.)
  const bool bulk_out = !EVEN;
  if (tid == 0) {
    for (int s = 0; s < S; ++s) {
      mbar_init(full + s, 1);
      mbar_init(empty + s, bulk_out ? 1 : kConsumerWarps);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();

  if (warp == kConsumerWarps) {
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
    };
    const bool whole_row = a.nz == kTmaTile;
    Job jobs[2];
    unsigned lane_bytes = 0;
#pragma unroll
    for (int k = 0; k < 2; ++k) {
      const int op = lane + 32 * k;
      Job jb{nullptr, 0, 0, 0, 0, 1, 0u, 0};
      if (op < Q) {
        const int slot = op;  // stage position op holds slot op (odd steps read opp(i) from it)
        const int cz = EVEN && !whole_row ? comp<L>(op, 2) : 0;
        jb.base = reinterpret_cast<const unsigned char*>(static_cast<const T*>(a.f) +
                                                         (size_t)slot * a.n);
        jb.cx = EVEN ? comp<L>(op, 0) : 0;
        jb.cy = EVEN ? comp<L>(op, 1) : 0;
        jb.hl = cz > 0 ? St::H : 0;
        jb.hr = cz < 0 ? St::H : 0;
        jb.es = sizeof(T);
        jb.dst = (unsigned)(((size_t)op * St::SEG + St::H - jb.hl) * sizeof(T));
        jb.kind = 1;
      } else if (op < Q + St::NG) {
        if constexpr (NT == 1) {
          const int i = op - Q;
          const int slot = i;
          const int cz = EVEN && !whole_row ? comp<TL>(i, 2) : 0;
          jb.base = reinterpret_cast<const unsigned char*>(a.tr[0].g + (size_t)slot * a.n);
          jb.cx = EVEN ? comp<TL>(i, 0) : 0;
          jb.cy = EVEN ? comp<TL>(i, 1) : 0;
          jb.hl = cz > 0 ? St::HG : 0;
          jb.hr = cz < 0 ? St::HG : 0;
          jb.es = sizeof(Real);
          jb.dst = (unsigned)(St::off_trc + ((size_t)i * St::SEGG + St::HG - jb.hl) * sizeof(Real));
          jb.kind = 1;
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
      if (jb.kind != 0) lane_bytes += (unsigned)((kTmaTile + jb.hl + jb.hr) * jb.es);
    }
    const unsigned expect = __reduce_add_sync(0xffffffffu, lane_bytes);
    const long long plane = (long long)a.ny * a.nz;
    bool ok = true;
    int produced = 0;
    TileWalker tw;
    tw.init(blockIdx.x, gridDim.x, a.ny, tiles_per_row);
    for (int j = 0; j < count && ok; ++j, tw.next()) {
      const int s = j % S;
      if (j >= S) ok = mbar_wait(empty + s, (unsigned)(((j / S) - 1) & 1));
      if (!__all_sync(0xffffffffu, ok)) break;
      const int x = tw.x, y = tw.y, z0 = tw.zt * kTmaTile;
      unsigned char* st = stage_ptr(s);
      const int xm = x == 0 ? a.nx - 1 : x - 1, xp = x == a.nx - 1 ? 0 : x + 1;
      const int ym = y == 0 ? a.ny - 1 : y - 1, yp = y == a.ny - 1 ? 0 : y + 1;
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
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const Job& jb = jobs[k];
        if (jb.kind == 1 && !by_map) {
          const int ux = jb.cx > 0 ? xm : (jb.cx < 0 ? xp : x);
          const int uy = jb.cy > 0 ? ym : (jb.cy < 0 ? yp : y);
          const unsigned char* row = jb.base + (size_t)(ux * plane + (long long)uy * a.nz) * jb.es;
          copy_row_segment(st + jb.dst, row, z0, jb.hl, jb.hr, a.nz, jb.es, full + s);
        } else if (jb.kind == 2) {
          const long long first = (long long)x * plane + (long long)y * a.nz + z0;
          bulk_copy(st + jb.dst, jb.base + (size_t)first * jb.es, (unsigned)(kTmaTile * jb.es),
                    full + s);
        }
      }
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

  // ---- consumer warps: thread tid owns cell z0 + tid of every tile.
  const bool whole_row = a.nz == kTmaTile;
  TileWalker tw;
  tw.init(blockIdx.x, gridDim.x, a.ny, tiles_per_row);
  for (int j = 0; j < count; ++j, tw.next()) {
    const int s = j % S;
    bool ok = mbar_wait(full + s, (unsigned)((j / S) & 1));
    if (bulk_out) ok = consumers_all(ok);  // the consumers stay in step: they share barrier 1
    if (!ok) {
      atomicOr(a.status, 2);
      break;  // the producer's own waits are bounded too
    }
    const int x = tw.x, y = tw.y, z0 = tw.zt * kTmaTile;
    const unsigned char* st = stage_ptr(s);
    Real fv[Q];
#pragma unroll
    for (int i = 0; i < Q; ++i) {
      const T* seg =
          reinterpret_cast<const T*>(st + (size_t)(EVEN ? i : opp(i)) * St::SEG * sizeof(T));
      const int zi = whole_row ? (tid - comp<L>(i, 2)) & (kTmaTile - 1) : tid - comp<L>(i, 2);
      const T v = EVEN ? seg[St::H + zi] : seg[tid];
      if constexpr (dev_in<K>())
        fv[i] = P::load_dev(&v, weight<L, Real>(i));
      else
        fv[i] = P::load(&v, weight<L, Real>(i));
    }
    Real g[NT == 1 ? TL::Q : 1];
    if constexpr (NT == 1) {
#pragma unroll
      for (int i = 0; i < St::NG; ++i) {
        const Real* seg = reinterpret_cast<const Real*>(
            st + St::off_trc + (size_t)(EVEN ? i : opp(i)) * St::SEGG * sizeof(Real));
        const int zi = whole_row ? (tid - comp<TL>(i, 2)) & (kTmaTile - 1) : tid - comp<TL>(i, 2);
        g[i] = EVEN ? seg[St::HG + zi] : seg[tid];
      }
    }
    const Real cval = a.acc_mode == kAccBoussinesq
                          ? reinterpret_cast<const Real*>(st + St::off_val)[tid]
                          : Real(0);
    const int flag = st[St::off_flag + tid];
    const CellPos c = make_cellpos(a, x, y, z0 + tid, EVEN && !bulk_out);
    if (!bulk_out) {
      __syncwarp();
      if (lane == 0) mbar_arrive(empty + s);  // this warp is done with stage s
      update_cell<L, TRT, K, EVEN, NT>(a, c, flag, fv, g, cval, a.om_pos, a.om_neg);
      continue;
    }
    const StageSink<St, L, TL> sink{const_cast<unsigned char*>(st), tid};
    update_cell<L, TRT, K, EVEN, NT>(a, c, flag, fv, g, cval, a.om_pos, a.om_neg, sink);
    fence_proxy_async();  // this thread's stage writes, visible to the bulk stores
    consumers_sync();
    if (warp == 0) {
      // Lane k stores slot k (and k + 32): the tile's row segment of the thread's own row (odd
      // steps) or the whole upstream row (even steps of one-tile rows).
      const long long plane = (long long)a.ny * a.nz;
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const int op = lane + 32 * k;
        if (op < Q) {
          const int ux = EVEN ? (x - comp<L>(op, 0) + a.nx) % a.nx : x;
          const int uy = EVEN ? (y - comp<L>(op, 1) + a.ny) % a.ny : y;
          T* dst = static_cast<T*>(a.f) + (size_t)op * a.n + (size_t)(ux * plane) +
                   (size_t)uy * a.nz + z0;
          bulk_store(dst, st + ((size_t)op * St::SEG + St::H) * sizeof(T),
                     (unsigned)(kTmaTile * sizeof(T)));
        } else if (op < Q + St::NG) {
          if constexpr (NT == 1) {
            const int i = op - Q;
            const int ux = EVEN ? (x - comp<TL>(i, 0) + a.nx) % a.nx : x;
            const int uy = EVEN ? (y - comp<TL>(i, 1) + a.ny) % a.ny : y;
            Real* dst = a.tr[0].g + (size_t)i * a.n + (size_t)(ux * plane) + (size_t)uy * a.nz + z0;
            bulk_store(dst, st + St::off_trc + ((size_t)i * St::SEGG + St::HG) * sizeof(Real),
                       (unsigned)(kTmaTile * sizeof(Real)));
          }
        }
      }
      bulk_commit();
      bulk_wait_read();
      __syncwarp();
      if (lane == 0) mbar_arrive(empty + s);  // the stage's contents have been read out
    }
  }
  if (bulk_out && warp == 0) bulk_wait_all();  // the tile stores are complete before exit
}

}  // namespace lbm
