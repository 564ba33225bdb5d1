// Pipelined variant of the AA step for 4- and 8-byte populations (F32, F64).
//
// The direct kernel (aa_step_kernel) keeps every in-flight load in a register, so the bytes in
// flight per SM are capped by the register file and the kernel is latency-bound (measured: 44%
// of DRAM peak for the D2Q9 TRT + tracer odd step). Here each thread walks down a column of
// rows -- the same z, rows r = blockIdx.y + k * gridDim.y -- and prefetches the operands of the
// next S-1 cells of its column into shared memory with per-thread asynchronous copies
// (cp.async, 4 or 8 bytes each), while it updates the current one. In-flight data then lives in
// shared memory (S stages x operands x threads), not in registers.
//
// No barrier is needed: a thread reads back only the stage slots its own copies filled, after
// cp.async.wait_group has retired them, and overwrites a stage only after its own previous
// update consumed it. Access patterns, and therefore the AA race-freedom argument, are those of
// the direct kernel: every population slot is read and written by exactly one thread per step.
#pragma once

#include "aa_step.cuh"

namespace lbm {

__device__ __forceinline__ unsigned shared_address(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(shared_address(smem)),
               "l"(gmem), "n"(BYTES)
               : "memory");
}

__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Operand slots per stage: Q populations, the fused tracer's populations, the coupled tracer
// value and the 4-byte word holding the cell's flag byte.
template <class L, int NT>
__host__ __device__ constexpr int pipe_slots() {
  return L::Q + (NT == 1 ? TracerLattice<L::D>::type::Q : 0) + 2;
}

template <class L, int K, int NT, int S>
__host__ __device__ constexpr size_t pipe_smem_bytes(int threads) {
  return (size_t)S * pipe_slots<L, NT>() * threads * sizeof(typename Pop<K>::type);
}

template <class L, bool TRT, int K, bool EVEN, int NT, int S>
__global__ void __launch_bounds__(256)
    aa_pipe_kernel(const __grid_constant__ StepArgs<typename Pop<K>::real> a) {
  using P = Pop<K>;
  using Real = typename P::real;
  using T = typename P::type;
  using TL = typename TracerLattice<L::D>::type;
  static_assert(sizeof(T) == sizeof(Real) && (sizeof(T) == 4 || sizeof(T) == 8),
                "the pipelined kernel copies whole 4- or 8-byte populations");
  constexpr int Q = L::Q;
  constexpr int NG = NT == 1 ? TL::Q : 0;
  constexpr int NS = pipe_slots<L, NT>();
  constexpr int W = sizeof(T);

  extern __shared__ __align__(16) unsigned char smem[];
  const int B = blockDim.x, tid = threadIdx.x;
  auto slot = [&](int stage, int j) -> unsigned char* {
    return smem + ((size_t)(stage * NS + j) * B + tid) * W;
  };

  const int z = blockIdx.x * B + tid;
  const bool active = z < a.nz;
  const int nrows = a.nx * a.ny;
  const int cnt = (int)blockIdx.y < nrows ? (nrows - 1 - (int)blockIdx.y) / (int)gridDim.y + 1 : 0;
  const T* f = static_cast<const T*>(a.f);

  auto position = [&](int k) {
    const int r = blockIdx.y + k * gridDim.y;
    const int x = r / a.ny;
    return make_cellpos(a, x, r - x * a.ny, z, EVEN);
  };

  // Enqueue the copies of the k-th cell of this thread's column into stage `stage`; always
  // commits a group (empty past the end) so the wait counts stay uniform.
  auto issue = [&](int k, int stage) {
    if (active && k < cnt) {
      const CellPos c = position(k);
#pragma unroll
      for (int i = 0; i < Q; ++i)
        cp_async<W>(slot(stage, i), EVEN ? f + (long long)i * a.n + c.upstream<L>(i)
                                         : f + (long long)opp(i) * a.n + c.cell);
      if constexpr (NT == 1) {
        const Real* g = a.tr[0].g;
#pragma unroll
        for (int i = 0; i < NG; ++i)
          cp_async<W>(slot(stage, Q + i), EVEN ? g + (long long)i * a.n + c.upstream<TL>(i)
                                               : g + (long long)opp(i) * a.n + c.cell);
      }
      if (a.acc_mode == kAccBoussinesq) cp_async<W>(slot(stage, Q + NG), a.coupled_val + c.cell);
      cp_async<4>(slot(stage, Q + NG + 1), a.flags + (c.cell & ~3LL));
    }
    cp_async_commit();
  };

#pragma unroll
  for (int s = 0; s < S - 1; ++s) issue(s, s);

#pragma unroll 1
  for (int k = 0; k < cnt; ++k) {
    const int stage = k % S;
    issue(k + S - 1, (k + S - 1) % S);
    cp_async_wait<S - 1>();
    if (active) {
      const CellPos c = position(k);
      Real fv[Q];
#pragma unroll
      for (int i = 0; i < Q; ++i) fv[i] = *reinterpret_cast<const T*>(slot(stage, i));
      Real g[NT == 1 ? TL::Q : 1];
      if constexpr (NT == 1) {
#pragma unroll
        for (int i = 0; i < NG; ++i) g[i] = *reinterpret_cast<const Real*>(slot(stage, Q + i));
      }
      const Real cval =
          a.acc_mode == kAccBoussinesq ? *reinterpret_cast<const Real*>(slot(stage, Q + NG)) : 0;
      const unsigned word = *reinterpret_cast<const unsigned*>(slot(stage, Q + NG + 1));
      const int flag = (int)((word >> (8 * (unsigned)(c.cell & 3))) & 0xFFu);
      update_cell<L, TRT, K, EVEN, NT>(a, c, flag, fv, g, cval);
    }
  }
  cp_async_wait<0>();
}

}  // namespace lbm
