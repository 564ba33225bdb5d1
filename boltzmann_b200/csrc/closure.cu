// Learned subgrid closure (3-layer CNN on the coarse lattice) and on-device post-processing.
//
// No counterpart in the reference. The network: 3x3 convolutions 4 -> 32 -> 32 -> 1 with GELU
// (tanh form) after the first two layers, zero padding at the domain edges, channels-last
// activations.
//
//   layer   forward                       backward
//   1 (4->32)   CUDA cores (36 MAC/out)    weights: CUDA cores; no input gradient
//   2 (32->32)  tcgen05 BF16, FP32 acc     data: tcgen05 (transposed conv, fused GELU');
//               (TMEM accumulators)        weights: mma.sync (cells are the reduction axis)
//               mma.sync kept selectable (lbm_closure_set_layer2_kernel)
//   3 (32->1)   CUDA cores                 data + weights: CUDA cores (fused GELU')
//
// Every product sum takes BF16 operands (weights, activations, pre-activation gradients rounded
// to nearest even) and accumulates in FP32. Reductions over cells run per tile in a fixed order
// into per-CTA partial rows, which one kernel adds row by row: results are deterministic.
//
// Cell tiles are 4 rows (x) by 64 columns (y, the contiguous axis). Shared-memory tiles keep 40
// BF16 per cell (80 bytes): eight consecutive cells then start in eight different 16-byte bank
// groups, so ldmatrix reads them without conflicts. Weight rows (one per output channel) are
// padded from 288 to 296 BF16 (592 bytes) for the same reason.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>

#include "../../include/lbm_closure.h"
#include "sim.h"

namespace {

using bf16 = __nv_bfloat16;

constexpr int C = LBM_CLOSURE_CHANNELS;
constexpr int kTX = 4, kTY = 64;             // cell tile
constexpr int kHX = kTX + 2, kHY = kTY + 2;  // tile plus a one-cell halo
constexpr int kCS = 40;                      // shared-memory BF16 per cell (32 used)
constexpr int kWS = 296;                     // shared-memory BF16 per weight row (288 used)
constexpr int kPartialRows = 296;            // CTAs of the reducing kernels (2 per SM)
constexpr int kLossBlocks = 296;

int fail(int code, const std::string& msg) {
  lbm::set_last_error(msg);
  return code;
}

#define CL_CUDA(call)                                                    \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess)                                               \
      return fail(LBM_ERR_CUDA, std::string("CUDA error in " #call ": ") + \
                                    cudaGetErrorString(e_));             \
  } while (0)

struct Grid {
  int64_t nx, ny, batch;
  int64_t tx, ty;   // tiles along x and y
  int64_t tiles;    // all tiles of the batch
  __host__ __device__ void tile(int64_t t, int64_t& b, int64_t& x0, int64_t& y0) const {
    const int64_t per = tx * ty;
    b = t / per;
    const int64_t r = t - b * per;
    x0 = (r / ty) * kTX;
    y0 = (r % ty) * kTY;
  }
  __host__ __device__ int64_t cell(int64_t b, int64_t x, int64_t y) const {
    return (b * nx + x) * ny + y;
  }
};

Grid make_grid(int64_t nx, int64_t ny, int64_t batch) {
  Grid g{nx, ny, batch, (nx + kTX - 1) / kTX, (ny + kTY - 1) / kTY, 0};
  g.tiles = g.tx * g.ty * batch;
  return g;
}

// ---------------------------------------------------------------------------------------------
// Scalar helpers

// GELU in its tanh form, 0.5 z (1 + tanh(sqrt(2/pi) (z + 0.044715 z^3))), written as
// z sigmoid(v) with v = z (a + b z^2), a = 2 sqrt(2/pi), b = 0.089430 sqrt(2/pi) (since
// 1 + tanh(u) = 2 sigmoid(2u)); evaluated with the fast exponential and division intrinsics
// (about 1e-6 relative, below the BF16 rounding every activation then takes). For v -> -inf the
// quotient goes to 0, as GELU does.
constexpr float kGeluA = 1.5957691216057308f;   // 2 sqrt(2/pi)
constexpr float kGeluB = 0.07135481627159709f;  // 2 sqrt(2/pi) 0.044715
__device__ __forceinline__ float gelu(float z) {
  const float v = z * fmaf(kGeluB, z * z, kGeluA);
  return __fdividef(z, 1.0f + __expf(-v));
}

// d/dz [z sigmoid(v(z))] = s (1 + z (1 - s) v'(z)), s = sigmoid(v), v' = a + 3 b z^2.
__device__ __forceinline__ float gelu_grad(float z) {
  const float z2 = z * z;
  const float v = z * fmaf(kGeluB, z2, kGeluA);
  const float sg = __fdividef(1.0f, 1.0f + __expf(-v));
  return sg * fmaf(z * (1.0f - sg), fmaf(3.0f * kGeluB, z2, kGeluA), 1.0f);
}

__device__ __forceinline__ float bf(bf16 v) { return __bfloat162float(v); }
__device__ __forceinline__ bf16 to_bf(float v) { return __float2bfloat16_rn(v); }

__device__ __forceinline__ bool fluid_cell(int32_t flag) { return (flag & 7) == 0; }

// np.gradient along one axis (unit spacing, first-order edges): f[i+1]-f[i-1] halved inside,
// f[1]-f[0] and f[n-1]-f[n-2] at the ends.
__device__ __forceinline__ float np_gradient(float lo, float mid, float hi, int64_t i, int64_t n) {
  if (i == 0) return __fsub_rn(hi, mid);
  if (i == n - 1) return __fsub_rn(mid, lo);
  return __fmul_rn(__fsub_rn(hi, lo), 0.5f);
}

// ---------------------------------------------------------------------------------------------
// Tensor-core helpers (sm_80+ warp-level BF16 MMA, FP32 accumulate).

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const bf16* p) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}

__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const bf16* p) {
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(a));
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// ---------------------------------------------------------------------------------------------
// Shared-memory tile loads (zero outside the domain).

// ROWS x COLS cells of a 32-channel BF16 field starting at (xs, ys), into dst[cell][kCS].
template <int ROWS, int COLS>
__device__ __forceinline__ void load_cells32(const bf16* __restrict__ src, const Grid& g,
                                             int64_t b, int64_t xs, int64_t ys, bf16* dst) {
  for (int i = threadIdx.x; i < ROWS * COLS * 4; i += blockDim.x) {
    const int chunk = i & 3, cell = i >> 2;
    const int r = cell / COLS, c = cell - r * COLS;
    const int64_t x = xs + r, y = ys + c;
    uint4 v = make_uint4(0, 0, 0, 0);
    if (x >= 0 && x < g.nx && y >= 0 && y < g.ny)
      v = __ldg(reinterpret_cast<const uint4*>(src + g.cell(b, x, y) * C) + chunk);
    *reinterpret_cast<uint4*>(dst + cell * kCS + chunk * 8) = v;
  }
}

// The 4-channel input features with the halo, into dst[cell][4].
__device__ __forceinline__ void load_cells4(const bf16* __restrict__ src, const Grid& g, int64_t b,
                                            int64_t x0, int64_t y0, bf16* dst) {
  for (int i = threadIdx.x; i < kHX * kHY; i += blockDim.x) {
    const int r = i / kHY, c = i - r * kHY;
    const int64_t x = x0 - 1 + r, y = y0 - 1 + c;
    uint2 v = make_uint2(0, 0);
    if (x >= 0 && x < g.nx && y >= 0 && y < g.ny)
      v = __ldg(reinterpret_cast<const uint2*>(src + g.cell(b, x, y) * 4));
    *reinterpret_cast<uint2*>(dst + i * 4) = v;
  }
}

// Layer-2 weights [32 out][288] into rows of kWS.
__device__ __forceinline__ void load_w2(const bf16* __restrict__ w2, bf16* ws) {
  for (int i = threadIdx.x; i < C * 36; i += blockDim.x) {
    const int co = i / 36, ch = i - co * 36;
    *reinterpret_cast<uint4*>(ws + co * kWS + ch * 8) =
        __ldg(reinterpret_cast<const uint4*>(w2 + co * 288) + ch);
  }
}

// ---------------------------------------------------------------------------------------------
// Post-processing and features

__global__ void curl2d_kernel(const float* __restrict__ vel, int64_t nx, int64_t ny,
                              float* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nx * ny) return;
  const int64_t x = i / ny, y = i - x * ny;
  const int64_t xm = x > 0 ? x - 1 : x, xp = x < nx - 1 ? x + 1 : x;
  const int64_t ym = y > 0 ? y - 1 : y, yp = y < ny - 1 ? y + 1 : y;
  const float dux_dy = np_gradient(vel[(x * ny + ym) * 2], vel[i * 2], vel[(x * ny + yp) * 2], y, ny);
  const float duy_dx =
      np_gradient(vel[(xm * ny + y) * 2 + 1], vel[i * 2 + 1], vel[(xp * ny + y) * 2 + 1], x, nx);
  out[i] = __fsub_rn(dux_dy, duy_dx);
}

__global__ void curl3d_kernel(const float* __restrict__ vel, int64_t nx, int64_t ny, int64_t nz,
                              float* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nx * ny * nz) return;
  const int64_t x = i / (ny * nz), y = (i / nz) % ny, z = i % nz;
  const int64_t pos[3] = {x, y, z}, len[3] = {nx, ny, nz}, stride[3] = {ny * nz, nz, 1};
  float d[3][3];  // d[axis][component]
  for (int a = 0; a < 3; ++a) {
    const int64_t lo = pos[a] > 0 ? i - stride[a] : i;
    const int64_t hi = pos[a] < len[a] - 1 ? i + stride[a] : i;
    for (int c = 0; c < 3; ++c)
      d[a][c] = np_gradient(vel[lo * 3 + c], vel[i * 3 + c], vel[hi * 3 + c], pos[a], len[a]);
  }
  out[i * 3 + 0] = __fsub_rn(d[2][1], d[1][2]);
  out[i * 3 + 1] = __fsub_rn(d[0][2], d[2][0]);
  out[i * 3 + 2] = __fsub_rn(d[1][0], d[0][1]);
}

__global__ void vmag_kernel(const float* __restrict__ vel, int64_t n, int dim,
                            float* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = __fmul_rn(vel[i * dim], vel[i * dim]);
  for (int c = 1; c < dim; ++c) s = __fadd_rn(s, __fmul_rn(vel[i * dim + c], vel[i * dim + c]));
  out[i] = sqrtf(s);
}

struct Norm {
  float mean[4], inv_std[4];
};

// Velocity read for the closure's curl: walls count as the no-slip value 0.
__device__ __forceinline__ float vel_or_wall(const float* vel, const int32_t* flags, int64_t b,
                                             int64_t n, int64_t cell, int c) {
  return (flags[cell] & 1) ? 0.0f : vel[(b * n + cell) * 2 + c];
}

// The four BF16 features of cell (x, y) of batch entry b, packed in two words (0 on walls).
__device__ __forceinline__ uint2 cell_features(const float* __restrict__ rho,
                                               const float* __restrict__ vel,
                                               const int32_t* __restrict__ flags, int64_t nx,
                                               int64_t ny, int64_t b, int64_t x, int64_t y,
                                               const Norm& norm) {
  const int64_t n = nx * ny;
  const int64_t cell = x * ny + y, i = b * n + cell;
  uint2 packed = make_uint2(0, 0);
  if (!(flags[cell] & 1)) {
    const int64_t xm = x > 0 ? x - 1 : x, xp = x < nx - 1 ? x + 1 : x;
    const int64_t ym = y > 0 ? y - 1 : y, yp = y < ny - 1 ? y + 1 : y;
    const float dux_dy =
        np_gradient(vel_or_wall(vel, flags, b, n, x * ny + ym, 0), vel[i * 2],
                    vel_or_wall(vel, flags, b, n, x * ny + yp, 0), y, ny);
    const float duy_dx =
        np_gradient(vel_or_wall(vel, flags, b, n, xm * ny + y, 1), vel[i * 2 + 1],
                    vel_or_wall(vel, flags, b, n, xp * ny + y, 1), x, nx);
    const float v[4] = {__fsub_rn(rho[i], 1.0f), vel[i * 2], vel[i * 2 + 1],
                        __fsub_rn(dux_dy, duy_dx)};
    bf16 h[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) h[c] = to_bf(__fmul_rn(__fsub_rn(v[c], norm.mean[c]), norm.inv_std[c]));
    packed.x = (uint32_t)__bfloat16_as_ushort(h[0]) | ((uint32_t)__bfloat16_as_ushort(h[1]) << 16);
    packed.y = (uint32_t)__bfloat16_as_ushort(h[2]) | ((uint32_t)__bfloat16_as_ushort(h[3]) << 16);
  }
  return packed;
}

__global__ void features_kernel(const float* __restrict__ rho, const float* __restrict__ vel,
                                const int32_t* __restrict__ flags, int64_t nx, int64_t ny,
                                int64_t batch, Norm norm, bf16* __restrict__ x_out) {
  const int64_t n = nx * ny;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n * batch) return;
  const int64_t b = i / n, cell = i - b * n;
  const int64_t x = cell / ny, y = cell - x * ny;
  reinterpret_cast<uint2*>(x_out)[i] = cell_features(rho, vel, flags, nx, ny, b, x, y, norm);
}

// ---------------------------------------------------------------------------------------------
// Layer 1 forward (CUDA cores): 36 MACs per output.

__global__ void __launch_bounds__(256)
    conv1_fwd_kernel(Grid g, const bf16* __restrict__ x, const bf16* __restrict__ w1,
                     const float* __restrict__ b1, float* __restrict__ z1, bf16* __restrict__ a1) {
  __shared__ __align__(16) bf16 xs[kHX * kHY * 4];
  __shared__ __align__(16) float ws[9 * 4 * C];  // [tap][ci][co]
  for (int i = threadIdx.x; i < 9 * 4 * C; i += blockDim.x) {
    const int co = i / 36, r = i - co * 36;  // w1 is [co][tap][ci]
    ws[r * C + co] = bf(w1[i]);
  }
  const int ti = threadIdx.x / kTY, tj = threadIdx.x % kTY;
  for (int64_t t = blockIdx.x; t < g.tiles; t += gridDim.x) {
    int64_t b, x0, y0;
    g.tile(t, b, x0, y0);
    __syncthreads();
    load_cells4(x, g, b, x0, y0, xs);
    __syncthreads();
    const int64_t xx = x0 + ti, yy = y0 + tj;
    if (xx >= g.nx || yy >= g.ny) continue;
    float acc[C];
#pragma unroll
    for (int co = 0; co < C; ++co) acc[co] = 0.0f;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int dx = tap / 3 - 1, dy = tap % 3 - 1;
      const bf16* xv = xs + ((ti + 1 + dx) * kHY + tj + 1 + dy) * 4;
#pragma unroll
      for (int ci = 0; ci < 4; ++ci) {
        const float v = bf(xv[ci]);
        const float4* wr = reinterpret_cast<const float4*>(ws + (tap * 4 + ci) * C);
#pragma unroll
        for (int q = 0; q < C / 4; ++q) {
          const float4 w = wr[q];
          acc[4 * q + 0] = fmaf(v, w.x, acc[4 * q + 0]);
          acc[4 * q + 1] = fmaf(v, w.y, acc[4 * q + 1]);
          acc[4 * q + 2] = fmaf(v, w.z, acc[4 * q + 2]);
          acc[4 * q + 3] = fmaf(v, w.w, acc[4 * q + 3]);
        }
      }
    }
    const int64_t cell = g.cell(b, xx, yy);
    uint32_t packed[C / 2];
#pragma unroll
    for (int co = 0; co < C; co += 2) {
      const float za = acc[co] + b1[co], zb = acc[co + 1] + b1[co + 1];
      acc[co] = za;
      acc[co + 1] = zb;
      packed[co / 2] = (uint32_t)__bfloat16_as_ushort(to_bf(gelu(za))) |
                       ((uint32_t)__bfloat16_as_ushort(to_bf(gelu(zb))) << 16);
    }
    if (z1 != nullptr) {
      float4* zp = reinterpret_cast<float4*>(z1 + cell * C);
#pragma unroll
      for (int q = 0; q < C / 4; ++q)
        zp[q] = make_float4(acc[4 * q], acc[4 * q + 1], acc[4 * q + 2], acc[4 * q + 3]);
    }
    uint4* ap = reinterpret_cast<uint4*>(a1 + cell * C);
#pragma unroll
    for (int q = 0; q < C / 8; ++q)
      ap[q] = make_uint4(packed[4 * q], packed[4 * q + 1], packed[4 * q + 2], packed[4 * q + 3]);
  }
}

// ---------------------------------------------------------------------------------------------
// Layer 2 on tensor cores: forward conv (BWD = false) or the transposed conv of the backward
// pass (BWD = true), as an implicit GEMM per tile: M = 64 cells of one row per warp (4 m-tiles
// of 16), N = 32 channels (4 n-tiles of 8), K = 9 taps x 32 channels (18 k-steps of 16).
//
// Forward:  z[p][co] = b[co] + sum_{tap,ci} W[co][tap][ci] a[p + tap][ci];  a2 = GELU(z) (BF16)
// Backward: d[q][ci] = sum_{tap,co} W[co][tap][ci] dz[q - tap][co];  dz1 = d GELU'(z1) (BF16),
//           plus the per-channel sums of dz1 (the layer-1 bias gradient) into partial rows.

constexpr int kConv32Threads = 128;
constexpr size_t kConv32Smem = (size_t)(kHX * kHY * kCS + C * kWS) * sizeof(bf16);

template <bool BWD>
__global__ void __launch_bounds__(kConv32Threads)
    conv32_kernel(Grid g, const bf16* __restrict__ in, const bf16* __restrict__ w2,
                  const float* __restrict__ bias, const float* __restrict__ zin,
                  float* __restrict__ zout, bf16* __restrict__ out, float* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  bf16* ins = reinterpret_cast<bf16*>(smem_raw);
  bf16* wsm = ins + kHX * kHY * kCS;
  __shared__ float colsum[kConv32Threads / 32][C];

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3;
  load_w2(w2, wsm);

  float bias_sum[4][2];  // BWD: this thread's running sums of dz1 for channels nt*8 + 2tq (+1)
#pragma unroll
  for (int nt = 0; nt < 4; ++nt) bias_sum[nt][0] = bias_sum[nt][1] = 0.0f;

  for (int64_t t = blockIdx.x; t < g.tiles; t += gridDim.x) {
    int64_t b, x0, y0;
    g.tile(t, b, x0, y0);
    __syncthreads();
    load_cells32<kHX, kHY>(in, g, b, x0 - 1, y0 - 1, ins);
    __syncthreads();

    float acc[4][4][4];
#pragma unroll
    for (int mt = 0; mt < 4; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[mt][nt][e] = 0.0f;

    const int mi = lane >> 3, rr = lane & 7;
#pragma unroll 1
    for (int tap = 0; tap < 9; ++tap) {
      const int dx = tap / 3 - 1, dy = tap % 3 - 1;
      const int sx = BWD ? -dx : dx, sy = BWD ? -dy : dy;
#pragma unroll
      for (int kc = 0; kc < 2; ++kc) {
        uint32_t bfrag[4][2];
#pragma unroll
        for (int np = 0; np < 2; ++np) {
          uint32_t r[4];
          if (!BWD) {
            const int co = (2 * np + (mi >> 1)) * 8 + rr;
            ldsm_x4(r, wsm + co * kWS + tap * 32 + kc * 16 + (mi & 1) * 8);
          } else {
            const int co = kc * 16 + (mi & 1) * 8 + rr;
            ldsm_x4_t(r, wsm + co * kWS + tap * 32 + (2 * np + (mi >> 1)) * 8);
          }
          bfrag[2 * np][0] = r[0];
          bfrag[2 * np][1] = r[1];
          bfrag[2 * np + 1][0] = r[2];
          bfrag[2 * np + 1][1] = r[3];
        }
        const int row = warp + 1 + sx;
        const int j = (lane & 7) + 8 * ((lane >> 3) & 1);
        const int koff = kc * 16 + 8 * (lane >> 4);
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
          uint32_t a[4];
          ldsm_x4(a, ins + (row * kHY + mt * 16 + j + 1 + sy) * kCS + koff);
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) mma_bf16(acc[mt][nt], a, bfrag[nt][0], bfrag[nt][1]);
        }
      }
    }

    // Epilogue: thread holds cells (gq, gq + 8) of each m-tile, channels nt*8 + 2tq (+1).
    const int64_t xx = x0 + warp;
#pragma unroll
    for (int mt = 0; mt < 4; ++mt) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int64_t yy = y0 + mt * 16 + gq + 8 * h;
        if (xx >= g.nx || yy >= g.ny) continue;
        const int64_t cell = g.cell(b, xx, yy);
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const int ch = nt * 8 + 2 * tq;
          const float v0 = acc[mt][nt][2 * h], v1 = acc[mt][nt][2 * h + 1];
          __nv_bfloat162 o;
          if (!BWD) {
            const float z0 = v0 + bias[ch], z1v = v1 + bias[ch + 1];
            if (zout != nullptr)
              *reinterpret_cast<float2*>(zout + cell * C + ch) = make_float2(z0, z1v);
            o.x = to_bf(gelu(z0));
            o.y = to_bf(gelu(z1v));
          } else {
            const float2 z = *reinterpret_cast<const float2*>(zin + cell * C + ch);
            o.x = to_bf(v0 * gelu_grad(z.x));
            o.y = to_bf(v1 * gelu_grad(z.y));
            bias_sum[nt][0] += bf(o.x);
            bias_sum[nt][1] += bf(o.y);
          }
          *reinterpret_cast<__nv_bfloat162*>(out + cell * C + ch) = o;
        }
      }
    }
  }

  if (BWD) {
    // Sum over the 8 lanes sharing tq, then over warps, in a fixed order.
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        float s = bias_sum[nt][e];
        s += __shfl_xor_sync(0xffffffffu, s, 4);
        s += __shfl_xor_sync(0xffffffffu, s, 8);
        s += __shfl_xor_sync(0xffffffffu, s, 16);
        if (gq == 0) colsum[warp][nt * 8 + 2 * tq + e] = s;
      }
    __syncthreads();
    if (threadIdx.x < C) {
      float s = 0.0f;
      for (int w = 0; w < kConv32Threads / 32; ++w) s += colsum[w][threadIdx.x];
      partial[(int64_t)blockIdx.x * LBM_CLOSURE_PARAMS + LBM_CLOSURE_OFF_B1 + threadIdx.x] = s;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Layer-2 weight gradient on tensor cores: dW[co][tap][ci] = sum_p dz[p][co] a1[p + tap][ci].
// One warp per tap: M = 32 output channels (2 m-tiles), N = 32 input channels (4 n-tiles),
// K = the cells of the CTA's tiles, 16 per k-step.

constexpr int kDw2Threads = 9 * 32;
constexpr size_t kDw2Smem = (size_t)(kTX * kTY * kCS + kHX * kHY * kCS) * sizeof(bf16);

__global__ void __launch_bounds__(kDw2Threads)
    conv32_wgrad_kernel(Grid g, const bf16* __restrict__ a1, const bf16* __restrict__ dz2,
                        float* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  bf16* dzs = reinterpret_cast<bf16*>(smem_raw);  // [kTX * kTY][kCS]
  bf16* as = dzs + kTX * kTY * kCS;               // [kHX * kHY][kCS]
  const int tap = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int dx = tap / 3 - 1, dy = tap % 3 - 1;
  const int mi = lane >> 3, rr = lane & 7;

  float acc[2][4][4];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[mt][nt][e] = 0.0f;

  for (int64_t t = blockIdx.x; t < g.tiles; t += gridDim.x) {
    int64_t b, x0, y0;
    g.tile(t, b, x0, y0);
    __syncthreads();
    load_cells32<kTX, kTY>(dz2, g, b, x0, y0, dzs);
    load_cells32<kHX, kHY>(a1, g, b, x0 - 1, y0 - 1, as);
    __syncthreads();
#pragma unroll 1
    for (int i = 0; i < kTX; ++i) {
#pragma unroll
      for (int c = 0; c < kTY / 16; ++c) {
        uint32_t afrag[2][4];
#pragma unroll
        for (int mt = 0; mt < 2; ++mt) {
          const int p = i * kTY + c * 16 + (mi >> 1) * 8 + rr;
          ldsm_x4_t(afrag[mt], dzs + p * kCS + mt * 16 + (mi & 1) * 8);
        }
        uint32_t bfrag[4][2];
#pragma unroll
        for (int np = 0; np < 2; ++np) {
          uint32_t r[4];
          const int col = c * 16 + (mi & 1) * 8 + rr;
          ldsm_x4_t(r, as + ((i + 1 + dx) * kHY + col + 1 + dy) * kCS + (2 * np + (mi >> 1)) * 8);
          bfrag[2 * np][0] = r[0];
          bfrag[2 * np][1] = r[1];
          bfrag[2 * np + 1][0] = r[2];
          bfrag[2 * np + 1][1] = r[3];
        }
#pragma unroll
        for (int mt = 0; mt < 2; ++mt)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) mma_bf16(acc[mt][nt], afrag[mt], bfrag[nt][0], bfrag[nt][1]);
      }
    }
  }

  float* row = partial + (int64_t)blockIdx.x * LBM_CLOSURE_PARAMS + LBM_CLOSURE_OFF_W2;
  const int gq = lane >> 2, tq = lane & 3;
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int co = mt * 16 + gq + 8 * h, ci = nt * 8 + 2 * tq;
        row[co * 288 + tap * 32 + ci] = acc[mt][nt][2 * h];
        row[co * 288 + tap * 32 + ci + 1] = acc[mt][nt][2 * h + 1];
      }
}

// ---------------------------------------------------------------------------------------------
// Layer 3 (32 -> 1) forward, CUDA cores: y[p] = b3 + sum_{tap,ci} w3[tap][ci] a2[p + tap][ci].

constexpr size_t kConv3Smem = (size_t)kHX * kHY * kCS * sizeof(bf16);

__global__ void __launch_bounds__(256)
    conv3_fwd_kernel(Grid g, const bf16* __restrict__ a2, const bf16* __restrict__ w3,
                     const float* __restrict__ b3, float* __restrict__ y) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  bf16* as = reinterpret_cast<bf16*>(smem_raw);
  __shared__ float ws[9 * C];
  for (int i = threadIdx.x; i < 9 * C; i += blockDim.x) ws[i] = bf(w3[i]);
  const int ti = threadIdx.x / kTY, tj = threadIdx.x % kTY;
  for (int64_t t = blockIdx.x; t < g.tiles; t += gridDim.x) {
    int64_t b, x0, y0;
    g.tile(t, b, x0, y0);
    __syncthreads();
    load_cells32<kHX, kHY>(a2, g, b, x0 - 1, y0 - 1, as);
    __syncthreads();
    const int64_t xx = x0 + ti, yy = y0 + tj;
    if (xx >= g.nx || yy >= g.ny) continue;
    float acc = 0.0f;
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
      const int dx = tap / 3 - 1, dy = tap % 3 - 1;
      const bf16* av = as + ((ti + 1 + dx) * kHY + tj + 1 + dy) * kCS;
#pragma unroll
      for (int q = 0; q < C / 8; ++q) {
        const uint4 v = *reinterpret_cast<const uint4*>(av + q * 8);
        const uint32_t w4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const float lo = __uint_as_float(w4[e] << 16), hi = __uint_as_float(w4[e] & 0xffff0000u);
          acc = fmaf(lo, ws[tap * C + q * 8 + 2 * e], acc);
          acc = fmaf(hi, ws[tap * C + q * 8 + 2 * e + 1], acc);
        }
      }
    }
    y[g.cell(b, xx, yy)] = acc + b3[0];
  }
}

// ---------------------------------------------------------------------------------------------
// Layer 3 backward, CUDA cores. Per tile:
//   dz2[q][ci] = BF16( GELU'(z2[q][ci]) sum_tap w3[tap][ci] dy[q - tap] )
//   dW3[tap][ci] += sum_p a2[p + tap][ci] dy[p],  db3 += sum_p dy[p],  db2[ci] += sum_q dz2[q][ci]

constexpr size_t kConv3BwdSmem =
    (size_t)kHX * kHY * kCS * sizeof(bf16) + (size_t)kTX * kTY * (C + 1) * sizeof(float);

__global__ void __launch_bounds__(256)
    conv3_bwd_kernel(Grid g, const bf16* __restrict__ a2, const float* __restrict__ z2,
                     const bf16* __restrict__ w3, const float* __restrict__ dy,
                     bf16* __restrict__ dz2, float* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  bf16* as = reinterpret_cast<bf16*>(smem_raw);                           // [kHX*kHY][kCS]
  float* dzs = reinterpret_cast<float*>(smem_raw + kHX * kHY * kCS * 2);  // [256][C + 1]
  __shared__ float ws[9 * C];
  __shared__ float dys[kHX * kHY];
  for (int i = threadIdx.x; i < 9 * C; i += blockDim.x) ws[i] = bf(w3[i]);
  const int ti = threadIdx.x / kTY, tj = threadIdx.x % kTY;
  float wacc[2] = {0.0f, 0.0f};  // outputs k = threadIdx.x and threadIdx.x + 256 of [dW3, db3]
  float bsum = 0.0f;             // threads < 32: db2[threadIdx.x]

  for (int64_t t = blockIdx.x; t < g.tiles; t += gridDim.x) {
    int64_t b, x0, y0;
    g.tile(t, b, x0, y0);
    __syncthreads();
    load_cells32<kHX, kHY>(a2, g, b, x0 - 1, y0 - 1, as);
    for (int i = threadIdx.x; i < kHX * kHY; i += blockDim.x) {
      const int r = i / kHY, c = i - r * kHY;
      const int64_t x = x0 - 1 + r, yv = y0 - 1 + c;
      dys[i] = (x >= 0 && x < g.nx && yv >= 0 && yv < g.ny) ? dy[g.cell(b, x, yv)] : 0.0f;
    }
    __syncthreads();

    const int64_t xx = x0 + ti, yy = y0 + tj;
    float* drow = dzs + threadIdx.x * (C + 1);
    if (xx < g.nx && yy < g.ny) {
      const int64_t cell = g.cell(b, xx, yy);
      float d[C];
#pragma unroll
      for (int ci = 0; ci < C; ++ci) d[ci] = 0.0f;
#pragma unroll
      for (int tap = 0; tap < 9; ++tap) {
        const int dx = tap / 3 - 1, dyy = tap % 3 - 1;
        const float v = dys[(ti + 1 - dx) * kHY + tj + 1 - dyy];
#pragma unroll
        for (int ci = 0; ci < C; ++ci) d[ci] = fmaf(ws[tap * C + ci], v, d[ci]);
      }
      uint32_t packed[C / 2];
#pragma unroll
      for (int ci = 0; ci < C; ci += 4) {
        const float4 z = *reinterpret_cast<const float4*>(z2 + cell * C + ci);
        const bf16 h0 = to_bf(d[ci] * gelu_grad(z.x)), h1 = to_bf(d[ci + 1] * gelu_grad(z.y));
        const bf16 h2 = to_bf(d[ci + 2] * gelu_grad(z.z)), h3 = to_bf(d[ci + 3] * gelu_grad(z.w));
        drow[ci] = bf(h0);
        drow[ci + 1] = bf(h1);
        drow[ci + 2] = bf(h2);
        drow[ci + 3] = bf(h3);
        packed[ci / 2] = (uint32_t)__bfloat16_as_ushort(h0) | ((uint32_t)__bfloat16_as_ushort(h1) << 16);
        packed[ci / 2 + 1] =
            (uint32_t)__bfloat16_as_ushort(h2) | ((uint32_t)__bfloat16_as_ushort(h3) << 16);
      }
      uint4* op = reinterpret_cast<uint4*>(dz2 + cell * C);
#pragma unroll
      for (int q = 0; q < C / 8; ++q)
        op[q] = make_uint4(packed[4 * q], packed[4 * q + 1], packed[4 * q + 2], packed[4 * q + 3]);
    } else {
#pragma unroll
      for (int ci = 0; ci < C; ++ci) drow[ci] = 0.0f;
    }
    __syncthreads();

    // Weight and bias sums over the tile's cells, each output owned by one thread.
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int k = threadIdx.x + 256 * e;
      if (k > 9 * C) continue;
      float s = 0.0f;
      if (k == 9 * C) {
        for (int p = 0; p < kTX * kTY; ++p) s += dys[(p / kTY + 1) * kHY + p % kTY + 1];
      } else {
        const int tap = k / C, ci = k % C;
        const int dx = tap / 3 - 1, dyy = tap % 3 - 1;
        for (int p = 0; p < kTX * kTY; ++p) {
          const int pi = p / kTY, pj = p % kTY;
          s = fmaf(bf(as[((pi + 1 + dx) * kHY + pj + 1 + dyy) * kCS + ci]),
                   dys[(pi + 1) * kHY + pj + 1], s);
        }
      }
      wacc[e] += s;
    }
    if (threadIdx.x < C) {
      float s = 0.0f;
      for (int p = 0; p < kTX * kTY; ++p) s += dzs[p * (C + 1) + threadIdx.x];
      bsum += s;
    }
  }

  float* row = partial + (int64_t)blockIdx.x * LBM_CLOSURE_PARAMS;
#pragma unroll
  for (int e = 0; e < 2; ++e) {
    const int k = threadIdx.x + 256 * e;
    if (k <= 9 * C) row[LBM_CLOSURE_OFF_W3 + k] = wacc[e];  // k == 288 is b3
  }
  if (threadIdx.x < C) row[LBM_CLOSURE_OFF_B2 + threadIdx.x] = bsum;
}

// ---------------------------------------------------------------------------------------------
// Layer-1 weight gradient, CUDA cores: dW1[co][tap][ci] = sum_p dz1[p][co] x[p + tap][ci].
// Thread (co, tap) owns the 4 input channels.

__global__ void __launch_bounds__(288)
    conv1_wgrad_kernel(Grid g, const bf16* __restrict__ x, const bf16* __restrict__ dz1,
                       float* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  bf16* dzs = reinterpret_cast<bf16*>(smem_raw);  // [kTX * kTY][kCS]
  __shared__ __align__(16) bf16 xs[kHX * kHY * 4];
  const int co = threadIdx.x / 9, tap = threadIdx.x % 9;
  const int dx = tap / 3 - 1, dy = tap % 3 - 1;
  float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  for (int64_t t = blockIdx.x; t < g.tiles; t += gridDim.x) {
    int64_t b, x0, y0;
    g.tile(t, b, x0, y0);
    __syncthreads();
    load_cells32<kTX, kTY>(dz1, g, b, x0, y0, dzs);
    load_cells4(x, g, b, x0, y0, xs);
    __syncthreads();
    for (int p = 0; p < kTX * kTY; ++p) {
      const int pi = p / kTY, pj = p % kTY;
      const float d = bf(dzs[p * kCS + co]);
      const uint2 v = *reinterpret_cast<const uint2*>(xs + ((pi + 1 + dx) * kHY + pj + 1 + dy) * 4);
      acc[0] = fmaf(d, __uint_as_float(v.x << 16), acc[0]);
      acc[1] = fmaf(d, __uint_as_float(v.x & 0xffff0000u), acc[1]);
      acc[2] = fmaf(d, __uint_as_float(v.y << 16), acc[2]);
      acc[3] = fmaf(d, __uint_as_float(v.y & 0xffff0000u), acc[3]);
    }
  }
  float* row = partial + (int64_t)blockIdx.x * LBM_CLOSURE_PARAMS + LBM_CLOSURE_OFF_W1;
#pragma unroll
  for (int ci = 0; ci < 4; ++ci) row[co * 36 + tap * 4 + ci] = acc[ci];
}

// Column sums of the partial rows, in row order (double accumulation).
__global__ void reduce_rows_kernel(const float* __restrict__ partial, int rows,
                                   float* __restrict__ out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= LBM_CLOSURE_PARAMS) return;
  double s = 0.0;
  for (int r = 0; r < rows; ++r) s += partial[(int64_t)r * LBM_CLOSURE_PARAMS + j];
  out[j] = (float)s;
}

// ---------------------------------------------------------------------------------------------
// Loss

__global__ void count_kernel(const int32_t* __restrict__ flags, int64_t n,
                             unsigned long long* __restrict__ count) {
  __shared__ unsigned long long s[32];
  unsigned long long c = 0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) c += fluid_cell(flags[i]) ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[w];
    *count = t;
  }
}

__global__ void loss_kernel(const float* __restrict__ y, const float* __restrict__ target,
                            const int32_t* __restrict__ flags, int64_t n, int64_t batch,
                            const unsigned long long* __restrict__ count, float* __restrict__ dy,
                            double* __restrict__ partial) {
  __shared__ double s[32];
  const double total = (double)(*count) * (double)batch;
  const float scale = total > 0 ? (float)(2.0 / total) : 0.0f;
  double acc = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n * batch;
       i += (int64_t)gridDim.x * blockDim.x) {
    const bool m = fluid_cell(flags[i % n]);
    const float d = y[i] - target[i];
    dy[i] = m ? scale * d : 0.0f;
    if (m) acc += (double)d * (double)d;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s[w];
    partial[blockIdx.x] = t;
  }
}

__global__ void loss_final_kernel(const double* __restrict__ partial, int blocks,
                                  const unsigned long long* __restrict__ count, int64_t batch,
                                  double* __restrict__ loss) {
  double t = 0.0;
  for (int i = 0; i < blocks; ++i) t += partial[i];
  const double total = (double)(*count) * (double)batch;
  *loss = total > 0 ? t / total : 0.0;
}

// ---------------------------------------------------------------------------------------------
// Blackwell tensor cores (tcgen05): MMAs issued by one thread on shared-memory operands,
// accumulators in tensor memory (TMEM), completion signalled through an mbarrier.

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, K-major without swizzle: rows (M or N) 16 bytes apart inside a
// group of 8 rows, `sbo` bytes between groups of 8 rows, `lbo` bytes between the two 8-element K
// halves of one MMA. Descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t umma_desc(unsigned start, unsigned lbo, unsigned sbo) {
  return (uint64_t)((start >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: BF16 A and B, FP32 accumulator, both K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                          uint32_t idesc, bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate ? 1u : 0u), "r"(0u), "r"(0u), "r"(0u),
      "r"(0u));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_addr(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
      "%12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, "
      "%30, %31}, [%32];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
        "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
        "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

constexpr unsigned kClosureSpinLimit = 1u << 22;

__device__ __forceinline__ void cl_mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

// Polls of the fused kernel's wait for its tensor-core products before it gives up
// (lbm_closure_set_spin_limit); the wait that drains MMAs still in flight keeps the default.
__device__ unsigned g_closure_spin_limit = kClosureSpinLimit;

// Bounded wait for the phase with the given parity; false after `limit` polls.
__device__ __forceinline__ bool cl_mbar_wait(uint64_t* bar, unsigned parity,
                                             unsigned limit = kClosureSpinLimit) {
  const unsigned addr = smem_addr(bar);
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

// Set (bit 0) when a closure kernel gave up waiting for its tensor-core work; read and cleared
// by lbm_closure_status.
__device__ int g_closure_status;

// ---------------------------------------------------------------------------------------------
// Inference in one pass: features, the three layers and the relaxation field for a tile of
// kFR x kFC output cells, every intermediate in shared memory (~213 KB, one CTA of 16 warps per
// SM). The raw fields of the tile's neighbourhood are staged first with coalesced loads. Each
// layer is evaluated on its own halo-extended region -- layer 3 reads layer 2 one cell around
// the tile, layer 2 reads layer 1 two cells around, layer 1 reads the features three cells
// around -- and outside the domain every layer's output is 0, the zero padding the
// layer-by-layer kernels apply. All three layers run on tensor cores (mma.sync BF16 -> FP32):
// layer 1 with K = 48 (9 taps x 4 channels, zero-padded from 36), layer 2 with K = 288, layer 3
// with K = 288 and N = 8 (one real output column). A warp's
// 16-row MMA tile is any 16 consecutive cells of a region in row-major order (ldmatrix takes one
// row address per lane), so the regions need not be multiples of 16 wide.

constexpr int kFR = 14, kFC = 64;               // output tile
constexpr int kA2R = kFR + 2, kA2C = kFC + 2;  // layer-2 region
constexpr int kA1R = kFR + 4, kA1C = kFC + 4;  // layer-1 region
constexpr int kXR = kFR + 6, kXC = kFC + 6;    // feature region
constexpr int kRawR = kFR + 8, kRawC = kFC + 8;  // raw fields (features read one cell around)
constexpr int kW1S = 56;                        // shared-memory BF16 per layer-1 weight row
constexpr int kFusedThreads = 512;
// Layer 1's output is stored "chunk-major" for the tensor-core descriptors: plane k (channels
// 8k .. 8k+7) holds 16 bytes per cell, cells in row-major order of the layer-1 region
// (kA1R x kA1C), padded so that every shifted 128-cell block stays inside the plane.
constexpr int kA1Pad = 1296;                    // >= 69 + 9 * 128 + 69 cells
constexpr int kL2Blocks = 9;                    // 128-cell blocks covering the layer-2 region
constexpr int kL2First = kA1C + 1;              // layer-1 flat index of layer-2 cell (0, 0)
constexpr size_t kFusedOffA1 = (size_t)kXR * kXC * 8;
constexpr size_t kFusedOffA2 = kFusedOffA1 + (size_t)4 * kA1Pad * 16;
constexpr size_t kFusedOffW1 = kFusedOffA2 + (size_t)kA2R * kA2C * kCS * 2;
constexpr size_t kFusedOffW2 = kFusedOffW1 + (size_t)C * kW1S * 2;
constexpr size_t kFusedOffW3 = kFusedOffW2 + (size_t)36 * C * 16;  // 36 K-chunks x 32 rows x 16 B
constexpr size_t kFusedOffB = kFusedOffW3 + (size_t)9 * C * 4;
constexpr size_t kFusedOffBar = kFusedOffB + (size_t)2 * C * 4;    // mbarrier + TMEM address
constexpr size_t kFusedSmem = kFusedOffBar + 16;
static_assert(kL2First + kL2Blocks * 128 + kA1C + 1 <= kA1Pad, "layer-1 planes too short");
static_assert(kL2First + kL2Blocks * 128 > (kA2R * kA1C) + kA2C, "blocks do not cover layer 2");
constexpr int kTmemCols = 512;  // 9 accumulators of 32 FP32 columns (power of two >= 288)
static_assert((size_t)kRawR * kRawC * 16 <= (size_t)kA2R * kA2C * kCS * 2,
              "the staged raw fields must fit in the layer-2 area");

struct FusedArgs {
  const float* params;
  const bf16* wb;
  const float* rho;
  const float* vel;
  const int32_t* flags;
  int64_t nx, ny;
  Norm norm;
  float tau0, gain, max_dtau;
  float* omega;
  int tiles_x, tiles_y;
};

__global__ void __launch_bounds__(kFusedThreads, 1)
    closure_fused_kernel(const __grid_constant__ FusedArgs f) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint32_t* xs = reinterpret_cast<uint32_t*>(smem_raw);  // [cell][2 words]: channels 0-1, 2-3
  unsigned char* a1c = smem_raw + kFusedOffA1;  // [4 planes][kA1Pad cells][16 B]
  bf16* a2s = reinterpret_cast<bf16*>(smem_raw + kFusedOffA2);
  bf16* w1s = reinterpret_cast<bf16*>(smem_raw + kFusedOffW1);
  unsigned char* w2c = smem_raw + kFusedOffW2;  // [36 K-chunks][32 out channels][16 B]
  bf16* w3b = reinterpret_cast<bf16*>(smem_raw + kFusedOffW3);  // [9][32]
  float* bs = reinterpret_cast<float*>(smem_raw + kFusedOffB);  // b1 [32], b2 [32]
  uint64_t* mma_done = reinterpret_cast<uint64_t*>(smem_raw + kFusedOffBar);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem_raw + kFusedOffBar + 8);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gq = lane >> 2, tq = lane & 3, mi = lane >> 3, rr = lane & 7;
  constexpr int kWarps = kFusedThreads / 32;

  for (int i = threadIdx.x; i < C * kW1S; i += blockDim.x) {
    const int co = i / kW1S, k = i - co * kW1S;
    w1s[i] = k < 36 ? f.wb[LBM_CLOSURE_OFF_W1 + co * 36 + k] : __float2bfloat16(0.0f);
  }
  // Layer-2 weights as the MMA's B operand: K-chunk kk (k = 8 kk .. 8 kk + 7, k = tap*32 + ci)
  // of output channel co at (kk * 32 + co) * 16 bytes.
  for (int i = threadIdx.x; i < 36 * C; i += blockDim.x) {
    const int kk = i / C, co = i - kk * C;
    *reinterpret_cast<uint4*>(w2c + (size_t)i * 16) =
        __ldg(reinterpret_cast<const uint4*>(f.wb + LBM_CLOSURE_OFF_W2 + co * 288 + kk * 8));
  }
  for (int i = threadIdx.x; i < 9 * C; i += blockDim.x) w3b[i] = f.wb[LBM_CLOSURE_OFF_W3 + i];
  for (int i = threadIdx.x; i < 2 * C; i += blockDim.x)
    bs[i] = f.params[i < C ? LBM_CLOSURE_OFF_B1 + i : LBM_CLOSURE_OFF_B2 + i - C];
  const float b3 = f.params[LBM_CLOSURE_OFF_B3];
  // Padding cells of the layer-1 planes feed only discarded rows; keep them finite.
  for (int i = threadIdx.x; i < 4 * kA1Pad; i += blockDim.x) {
    if (i % kA1Pad >= kA1R * kA1C)
      *reinterpret_cast<uint4*>(a1c + (size_t)i * 16) = make_uint4(0, 0, 0, 0);
  }
  if (threadIdx.x == 0) {
    cl_mbar_init(mma_done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = umma_idesc_bf16(128, 32);
  const unsigned a1c_addr = smem_addr(a1c), w2c_addr = smem_addr(w2c);
  bool healthy = true;
  const unsigned spin_limit = g_closure_spin_limit;
  // Layer-1 A fragments: element e of k-step kk holds input k = 16 kk + 2 tq + 8 (e >> 1), that
  // is tap k / 4 and the channel pair (k & 3) / 2 of the feature cell shifted by the tap. The
  // offset of that word from the cell's own (in 32-bit words of the feature region) depends on
  // the lane only; taps past 8 are the K padding (zero).
  int l1off[3][2];
  unsigned l1valid = 0;
#pragma unroll
  for (int kk = 0; kk < 3; ++kk)
#pragma unroll
    for (int hi = 0; hi < 2; ++hi) {
      const int k = kk * 16 + 2 * tq + 8 * hi, tap = k >> 2;
      l1off[kk][hi] = 2 * ((tap / 3 - 1) * kXC + tap % 3 - 1) + ((k & 3) >> 1);
      if (tap < 9) l1valid |= 1u << (2 * kk + hi);
    }
  unsigned phase = 0;

  const int ntiles = f.tiles_x * f.tiles_y;
  // Raw fields and features of tile t (the raw fields pass through the layer-2 area, which is
  // free from a tile's layer 3 until the next tile's epilogue), by warps 1 .. 15: warp 0 issues
  // the layer-2 MMAs meanwhile. Named barrier 1 orders the staging before the features.
  constexpr int kStageThreads = kFusedThreads - 32;
  auto stage_features = [&](int t) {
    if (warp == 0) return;
    const int st = threadIdx.x - 32;
    const int64_t x0 = (int64_t)(t / f.tiles_y) * kFR, y0 = (int64_t)(t % f.tiles_y) * kFC;
    // Raw fields on [x0 - 4, x0 + kFR + 4) x [y0 - 4, y0 + kFC + 4), staged with coalesced loads
    // into the layer-2 area; velocities on walls read as 0.
    float* raw_rho = reinterpret_cast<float*>(a2s);
    float2* raw_vel = reinterpret_cast<float2*>(raw_rho + kRawR * kRawC);
    int* raw_flag = reinterpret_cast<int*>(raw_vel + kRawR * kRawC);
    for (int i = st; i < kRawR * kRawC; i += kStageThreads) {
      const int r = i / kRawC, c = i - r * kRawC;
      const int64_t x = x0 - 4 + r, y = y0 - 4 + c;
      float rv = 0.0f;
      float2 vv = make_float2(0.0f, 0.0f);
      int fl = 0;
      if (x >= 0 && x < f.nx && y >= 0 && y < f.ny) {
        const int64_t cell = x * f.ny + y;
        rv = f.rho[cell];
        vv = *reinterpret_cast<const float2*>(f.vel + 2 * cell);
        fl = f.flags[cell];
      }
      raw_rho[i] = rv;
      raw_vel[i] = vv;
      raw_flag[i] = fl;
    }
    asm volatile("bar.sync 1, %0;" ::"r"(kStageThreads) : "memory");
    // Features on [x0 - 3, x0 + kFR + 3) x [y0 - 3, y0 + kFC + 3), the arithmetic of
    // cell_features (np.gradient edges, walls at rest, normalise, BF16) on the staged fields.
    for (int i = st; i < kXR * kXC; i += kStageThreads) {
      const int r = i / kXC, c = i - r * kXC;
      const int64_t x = x0 - 3 + r, y = y0 - 3 + c;
      uint2 packed = make_uint2(0, 0);
      const int ri = (r + 1) * kRawC + c + 1;  // this cell in the raw region
      if (x >= 0 && x < f.nx && y >= 0 && y < f.ny && !(raw_flag[ri] & 1)) {
        const int im = x > 0 ? ri - kRawC : ri, ip = x < f.nx - 1 ? ri + kRawC : ri;
        const int jm = y > 0 ? ri - 1 : ri, jp = y < f.ny - 1 ? ri + 1 : ri;
        auto vx = [&](int k) { return (raw_flag[k] & 1) ? 0.0f : raw_vel[k].x; };
        auto vy = [&](int k) { return (raw_flag[k] & 1) ? 0.0f : raw_vel[k].y; };
        const float dux_dy = np_gradient(vx(jm), raw_vel[ri].x, vx(jp), y, f.ny);
        const float duy_dx = np_gradient(vy(im), raw_vel[ri].y, vy(ip), x, f.nx);
        const float v[4] = {__fsub_rn(raw_rho[ri], 1.0f), raw_vel[ri].x, raw_vel[ri].y,
                            __fsub_rn(dux_dy, duy_dx)};
        bf16 h[4];
#pragma unroll
        for (int ch = 0; ch < 4; ++ch)
          h[ch] = to_bf(__fmul_rn(__fsub_rn(v[ch], f.norm.mean[ch]), f.norm.inv_std[ch]));
        packed.x = (uint32_t)__bfloat16_as_ushort(h[0]) | ((uint32_t)__bfloat16_as_ushort(h[1]) << 16);
        packed.y = (uint32_t)__bfloat16_as_ushort(h[2]) | ((uint32_t)__bfloat16_as_ushort(h[3]) << 16);
      }
      xs[2 * i] = packed.x;
      xs[2 * i + 1] = packed.y;
    }
  };
  // Tile t's layer-2 MMAs run while the CTA stages and featurises its next tile.
  if ((int)blockIdx.x < ntiles) stage_features(blockIdx.x);
  for (int t = blockIdx.x; t < ntiles && healthy; t += gridDim.x) {
    const int64_t x0 = (int64_t)(t / f.tiles_y) * kFR, y0 = (int64_t)(t % f.tiles_y) * kFC;
    tc_fence_before();
    __syncthreads();  // tile t's features are in place; the previous tile is done with a1c, a2s
                      // and every TMEM column
    tc_fence_after();

    // Layer 1 on [x0 - 2, ..) x [y0 - 2, ..): A fragments gathered from the features by tap.
    constexpr int n1 = kA1R * kA1C;
    for (int mt = warp; mt * 16 < n1; mt += kWarps) {
      int rq[2], cq[2], xw[2];  // xw: word index of the cell in the feature region
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int q = min(mt * 16 + gq + 8 * h, n1 - 1);
        rq[h] = q / kA1C;
        cq[h] = q - rq[h] * kA1C;
        xw[h] = 2 * ((rq[h] + 1) * kXC + cq[h] + 1);
      }
      float acc[4][4];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[nt][e] = 0.0f;
#pragma unroll
      for (int kk = 0; kk < 3; ++kk) {
        uint32_t a[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          const int h = e & 1, hi = e >> 1;
          a[e] = (l1valid >> (2 * kk + hi)) & 1u ? xs[xw[h] + l1off[kk][hi]] : 0u;
        }
        uint32_t bfr[4][2];
#pragma unroll
        for (int np = 0; np < 2; ++np) {
          uint32_t r4[4];
          ldsm_x4(r4, w1s + ((2 * np + (mi >> 1)) * 8 + rr) * kW1S + kk * 16 + (mi & 1) * 8);
          bfr[2 * np][0] = r4[0];
          bfr[2 * np][1] = r4[1];
          bfr[2 * np + 1][0] = r4[2];
          bfr[2 * np + 1][1] = r4[3];
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) mma_bf16(acc[nt], a, bfr[nt][0], bfr[nt][1]);
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int q = mt * 16 + gq + 8 * h;
        if (q >= n1) continue;
        const int64_t x = x0 - 2 + rq[h], y = y0 - 2 + cq[h];
        const bool inside = x >= 0 && x < f.nx && y >= 0 && y < f.ny;
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const int ch = nt * 8 + 2 * tq;
          __nv_bfloat162 o;
          o.x = to_bf(inside ? gelu(acc[nt][2 * h] + bs[ch]) : 0.0f);
          o.y = to_bf(inside ? gelu(acc[nt][2 * h + 1] + bs[ch + 1]) : 0.0f);
          *reinterpret_cast<__nv_bfloat162*>(a1c + ((size_t)nt * kA1Pad + q) * 16 + tq * 4) = o;
        }
      }
    }
    __syncthreads();

    // Layer 2 on tcgen05: nine blocks of 128 consecutive layer-1 cells (flat index from the
    // layer-1 cell of layer-2 cell (0, 0)), each an M = 128, N = 32, K = 288 product into its own
    // 32 TMEM columns. Tap (dx, dy) reads the block shifted by dx * kA1C + dy cells: with the
    // chunk-major planes that is an offset of the descriptor's start address (16 bytes a cell).
    // Rows that fall on the region's first or last column are computed and discarded.
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // layer 1 visible to the MMAs
    __syncthreads();
    if (threadIdx.x == 0) {
      tc_fence_after();
      // K-slice outer, block inner: consecutive MMAs accumulate into different TMEM columns.
#pragma unroll 1
      for (int tap = 0; tap < 9; ++tap) {
        const int off = (tap / 3 - 1) * kA1C + (tap % 3 - 1);
#pragma unroll
        for (int kc = 0; kc < 2; ++kc) {
          const int sidx = tap * 2 + kc;
          const uint64_t bdesc = umma_desc(w2c_addr + (unsigned)(sidx * 1024), C * 16, 128);
          const unsigned a_base = a1c_addr + (unsigned)((2 * kc * kA1Pad + kL2First + off) * 16);
#pragma unroll
          for (int m = 0; m < kL2Blocks; ++m)
            umma_bf16(tmem + (uint32_t)(m * 32),
                      umma_desc(a_base + (unsigned)(m * 128 * 16), kA1Pad * 16, 128), bdesc,
                      idesc, sidx != 0);
        }
      }
      umma_commit(mma_done);
    }
    if (t + (int)gridDim.x < ntiles) stage_features(t + gridDim.x);
    const bool got = cl_mbar_wait(mma_done, phase, spin_limit);
    phase ^= 1u;
    if (!__syncthreads_and(got)) {
      healthy = false;
      break;
    }
    tc_fence_after();
    // Epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its sub-partition) of blocks
    // w / 4, w / 4 + 4, w / 4 + 8; one thread per cell, its 32 channels in registers.
    for (int m = warp >> 2; m < kL2Blocks; m += kWarps / 4) {
      const int sp = warp & 3;
      uint32_t r32[32];
      tmem_ld32(tmem + ((uint32_t)(32 * sp) << 16) + (uint32_t)(m * 32), r32);
      const int p = kL2First + 128 * m + 32 * sp + lane;  // layer-1 flat index of this row
      const int r = p / kA1C - 1, c = p % kA1C - 1;      // layer-2 region coordinates
      if (r < 0 || r >= kA2R || c < 0 || c >= kA2C) continue;
      const int64_t x = x0 - 1 + r, y = y0 - 1 + c;
      const bool inside = x >= 0 && x < f.nx && y >= 0 && y < f.ny;
      uint32_t packed[C / 2];
#pragma unroll
      for (int ch = 0; ch < C; ch += 2) {
        const float v0 = inside ? gelu(__uint_as_float(r32[ch]) + bs[C + ch]) : 0.0f;
        const float v1 = inside ? gelu(__uint_as_float(r32[ch + 1]) + bs[C + ch + 1]) : 0.0f;
        packed[ch / 2] = (uint32_t)__bfloat16_as_ushort(to_bf(v0)) |
                         ((uint32_t)__bfloat16_as_ushort(to_bf(v1)) << 16);
      }
      uint4* dst = reinterpret_cast<uint4*>(a2s + (r * kA2C + c) * kCS);
#pragma unroll
      for (int q = 0; q < C / 8; ++q)
        dst[q] = make_uint4(packed[4 * q], packed[4 * q + 1], packed[4 * q + 2], packed[4 * q + 3]);
    }
    __syncthreads();

    // Layer 3 on tensor cores (N = 8 with only column 0 carrying w3; K = 288) and the relaxation
    // rate (the mapping of omega_kernel) on the output tile: 16 cells of one tile row per MMA tile.
    constexpr int n3 = kFR * kFC;
    for (int mt = warp; mt * 16 < n3; mt += kWarps) {
      const int j = (lane & 7) + 8 * ((lane >> 3) & 1);
      const int qa = mt * 16 + j;
      const int ra = qa / kFC, ca = qa - ra * kFC;
      float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll 1
      for (int tap = 0; tap < 9; ++tap) {
        const int dx = tap / 3 - 1, dy = tap % 3 - 1;
        const bf16* arow = a2s + ((ra + 1 + dx) * kA2C + ca + 1 + dy) * kCS + 8 * (lane >> 4);
#pragma unroll
        for (int kc = 0; kc < 2; ++kc) {
          uint32_t a[4];
          ldsm_x4(a, arow + kc * 16);
          // B column 0 = w3[tap][kc*16 + k]; lanes of the other columns hold zeros.
          uint32_t b0 = 0u, b1 = 0u;
          if (gq == 0) {
            const int k0 = tap * C + kc * 16 + 2 * tq;
            b0 = *reinterpret_cast<const uint32_t*>(w3b + k0);
            b1 = *reinterpret_cast<const uint32_t*>(w3b + k0 + 8);
          }
          mma_bf16(acc, a, b0, b1);
        }
      }
      if (tq == 0) {  // column 0: rows gq and gq + 8 of this tile
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int q = mt * 16 + gq + 8 * h;
          const int r = q / kFC, c = q - r * kFC;
          const int64_t x = x0 + r, y = y0 + c;
          if (x >= f.nx || y >= f.ny) continue;
          const float yv = acc[2 * h] + b3;
          const int64_t cell = x * f.ny + y;
          float tau = f.tau0;
          if (fluid_cell(f.flags[cell])) tau += fminf(f.max_dtau, f.gain * fmaxf(yv, 0.0f));
          f.omega[cell] = 1.0f / tau;
        }
      }
    }
  }
  if (!healthy) {
    if (threadIdx.x == 0) {
      atomicOr(&g_closure_status, 1);
      cl_mbar_wait(mma_done, phase ^ 1u);  // give MMAs still in flight a bounded chance to end
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols)
                 : "memory");
  }
}

// ---------------------------------------------------------------------------------------------
// Layer 2 of the training path on tcgen05: the forward conv (BWD = false: z2 = b2 + W * a1,
// a2 = GELU(z2) in BF16) and the transposed conv of the backward pass (BWD = true:
// d = W^T * dz2, dz1 = BF16(d GELU'(z1)), plus the per-channel sums of dz1 for the layer-1 bias
// gradient in this CTA's partial row). Same products as conv32_kernel, on the fifth-generation
// tensor cores with the layout of the fused inference kernel's layer 2:
//   - a tile of kTR x kTC output cells reads a (kTR + 2) x (kTC + 2) input region, staged
//     chunk-major: plane k (channels 8k .. 8k+7) holds 16 bytes a cell, cells in row-major order
//     of the region, so a tap shift (dx, dy) of the 3x3 stencil is an offset of the descriptor's
//     start address, dx (kTC + 2) + dy cells (the negated shift for the transposed conv);
//   - kTBlocks blocks of 128 consecutive region cells starting at output cell (0, 0), each an
//     M = 128, N = 32, K = 288 product into its own 32 TMEM columns; rows that fall on the
//     region's first or last column are computed and discarded;
//   - the B operand is the weights as K-chunks of 8: [k chunk][n][8] with k = (tap, ci) and
//     n = co for the forward conv, k = (tap, co) and n = ci for the transposed one.
// One thread issues the MMAs and commits them to an mbarrier (bounded wait, as everywhere); the
// epilogue reads each cell's 32 accumulators with tcgen05.ld. Two CTAs share an SM, so one stages
// its next tile while the other's MMAs and epilogue run.

constexpr int kTR = 14, kTC = 64;                  // output tile
constexpr int kTRegR = kTR + 2, kTRegC = kTC + 2;  // input region
constexpr int kTFirst = kTRegC + 1;                // region index of output cell (0, 0)
constexpr int kTBlocks = (kTR * kTRegC + 127) / 128;  // 128-cell blocks covering the output rows
constexpr int kTPad = 1168;  // cells per plane: >= kTFirst + 128 kTBlocks + kTRegC + 1, and a
                             // multiple of 8 so that every plane starts on a 128-byte boundary
constexpr int kTThreads = 256;
constexpr int kTTmemCols = 256;  // 8 accumulators of 32 FP32 columns
constexpr size_t kTOffW = (size_t)4 * kTPad * 16;
constexpr size_t kTOffBias = kTOffW + (size_t)36 * C * 16;
constexpr size_t kTOffBar = kTOffBias + (size_t)C * 4;  // MMA mbarrier, load mbarrier, TMEM addr
constexpr size_t kTSmem = kTOffBar + 24;
constexpr unsigned kTLoadBytes = 4u * kTRegR * kTRegC * 16;  // the four plane boxes of a tile
static_assert((size_t)kTThreads * (C + 1) * 4 <= kTOffW, "bias partial sums must fit the region");
static_assert(kTBlocks * 32 <= kTTmemCols, "accumulators exceed the TMEM allocation");
static_assert(kTFirst + kTBlocks * 128 + kTRegC + 1 <= kTPad, "planes too short for the shifts");
static_assert(kTFirst + kTBlocks * 128 - 1 >= (kTR * kTRegC) + kTC, "blocks do not cover the tile");
static_assert(kTFirst - kTRegC - 1 >= 0, "a negative shift leaves the plane");

// One plane of a tile's input region by the tensor engine: the activations as a 5D tensor
// (8 channels, 4 channel chunks, y, x, batch), box {8, 1, kTRegC, kTRegR, 1} at (0, chunk,
// y0 - 1, x0 - 1, b), which lands as kTRegR x kTRegC cells of 16 bytes in row-major order;
// cells outside the domain read as zero (the box may start at -1).
__device__ __forceinline__ void tc_plane_copy(void* dst, const CUtensorMap* map, int chunk, int y,
                                              int x, int b, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], "
      "[%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(chunk), "r"(y), "r"(x), "r"(b),
      "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void tc_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

template <bool BWD>
__global__ void __launch_bounds__(kTThreads, 2)
    conv32_tc_kernel(Grid g, const __grid_constant__ CUtensorMap in_map,
                     const bf16* __restrict__ w2, const float* __restrict__ bias,
                     const float* __restrict__ zin, float* __restrict__ zout,
                     bf16* __restrict__ out, float* __restrict__ partial) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* ac = smem_raw;                    // [4 planes][kTPad cells][16 B]
  unsigned char* wc = smem_raw + kTOffW;           // [36 K-chunks][32 n][16 B]
  float* bs = reinterpret_cast<float*>(smem_raw + kTOffBias);  // forward: b2
  uint64_t* mma_done = reinterpret_cast<uint64_t*>(smem_raw + kTOffBar);
  uint64_t* loaded = reinterpret_cast<uint64_t*>(smem_raw + kTOffBar + 8);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(smem_raw + kTOffBar + 16);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  constexpr int kWarps = kTThreads / 32;

  // The B operand. Forward: chunk kk = (tap, ci chunk) of output channel co, 8 consecutive
  // weights of the [co][288] row. Transposed: chunk kk = (tap, co chunk) of input channel ci,
  // weights W[8 cc .. 8 cc + 7][tap][ci].
  for (int i = threadIdx.x; i < 36 * C; i += blockDim.x) {
    const int kk = i / C, n = i - kk * C;
    if (!BWD) {
      *reinterpret_cast<uint4*>(wc + (size_t)i * 16) =
          __ldg(reinterpret_cast<const uint4*>(w2 + n * 288 + kk * 8));
    } else {
      const int tap = kk >> 2, cc = kk & 3;
      bf16 v[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) v[j] = w2[(cc * 8 + j) * 288 + tap * 32 + n];
      *reinterpret_cast<uint4*>(wc + (size_t)i * 16) = *reinterpret_cast<const uint4*>(v);
    }
  }
  if (!BWD && threadIdx.x < C) bs[threadIdx.x] = bias[threadIdx.x];
  // Plane cells past the region feed only discarded rows; keep them finite.
  for (int i = threadIdx.x; i < 4 * kTPad; i += blockDim.x)
    if (i % kTPad >= kTRegR * kTRegC)
      *reinterpret_cast<uint4*>(ac + (size_t)i * 16) = make_uint4(0, 0, 0, 0);
  // The weights and the zeroed plane tails, written here, are read by the MMAs (async proxy).
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (threadIdx.x == 0) {
    cl_mbar_init(mma_done, 1);
    cl_mbar_init(loaded, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(tmem_slot)),
                 "r"(kTTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t idesc = umma_idesc_bf16(128, 32);
  const unsigned ac_addr = smem_addr(ac), wc_addr = smem_addr(wc);
  const unsigned spin_limit = g_closure_spin_limit;
  bool healthy = true;
  unsigned phase = 0, load_phase = 0;
  float bias_sum[C];  // BWD: this thread's running sums of dz1 per channel
#pragma unroll
  for (int c = 0; c < C; ++c) bias_sum[c] = 0.0f;

  for (int64_t t = blockIdx.x; t < g.tiles && healthy; t += gridDim.x) {
    int64_t b, x0, y0;
    {
      const int64_t per = g.tx * g.ty;  // this kernel's tiles are kTR x kTC (see the launcher)
      b = t / per;
      const int64_t r = t - b * per;
      x0 = (r / g.ty) * kTR;
      y0 = (r % g.ty) * kTC;
    }
    // The input region, chunk-major, by four tensor copies (zero outside the domain).
    if (threadIdx.x == 0) {
      tc_expect_tx(loaded, kTLoadBytes);
#pragma unroll
      for (int k = 0; k < 4; ++k)
        tc_plane_copy(ac + (size_t)k * kTPad * 16, &in_map, k, (int)y0 - 1, (int)x0 - 1, (int)b,
                      loaded);
    }
    const bool have = cl_mbar_wait(loaded, load_phase);  // the copies take no spin limit: the
    load_phase ^= 1u;                                     // tile's MMAs need them
    if (!__syncthreads_and(have)) {
      healthy = false;
      break;
    }
    if (threadIdx.x == 0) {
      tc_fence_after();
      // K-slice outer, block inner: consecutive MMAs accumulate into different TMEM columns.
#pragma unroll 1
      for (int tap = 0; tap < 9; ++tap) {
        const int sh = (tap / 3 - 1) * kTRegC + (tap % 3 - 1);
        const int off = BWD ? -sh : sh;
#pragma unroll
        for (int kc = 0; kc < 2; ++kc) {
          const int sidx = tap * 2 + kc;
          const uint64_t bdesc = umma_desc(wc_addr + (unsigned)(sidx * 1024), C * 16, 128);
          const unsigned a_base = ac_addr + (unsigned)((2 * kc * kTPad + kTFirst + off) * 16);
#pragma unroll
          for (int m = 0; m < kTBlocks; ++m)
            umma_bf16(tmem + (uint32_t)(m * 32),
                      umma_desc(a_base + (unsigned)(m * 128 * 16), kTPad * 16, 128), bdesc, idesc,
                      sidx != 0);
        }
      }
      umma_commit(mma_done);
    }
    const bool got = cl_mbar_wait(mma_done, phase, spin_limit);
    phase ^= 1u;
    if (!__syncthreads_and(got)) {
      healthy = false;
      break;
    }
    tc_fence_after();
    // Epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its sub-partition) of blocks
    // w / 4, w / 4 + 2, ...; one thread per cell, its 32 channels in registers.
    for (int m = warp >> 2; m < kTBlocks; m += kWarps / 4) {
      const int sp = warp & 3;
      uint32_t r32[32];
      tmem_ld32(tmem + ((uint32_t)(32 * sp) << 16) + (uint32_t)(m * 32), r32);
      const int q = kTFirst + 128 * m + 32 * sp + lane;  // region index of this row
      const int r = q / kTRegC - 1, c = q % kTRegC - 1;   // output tile coordinates
      if (r < 0 || r >= kTR || c < 0 || c >= kTC) continue;
      const int64_t x = x0 + r, y = y0 + c;
      if (x >= g.nx || y >= g.ny) continue;
      const int64_t cell = g.cell(b, x, y);
      uint32_t packed[C / 2];
      if (!BWD) {
        float z[C];
#pragma unroll
        for (int ch = 0; ch < C; ++ch) z[ch] = __uint_as_float(r32[ch]) + bs[ch];
        if (zout != nullptr) {
          float4* zp = reinterpret_cast<float4*>(zout + cell * C);
#pragma unroll
          for (int k = 0; k < C / 4; ++k)
            zp[k] = make_float4(z[4 * k], z[4 * k + 1], z[4 * k + 2], z[4 * k + 3]);
        }
#pragma unroll
        for (int ch = 0; ch < C; ch += 2)
          packed[ch / 2] = (uint32_t)__bfloat16_as_ushort(to_bf(gelu(z[ch]))) |
                           ((uint32_t)__bfloat16_as_ushort(to_bf(gelu(z[ch + 1]))) << 16);
      } else {
        const float4* zp = reinterpret_cast<const float4*>(zin + cell * C);
#pragma unroll
        for (int k = 0; k < C / 4; ++k) {
          const float4 zz = zp[k];
          const float zv[4] = {zz.x, zz.y, zz.z, zz.w};
#pragma unroll
          for (int e = 0; e < 4; e += 2) {
            const int ch = 4 * k + e;
            const bf16 o0 = to_bf(__uint_as_float(r32[ch]) * gelu_grad(zv[e]));
            const bf16 o1 = to_bf(__uint_as_float(r32[ch + 1]) * gelu_grad(zv[e + 1]));
            bias_sum[ch] += bf(o0);
            bias_sum[ch + 1] += bf(o1);
            packed[ch / 2] =
                (uint32_t)__bfloat16_as_ushort(o0) | ((uint32_t)__bfloat16_as_ushort(o1) << 16);
          }
        }
      }
      uint4* op = reinterpret_cast<uint4*>(out + cell * C);
#pragma unroll
      for (int k = 0; k < C / 8; ++k)
        op[k] = make_uint4(packed[4 * k], packed[4 * k + 1], packed[4 * k + 2], packed[4 * k + 3]);
    }
    tc_fence_before();
    __syncthreads();  // the region and every TMEM column are free for the next tile
  }
  if (!healthy) {
    if (threadIdx.x == 0) {
      atomicOr(&g_closure_status, 1);
      // Give the copies and MMAs still in flight a bounded chance to end.
      cl_mbar_wait(loaded, load_phase ^ 1u);
      cl_mbar_wait(mma_done, phase ^ 1u);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTTmemCols)
                 : "memory");
  }
  if (BWD) {
    // Per-channel sums of this CTA's dz1 in a fixed order: thread sums in the region area (free
    // now; rows padded to C + 1 against bank conflicts), then channel c adds the 256 threads'
    // values in thread order.
    float* sums = reinterpret_cast<float*>(ac);  // [kTThreads][C + 1]
#pragma unroll
    for (int c = 0; c < C; ++c) sums[threadIdx.x * (C + 1) + c] = bias_sum[c];
    __syncthreads();
    if (threadIdx.x < C) {
      float s = 0.0f;
      for (int k = 0; k < kTThreads; ++k) s += sums[k * (C + 1) + threadIdx.x];
      partial[(int64_t)blockIdx.x * LBM_CLOSURE_PARAMS + LBM_CLOSURE_OFF_B1 + threadIdx.x] = s;
    }
  }
}

// The [batch][nx][ny][32] BF16 activations as conv32_tc_kernel's 5D tensor map (through the
// runtime's driver entry point: no link against libcuda). False when it cannot be encoded.
bool tc_input_map(CUtensorMap* map, const void* base, int64_t nx, int64_t ny, int64_t batch) {
  static PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  if (encode == nullptr || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
  if (nx >= (1ll << 31) || ny >= (1ll << 31) || batch >= (1ll << 31)) return false;
  const cuuint64_t dims[5] = {8, 4, (cuuint64_t)ny, (cuuint64_t)nx, (cuuint64_t)batch};
  const cuuint64_t strides[4] = {16, 64, (cuuint64_t)ny * 64, (cuuint64_t)(nx * ny) * 64};
  const cuuint32_t box[5] = {8, 1, (cuuint32_t)kTRegC, (cuuint32_t)kTRegR, 1};
  const cuuint32_t elem[5] = {1, 1, 1, 1, 1};
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 5, const_cast<void*>(base), dims, strides,
                box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tiles of kTR x kTC cells for conv32_tc_kernel.
Grid tc_grid(int64_t nx, int64_t ny, int64_t batch) {
  Grid g{nx, ny, batch, (nx + kTR - 1) / kTR, (ny + kTC - 1) / kTC, 0};
  g.tiles = g.tx * g.ty * batch;
  return g;
}

// Which kernel runs layer 2 of the training path (lbm_closure_set_layer2_kernel).
int g_layer2_kernel = LBM_CLOSURE_LAYER2_TCGEN05;

// ---------------------------------------------------------------------------------------------
// Optimiser, relaxation field, coarsening

__global__ void adam_kernel(float* __restrict__ p, bf16* __restrict__ pb, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, float lr, float beta1,
                            float beta2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= LBM_CLOSURE_PARAMS) return;
  const float gi = g[i];
  const float mi = beta1 * m[i] + (1.0f - beta1) * gi;
  const float vi = beta2 * v[i] + (1.0f - beta2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
  p[i] = pi;
  pb[i] = to_bf(pi);
}

__global__ void sync_bf16_kernel(const float* __restrict__ p, bf16* __restrict__ pb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < LBM_CLOSURE_PARAMS) pb[i] = to_bf(p[i]);
}

__global__ void omega_kernel(const float* __restrict__ y, const int32_t* __restrict__ flags,
                             int64_t n, float tau0, float gain, float max_dtau,
                             float* __restrict__ omega) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float tau = tau0;
  if (fluid_cell(flags[i])) tau += fminf(max_dtau, gain * fmaxf(y[i], 0.0f));
  omega[i] = 1.0f / tau;
}

__global__ void coarsen_kernel(const float* __restrict__ rho, const float* __restrict__ vel,
                               const float* __restrict__ c, int64_t nx, int64_t ny, int f,
                               float* __restrict__ rho_c, float* __restrict__ vel_c,
                               float* __restrict__ c_c, float* __restrict__ sgs) {
  const int64_t cx_n = nx / f, cy_n = ny / f;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= cx_n * cy_n) return;
  const int64_t cx = i / cy_n, cy = i - cx * cy_n;
  float sr = 0.0f, su = 0.0f, sv = 0.0f, sc = 0.0f;
  for (int a = 0; a < f; ++a)
    for (int b = 0; b < f; ++b) {
      const int64_t j = (cx * f + a) * ny + cy * f + b;
      sr += rho[j];
      su += vel[2 * j];
      sv += vel[2 * j + 1];
      if (c != nullptr) sc += c[j];
    }
  const float inv = 1.0f / (float)(f * f);
  const float mu = su * inv, mv = sv * inv;
  float k = 0.0f;
  for (int a = 0; a < f; ++a)
    for (int b = 0; b < f; ++b) {
      const int64_t j = (cx * f + a) * ny + cy * f + b;
      const float du = vel[2 * j] - mu, dv = vel[2 * j + 1] - mv;
      k = fmaf(du, du, fmaf(dv, dv, k));
    }
  if (rho_c != nullptr) rho_c[i] = sr * inv;
  if (vel_c != nullptr) {
    vel_c[2 * i] = mu;
    vel_c[2 * i + 1] = mv;
  }
  if (c_c != nullptr && c != nullptr) c_c[i] = sc * inv;
  if (sgs != nullptr) sgs[i] = sqrtf(0.5f * k * inv);
}

// ---------------------------------------------------------------------------------------------

int blocks_for(int64_t n, int threads) { return (int)((n + threads - 1) / threads); }

int device_sms() {
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess)
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

bool shape_ok(int64_t nx, int64_t ny, int64_t batch) {
  return nx >= 2 && ny >= 2 && batch >= 1 && nx * ny * batch < (int64_t(1) << 40);
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

int set_smem(const void* fn, size_t bytes) {
  CL_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return LBM_OK;
}

// Workspace: [count (8 B, padded to 256)][loss partials (kLossBlocks doubles, padded)]
//            [dz2 BF16 [cells][32]][dz1 BF16 [cells][32]][partial rows FP32 [kPartialRows][P]]
constexpr int64_t kWsCount = 0;
constexpr int64_t kWsLoss = 256;
constexpr int64_t kWsDz = kWsLoss + ((kLossBlocks * 8 + 255) / 256) * 256;

int64_t round256(int64_t v) { return (v + 255) / 256 * 256; }

}  // namespace

extern "C" {

int lbm_postproc_curl2d(const float* vel, int64_t nx, int64_t ny, float* out, void* stream) {
  if (!vel || !out || nx < 2 || ny < 2) return fail(LBM_ERR_ARGUMENT, "curl2d: bad arguments");
  curl2d_kernel<<<blocks_for(nx * ny, 256), 256, 0, (cudaStream_t)stream>>>(vel, nx, ny, out);
  CL_CUDA(cudaGetLastError());
  return LBM_OK;
}

int lbm_postproc_curl3d(const float* vel, int64_t nx, int64_t ny, int64_t nz, float* out,
                        void* stream) {
  if (!vel || !out || nx < 2 || ny < 2 || nz < 2)
    return fail(LBM_ERR_ARGUMENT, "curl3d: bad arguments");
  curl3d_kernel<<<blocks_for(nx * ny * nz, 256), 256, 0, (cudaStream_t)stream>>>(vel, nx, ny, nz,
                                                                                 out);
  CL_CUDA(cudaGetLastError());
  return LBM_OK;
}

int lbm_postproc_vmag(const float* vel, int64_t n, int dim, float* out, void* stream) {
  if (!vel || !out || n < 0 || dim < 1 || dim > 3) return fail(LBM_ERR_ARGUMENT, "vmag: bad arguments");
  if (n == 0) return LBM_OK;
  vmag_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(vel, n, dim, out);
  CL_CUDA(cudaGetLastError());
  return LBM_OK;
}

int lbm_closure_features(const float* rho, const float* vel, const int32_t* flags, int64_t nx,
                         int64_t ny, int64_t batch, const float* norm, uint16_t* x, void* stream) {
  if (!rho || !vel || !flags || !norm || !x || !shape_ok(nx, ny, batch))
    return fail(LBM_ERR_ARGUMENT, "closure features: bad arguments");
  if (!aligned16(x)) return fail(LBM_ERR_ARGUMENT, "closure features: x must be 16-byte aligned");
  Norm nm;
  for (int c = 0; c < 4; ++c) {
    nm.mean[c] = norm[c];
    nm.inv_std[c] = norm[4 + c];
  }
  features_kernel<<<blocks_for(nx * ny * batch, 256), 256, 0, (cudaStream_t)stream>>>(
      rho, vel, flags, nx, ny, batch, nm, reinterpret_cast<bf16*>(x));
  CL_CUDA(cudaGetLastError());
  return LBM_OK;
}

int lbm_closure_forward(const float* params, const uint16_t* params_bf16, const uint16_t* x,
                        int64_t nx, int64_t ny, int64_t batch, float* z1, uint16_t* a1, float* z2,
                        uint16_t* a2, float* y, void* stream) {
  if (!params || !params_bf16 || !x || !a1 || !a2 || !y || !shape_ok(nx, ny, batch))
    return fail(LBM_ERR_ARGUMENT, "closure forward: bad arguments");
  if (!aligned16(params_bf16) || !aligned16(x) || !aligned16(a1) || !aligned16(a2) ||
      (z1 && !aligned16(z1)) || (z2 && !aligned16(z2)))
    return fail(LBM_ERR_ARGUMENT, "closure forward: arrays must be 16-byte aligned");
  static thread_local bool configured = false;
  if (!configured) {
    if (int rc = set_smem((const void*)conv32_kernel<false>, kConv32Smem)) return rc;
    if (int rc = set_smem((const void*)conv32_kernel<true>, kConv32Smem)) return rc;
    if (int rc = set_smem((const void*)conv32_tc_kernel<false>, kTSmem)) return rc;
    if (int rc = set_smem((const void*)conv3_fwd_kernel, kConv3Smem)) return rc;
    configured = true;
  }
  const Grid g = make_grid(nx, ny, batch);
  const cudaStream_t s = (cudaStream_t)stream;
  const int sms = device_sms();
  const auto* wb = reinterpret_cast<const bf16*>(params_bf16);
  const int grid_small = (int)std::min<int64_t>(g.tiles, (int64_t)sms * 4);
  conv1_fwd_kernel<<<grid_small, 256, 0, s>>>(g, reinterpret_cast<const bf16*>(x),
                                              wb + LBM_CLOSURE_OFF_W1, params + LBM_CLOSURE_OFF_B1,
                                              z1, reinterpret_cast<bf16*>(a1));
  CL_CUDA(cudaGetLastError());
  CUtensorMap a1_map;
  if (g_layer2_kernel == LBM_CLOSURE_LAYER2_TCGEN05 && tc_input_map(&a1_map, a1, nx, ny, batch)) {
    const Grid gt = tc_grid(nx, ny, batch);
    const int grid_tc = (int)std::min<int64_t>(gt.tiles, (int64_t)sms * 2);
    conv32_tc_kernel<false><<<grid_tc, kTThreads, kTSmem, s>>>(
        gt, a1_map, wb + LBM_CLOSURE_OFF_W2, params + LBM_CLOSURE_OFF_B2, nullptr, z2,
        reinterpret_cast<bf16*>(a2), nullptr);
  } else {
    const int grid32 = (int)std::min<int64_t>(g.tiles, (int64_t)sms * 4);
    conv32_kernel<false><<<grid32, kConv32Threads, kConv32Smem, s>>>(
        g, reinterpret_cast<const bf16*>(a1), wb + LBM_CLOSURE_OFF_W2,
        params + LBM_CLOSURE_OFF_B2, nullptr, z2, reinterpret_cast<bf16*>(a2), nullptr);
  }
  CL_CUDA(cudaGetLastError());
  conv3_fwd_kernel<<<grid_small, 256, kConv3Smem, s>>>(g, reinterpret_cast<const bf16*>(a2),
                                                       wb + LBM_CLOSURE_OFF_W3,
                                                       params + LBM_CLOSURE_OFF_B3, y);
  CL_CUDA(cudaGetLastError());
  return LBM_OK;
}

int64_t lbm_closure_workspace_bytes(int64_t nx, int64_t ny, int64_t batch) {
  if (!shape_ok(nx, ny, batch)) return -1;
  const int64_t dz = round256(nx * ny * batch * C * 2);
  return kWsDz + 2 * dz + (int64_t)kPartialRows * LBM_CLOSURE_PARAMS * 4;
}

int lbm_closure_loss(const float* y, const float* target, const int32_t* flags, int64_t nx,
                     int64_t ny, int64_t batch, float* dy, double* loss, void* workspace,
                     void* stream) {
  if (!y || !target || !flags || !dy || !loss || !workspace || !shape_ok(nx, ny, batch))
    return fail(LBM_ERR_ARGUMENT, "closure loss: bad arguments");
  const cudaStream_t s = (cudaStream_t)stream;
  auto* base = static_cast<unsigned char*>(workspace);
  auto* count = reinterpret_cast<unsigned long long*>(base + kWsCount);
  auto* partial = reinterpret_cast<double*>(base + kWsLoss);
  const int64_t n = nx * ny;
  count_kernel<<<1, 1024, 0, s>>>(flags, n, count);
  CL_CUDA(cudaGetLastError());
  loss_kernel<<<kLossBlocks, 256, 0, s>>>(y, target, flags, n, batch, count, dy, partial);
  CL_CUDA(cudaGetLastError());
  loss_final_kernel<<<1, 1, 0, s>>>(partial, kLossBlocks, count, batch, loss);
  CL_CUDA(cudaGetLastError());
  return LBM_OK;
}

int lbm_closure_backward(const float* params, const uint16_t* params_bf16, const uint16_t* x,
                         const float* z1, const uint16_t* a1, const float* z2, const uint16_t* a2,
                         const float* dy, int64_t nx, int64_t ny, int64_t batch, float* grad,
                         void* workspace, void* stream) {
  if (!params || !params_bf16 || !x || !z1 || !a1 || !z2 || !a2 || !dy || !grad || !workspace ||
      !shape_ok(nx, ny, batch))
    return fail(LBM_ERR_ARGUMENT, "closure backward: bad arguments");
  if (!aligned16(workspace) || !aligned16(params_bf16) || !aligned16(x) || !aligned16(z1) ||
      !aligned16(a1) || !aligned16(z2) || !aligned16(a2))
    return fail(LBM_ERR_ARGUMENT, "closure backward: arrays must be 16-byte aligned");
  static thread_local bool configured = false;
  if (!configured) {
    if (int rc = set_smem((const void*)conv32_kernel<false>, kConv32Smem)) return rc;
    if (int rc = set_smem((const void*)conv32_kernel<true>, kConv32Smem)) return rc;
    if (int rc = set_smem((const void*)conv32_tc_kernel<true>, kTSmem)) return rc;
    if (int rc = set_smem((const void*)conv32_wgrad_kernel, kDw2Smem)) return rc;
    if (int rc = set_smem((const void*)conv3_bwd_kernel, kConv3BwdSmem)) return rc;
    configured = true;
  }
  const Grid g = make_grid(nx, ny, batch);
  const cudaStream_t s = (cudaStream_t)stream;
  auto* base = static_cast<unsigned char*>(workspace);
  const int64_t dzb = round256(nx * ny * batch * C * 2);
  auto* dz2 = reinterpret_cast<bf16*>(base + kWsDz);
  auto* dz1 = reinterpret_cast<bf16*>(base + kWsDz + dzb);
  auto* partial = reinterpret_cast<float*>(base + kWsDz + 2 * dzb);
  const auto* wb = reinterpret_cast<const bf16*>(params_bf16);
  const int rows = (int)std::min<int64_t>(g.tiles, kPartialRows);

  conv3_bwd_kernel<<<rows, 256, kConv3BwdSmem, s>>>(g, reinterpret_cast<const bf16*>(a2), z2,
                                                    wb + LBM_CLOSURE_OFF_W3, dy, dz2, partial);
  CL_CUDA(cudaGetLastError());
  conv32_wgrad_kernel<<<rows, kDw2Threads, kDw2Smem, s>>>(g, reinterpret_cast<const bf16*>(a1),
                                                          dz2, partial);
  CL_CUDA(cudaGetLastError());
  CUtensorMap dz2_map;
  if (g_layer2_kernel == LBM_CLOSURE_LAYER2_TCGEN05 && tc_input_map(&dz2_map, dz2, nx, ny, batch)) {
    // Same number of CTAs (partial rows) as the other reducing kernels: a CTA without a tile
    // writes a zero row.
    conv32_tc_kernel<true><<<rows, kTThreads, kTSmem, s>>>(
        tc_grid(nx, ny, batch), dz2_map, wb + LBM_CLOSURE_OFF_W2, nullptr, z1, nullptr, dz1,
        partial);
  } else {
    conv32_kernel<true><<<rows, kConv32Threads, kConv32Smem, s>>>(
        g, dz2, wb + LBM_CLOSURE_OFF_W2, nullptr, z1, nullptr, dz1, partial);
  }
  CL_CUDA(cudaGetLastError());
  conv1_wgrad_kernel<<<rows, 288, kTX * kTY * kCS * sizeof(bf16), s>>>(
      g, reinterpret_cast<const bf16*>(x), dz1, partial);
  CL_CUDA(cudaGetLastError());
  reduce_rows_kernel<<<blocks_for(LBM_CLOSURE_PARAMS, 256), 256, 0, s>>>(partial, rows, grad);
  CL_CUDA(cudaGetLastError());
  return LBM_OK;
}

int lbm_closure_adam(float* params, uint16_t* params_bf16, const float* grad, float* m, float* v,
                     float lr, float beta1, float beta2, float eps, int64_t step, void* stream) {
  if (!params || !params_bf16 || !grad || !m || !v || step < 1)
    return fail(LBM_ERR_ARGUMENT, "closure adam: bad arguments");
  const float c1 = (float)(1.0 / (1.0 - std::pow((double)beta1, (double)step)));
  const float c2 = (float)(1.0 / (1.0 - std::pow((double)beta2, (double)step)));
  adam_kernel<<<blocks_for(LBM_CLOSURE_PARAMS, 256), 256, 0, (cudaStream_t)stream>>>(
      params, reinterpret_cast<bf16*>(params_bf16), grad, m, v, lr, beta1, beta2, eps, c1, c2);
  CL_CUDA(cudaGetLastError());
  return LBM_OK;
}

int lbm_closure_sync_bf16(const float* params, uint16_t* params_bf16, void* stream) {
  if (!params || !params_bf16) return fail(LBM_ERR_ARGUMENT, "closure sync: bad arguments");
  sync_bf16_kernel<<<blocks_for(LBM_CLOSURE_PARAMS, 256), 256, 0, (cudaStream_t)stream>>>(
      params, reinterpret_cast<bf16*>(params_bf16));
  CL_CUDA(cudaGetLastError());
  return LBM_OK;
}

int lbm_closure_omega(const float* y, const int32_t* flags, int64_t nx, int64_t ny, float tau0,
                      float gain, float max_dtau, float* omega, void* stream) {
  if (!y || !flags || !omega || nx < 1 || ny < 1 || !(tau0 > 0.5f) || !(max_dtau >= 0.0f))
    return fail(LBM_ERR_ARGUMENT, "closure omega: bad arguments");
  omega_kernel<<<blocks_for(nx * ny, 256), 256, 0, (cudaStream_t)stream>>>(y, flags, nx * ny, tau0,
                                                                         gain, max_dtau, omega);
  CL_CUDA(cudaGetLastError());
  return LBM_OK;
}

int lbm_closure_relaxation(const float* params, const uint16_t* params_bf16, const float* rho,
                           const float* vel, const int32_t* flags, int64_t nx, int64_t ny,
                           const float* norm, float tau0, float gain, float max_dtau,
                           float* omega, void* stream) {
  if (!params || !params_bf16 || !rho || !vel || !flags || !norm || !omega || nx < 2 || ny < 2 ||
      !(tau0 > 0.5f) || !(max_dtau >= 0.0f))
    return fail(LBM_ERR_ARGUMENT, "closure relaxation: bad arguments");
  if (!aligned16(params_bf16))
    return fail(LBM_ERR_ARGUMENT, "closure relaxation: params_bf16 must be 16-byte aligned");
  static thread_local bool configured = false;
  if (!configured) {
    if (int rc = set_smem((const void*)closure_fused_kernel, kFusedSmem)) return rc;
    configured = true;
  }
  FusedArgs fa;
  fa.params = params;
  fa.wb = reinterpret_cast<const bf16*>(params_bf16);
  fa.rho = rho;
  fa.vel = vel;
  fa.flags = flags;
  fa.nx = nx;
  fa.ny = ny;
  for (int c = 0; c < 4; ++c) {
    fa.norm.mean[c] = norm[c];
    fa.norm.inv_std[c] = norm[4 + c];
  }
  fa.tau0 = tau0;
  fa.gain = gain;
  fa.max_dtau = max_dtau;
  fa.omega = omega;
  fa.tiles_x = (int)((nx + kFR - 1) / kFR);
  fa.tiles_y = (int)((ny + kFC - 1) / kFC);
  const int64_t ntiles = (int64_t)fa.tiles_x * fa.tiles_y;
  const int grid = (int)std::min<int64_t>(ntiles, (int64_t)device_sms());
  closure_fused_kernel<<<grid, kFusedThreads, kFusedSmem, (cudaStream_t)stream>>>(fa);
  CL_CUDA(cudaGetLastError());
  return LBM_OK;
}

int lbm_closure_set_layer2_kernel(int kind) {
  if (kind != LBM_CLOSURE_LAYER2_TCGEN05 && kind != LBM_CLOSURE_LAYER2_WARP_MMA)
    return fail(LBM_ERR_ARGUMENT, "unknown layer-2 kernel");
  g_layer2_kernel = kind;
  return LBM_OK;
}

int lbm_closure_set_spin_limit(int64_t polls) {
  const unsigned v = polls < 0 ? kClosureSpinLimit
                               : (unsigned)std::min<int64_t>(polls, (int64_t)kClosureSpinLimit);
  CL_CUDA(cudaMemcpyToSymbol(g_closure_spin_limit, &v, sizeof(unsigned)));
  return LBM_OK;
}

int lbm_closure_status(void) {
  int word = 0;
  CL_CUDA(cudaMemcpyFromSymbol(&word, g_closure_status, sizeof(int)));
  if (word == 0) return LBM_OK;
  const int zero = 0;
  CL_CUDA(cudaMemcpyToSymbol(g_closure_status, &zero, sizeof(int)));
  return fail(LBM_ERR_STATE,
              "closure relaxation: a kernel gave up waiting for its tensor-core products");
}

int lbm_closure_coarsen(const float* rho, const float* vel, const float* c, int64_t nx, int64_t ny,
                        int factor, float* rho_c, float* vel_c, float* c_c, float* sgs,
                        void* stream) {
  if (!rho || !vel || factor < 1 || nx % factor != 0 || ny % factor != 0 || nx < 1 || ny < 1)
    return fail(LBM_ERR_ARGUMENT, "closure coarsen: nx and ny must be multiples of the factor");
  const int64_t n = (nx / factor) * (ny / factor);
  coarsen_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(rho, vel, c, nx, ny, factor,
                                                                       rho_c, vel_c, c_c, sgs);
  CL_CUDA(cudaGetLastError());
  return LBM_OK;
}

}  // extern "C"
