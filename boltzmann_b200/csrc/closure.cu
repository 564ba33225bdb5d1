// Learned subgrid closure (3-layer CNN on the coarse lattice) and on-device post-processing.
//
// No counterpart in the reference. The network: 3x3 convolutions 4 -> 32 -> 32 -> 1 with GELU
// after the first two layers, zero padding at the domain edges, channels-last activations.
//
//   layer   forward                       backward
//   1 (4->32)   CUDA cores (36 MAC/out)    weights: CUDA cores; no input gradient
//   2 (32->32)  mma.sync BF16, FP32 acc    data: mma.sync (transposed conv, fused GELU');
//                                          weights: mma.sync (cells are the reduction axis)
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
#include <cuda_bf16.h>
#include <cuda_runtime.h>

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

__device__ __forceinline__ float gelu(float z) {
  return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}

__device__ __forceinline__ float gelu_grad(float z) {
  const float cdf = 0.5f * (1.0f + erff(z * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
  return cdf + z * pdf;
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

__global__ void features_kernel(const float* __restrict__ rho, const float* __restrict__ vel,
                                const int32_t* __restrict__ flags, int64_t nx, int64_t ny,
                                int64_t batch, Norm norm, bf16* __restrict__ x_out) {
  const int64_t n = nx * ny;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n * batch) return;
  const int64_t b = i / n, cell = i - b * n;
  const int64_t x = cell / ny, y = cell - x * ny;
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
  reinterpret_cast<uint2*>(x_out)[i] = packed;
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
  const int grid32 = (int)std::min<int64_t>(g.tiles, (int64_t)sms * 4);
  conv32_kernel<false><<<grid32, kConv32Threads, kConv32Smem, s>>>(
      g, reinterpret_cast<const bf16*>(a1), wb + LBM_CLOSURE_OFF_W2, params + LBM_CLOSURE_OFF_B2,
      nullptr, z2, reinterpret_cast<bf16*>(a2), nullptr);
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
  conv32_kernel<true><<<rows, kConv32Threads, kConv32Smem, s>>>(
      g, dz2, wb + LBM_CLOSURE_OFF_W2, nullptr, z1, nullptr, dz1, partial);
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
