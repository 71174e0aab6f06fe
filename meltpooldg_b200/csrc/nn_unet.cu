// Learned initial guess: a small 3D U-Net (BF16 weights and activations, FP32
// accumulation) with its own forward, backward and Adam kernels, behind the C
// ABI (mpdg_unet_* in include/mpdg_heat.h).
//
// Network (channels per level 16/32/48/64, 3x3x3 convolutions, zero padding):
//   e0 = relu(c(relu(c(x))))            3 -> 16 -> 16     level 0 (input grid)
//   e1 = relu(c(relu(c(pool(e0)))))     16 -> 32 -> 32    level 1 (ceil(n/2))
//   e2 = relu(c(relu(c(pool(e1)))))     32 -> 48 -> 48    level 2
//   e3 = relu(c(relu(c(pool(e2)))))     48 -> 64 -> 64    level 3
//   d2 = relu(c(relu(c(up(e3)) + e2)))  64 -> 48 -> 48
//   d1 = relu(c(relu(c(up(d2)) + e1)))  48 -> 32 -> 32
//   d0 = relu(c(relu(c(up(d1)) + e0)))  32 -> 16 -> 16
//   y  = c(d0)                          16 -> 1, linear, FP32
// pool = 2x2x2 average over the in-range children, up = nearest-neighbour.
//
// Tensors are planar [C][z][y][x]; activations BF16, activation gradients FP32,
// weights [Cout][Cin][27] as FP32 masters plus a BF16 copy used by the kernels.
// The forward convolutions run on the tensor cores (tcgen05 implicit GEMM,
// nn_conv_tc.cuh), and so do the data gradients of the backward pass: the
// output gradient, rounded to BF16, convolved with the flipped, channel-
// transposed weights (packed beside the forward ones), FP32 out
// (MPDG_UNET_TC_BWD=0 keeps them on the CUDA cores in FP32). The weight
// gradients and the CUDA-core forward (MPDG_UNET_TC=0) use k_conv3d: a CTA
// holds an 8x8x4 output tile and 16 output channels, stages one input
// channel's tile plus halo and its 16 x 27 weights in shared memory at a time
// and accumulates in FP32 registers.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mpdg_heat.h"
#include "nn_conv_tc.cuh"
#include "reduce.cuh"

using namespace mpdg;

namespace {

thread_local std::string g_nn_err;
int nn_fail(int code, const std::string &m)
{
  g_nn_err = m;
  return code;
}
#define NNCU(call)                                                                               \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess)                                                                       \
      return nn_fail(e_ == cudaErrorMemoryAllocation ? MPDG_ERR_OUT_OF_MEMORY : MPDG_ERR_CUDA,   \
                     std::string(#call) + ": " + cudaGetErrorString(e_));                         \
  } while (0)
#define NNTRY(call)                \
  do {                             \
    int r_ = (call);               \
    if (r_ != MPDG_OK) return r_;  \
  } while (0)

constexpr int TX = 8, TY = 8, TZ = 4, TP = TX * TY * TZ;  // output tile
constexpr int HX = TX + 2, HY = TY + 2, HZ = TZ + 2, HP = HX * HY * HZ;
constexpr int COB = 16;  // output channels per CTA

struct Grid3 {
  int nx, ny, nz;
  __host__ __device__ int64_t n() const { return (int64_t)nx * ny * nz; }
};

template <typename T> __device__ __forceinline__ float tof(T v);
template <> __device__ __forceinline__ float tof<float>(float v) { return v; }
template <> __device__ __forceinline__ float tof<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <typename T> __device__ __forceinline__ T fromf(float v);
template <> __device__ __forceinline__ float fromf<float>(float v) { return v; }
template <> __device__ __forceinline__ __nv_bfloat16 fromf<__nv_bfloat16>(float v) { return __float2bfloat16(v); }

// BF16 activations are channel-chunked, [ceil(C/8)][points][8] (one 16-byte vector per point and
// 8-channel chunk, pad channels zero); FP32 tensors (gradients, the output) are planar [C][points]
__host__ __device__ __forceinline__ int64_t aidx(int c, int64_t p, int64_t np)
{
  return ((int64_t)(c >> 3) * np + p) * 8 + (c & 7);
}
template <typename T> __device__ __forceinline__ int64_t tidx(int c, int64_t p, int64_t np);
template <> __device__ __forceinline__ int64_t tidx<float>(int c, int64_t p, int64_t np)
{
  return (int64_t)c * np + p;
}
template <> __device__ __forceinline__ int64_t tidx<__nv_bfloat16>(int c, int64_t p, int64_t np)
{
  return aidx(c, p, np);
}
__host__ __device__ constexpr int pad8(int c) { return (c + 7) & ~7; }

// out[co][p] = bias[co] + sum_ci sum_o w[co][ci][o] in[ci][p + o - 1]
//   (+ add[co][p]) ; relu ; (* (mask[co][p] > 0))
// flip: use w[ci][co][26 - o] (the transposed convolution of the backward pass)
template <typename TI, typename TO, bool RELU, bool ADD, bool MASK, bool FLIP>
__global__ void __launch_bounds__(TP) k_conv3d(Grid3 g, int Ci, int Co, const TI *__restrict__ in,
                                               const __nv_bfloat16 *__restrict__ w,
                                               const float *__restrict__ bias,
                                               const __nv_bfloat16 *__restrict__ add,
                                               const __nv_bfloat16 *__restrict__ mask, TO *out)
{
  __shared__ float s_in[HP];
  __shared__ float s_w[COB * 27];
  const int tiles_x = (g.nx + TX - 1) / TX, tiles_y = (g.ny + TY - 1) / TY;
  const int tile = blockIdx.x;
  const int bx = (tile % tiles_x) * TX, by = ((tile / tiles_x) % tiles_y) * TY,
            bz = (tile / (tiles_x * tiles_y)) * TZ;
  const int co0 = blockIdx.y * COB;
  const int tx = threadIdx.x % TX, ty = (threadIdx.x / TX) % TY, tz = threadIdx.x / (TX * TY);
  const int x = bx + tx, y = by + ty, z = bz + tz;
  const bool inside = x < g.nx && y < g.ny && z < g.nz;
  const int64_t np = g.n();
  float acc[COB];
#pragma unroll
  for (int c = 0; c < COB; ++c) acc[c] = 0.f;
  for (int ci = 0; ci < Ci; ++ci) {
    for (int i = threadIdx.x; i < HP; i += TP) {
      const int hx = i % HX, hy = (i / HX) % HY, hz = i / (HX * HY);
      const int gx = bx + hx - 1, gy = by + hy - 1, gz = bz + hz - 1;
      float v = 0.f;
      if (gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny && gz >= 0 && gz < g.nz)
        v = tof<TI>(in[tidx<TI>(ci, (int64_t)gx + (int64_t)g.nx * (gy + (int64_t)g.ny * gz), np)]);
      s_in[i] = v;
    }
    for (int i = threadIdx.x; i < COB * 27; i += TP) {
      const int c = i / 27, o = i % 27;
      const int co = co0 + c;
      float v = 0.f;
      if (co < Co)
        v = FLIP ? __bfloat162float(w[((int64_t)ci * Co + co) * 27 + (26 - o)])
                 : __bfloat162float(w[((int64_t)co * Ci + ci) * 27 + o]);
      s_w[i] = v;
    }
    __syncthreads();
    float v[27];
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
      for (int dy = 0; dy < 3; ++dy)
#pragma unroll
        for (int dx = 0; dx < 3; ++dx)
          v[dx + 3 * (dy + 3 * dz)] = s_in[(tx + dx) + HX * ((ty + dy) + HY * (tz + dz))];
#pragma unroll
    for (int c = 0; c < COB; ++c) {
      float s = acc[c];
#pragma unroll
      for (int o = 0; o < 27; ++o) s = fmaf(s_w[c * 27 + o], v[o], s);
      acc[c] = s;
    }
    __syncthreads();
  }
  if (!inside) return;
  const int64_t p = (int64_t)x + (int64_t)g.nx * (y + (int64_t)g.ny * z);
#pragma unroll
  for (int c = 0; c < COB; ++c) {
    const int co = co0 + c;
    if (co >= Co) break;
    float r = acc[c] + (bias ? bias[co] : 0.f);
    if (ADD) r += __bfloat162float(add[aidx(co, p, np)]);
    if (RELU) r = fmaxf(r, 0.f);
    if (MASK) r = __bfloat162float(mask[aidx(co, p, np)]) > 0.f ? r : 0.f;
    out[tidx<TO>(co, p, np)] = fromf<TO>(r);
  }
}

// dw[co][ci][o] += sum_p gout[co][p] in[ci][p + o - 1] ; db[co] += sum_p gout[co][p]
// CTA: one 8x8x4 tile, 16 co x 16 ci, thread (co, ci) keeps 27 accumulators.
constexpr int CIB = 8;  // 16 co x 8 ci per CTA keeps the staged tiles under 48 KB
__global__ void __launch_bounds__(COB * CIB) k_conv3d_wgrad(Grid3 g, int Ci, int Co,
                                                      const __nv_bfloat16 *__restrict__ in,
                                                      const float *__restrict__ gout, float *dw,
                                                      float *db)
{
  __shared__ float s_g[COB * TP];
  __shared__ float s_in[CIB * HP];
  const int tiles_x = (g.nx + TX - 1) / TX, tiles_y = (g.ny + TY - 1) / TY;
  const int tile = blockIdx.x;
  const int bx = (tile % tiles_x) * TX, by = ((tile / tiles_x) % tiles_y) * TY,
            bz = (tile / (tiles_x * tiles_y)) * TZ;
  const int co0 = blockIdx.y * COB, ci0 = blockIdx.z * CIB;
  const int64_t np = g.n();
  for (int i = threadIdx.x; i < COB * TP; i += blockDim.x) {
    const int c = i / TP, t = i % TP;
    const int x = bx + t % TX, y = by + (t / TX) % TY, z = bz + t / (TX * TY);
    const int co = co0 + c;
    float v = 0.f;
    if (co < Co && x < g.nx && y < g.ny && z < g.nz)
      v = gout[(int64_t)co * np + x + (int64_t)g.nx * (y + (int64_t)g.ny * z)];
    s_g[i] = v;
  }
  for (int i = threadIdx.x; i < CIB * HP; i += blockDim.x) {
    const int c = i / HP, hh = i % HP;
    const int hx = hh % HX, hy = (hh / HX) % HY, hz = hh / (HX * HY);
    const int gx = bx + hx - 1, gy = by + hy - 1, gz = bz + hz - 1;
    const int ci = ci0 + c;
    float v = 0.f;
    if (ci < Ci && gx >= 0 && gx < g.nx && gy >= 0 && gy < g.ny && gz >= 0 && gz < g.nz)
      v = __bfloat162float(in[aidx(ci, gx + (int64_t)g.nx * (gy + (int64_t)g.ny * gz), np)]);
    s_in[i] = v;
  }
  __syncthreads();
  const int c = threadIdx.x / CIB, k = threadIdx.x % CIB;  // c: co offset, k: ci offset
  float acc[27];
#pragma unroll
  for (int o = 0; o < 27; ++o) acc[o] = 0.f;
  float bsum = 0.f;
  for (int t = 0; t < TP; ++t) {
    const float gv = s_g[c * TP + t];
    bsum += gv;
    const int tx = t % TX, ty = (t / TX) % TY, tz = t / (TX * TY);
    const float *sp = s_in + k * HP + tx + HX * (ty + HY * tz);
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
      for (int dy = 0; dy < 3; ++dy)
#pragma unroll
        for (int dx = 0; dx < 3; ++dx)
          acc[dx + 3 * (dy + 3 * dz)] = fmaf(gv, sp[dx + HX * (dy + HY * dz)], acc[dx + 3 * (dy + 3 * dz)]);
  }
  const int co = co0 + c, ci = ci0 + k;
  if (co < Co && ci < Ci) {
#pragma unroll
    for (int o = 0; o < 27; ++o) atomicAdd(dw + ((int64_t)co * Ci + ci) * 27 + o, acc[o]);
  }
  if (db && blockIdx.z == 0 && k == 0 && co < Co) atomicAdd(db + co, bsum);
}

__host__ __device__ inline Grid3 coarse(Grid3 g) { return {(g.nx + 1) / 2, (g.ny + 1) / 2, (g.nz + 1) / 2}; }

// 2x2x2 average over the in-range children
__global__ void k_pool(Grid3 f, int C, const __nv_bfloat16 *__restrict__ in, __nv_bfloat16 *out)
{
  const Grid3 c = coarse(f);
  const int64_t n = c.n() * C;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int ch = (int)(t / c.n());
    const int64_t p = t % c.n();
    const int X = (int)(p % c.nx), Y = (int)((p / c.nx) % c.ny), Z = (int)(p / ((int64_t)c.nx * c.ny));
    float s = 0.f;
    int cnt = 0;
    for (int dz = 0; dz < 2; ++dz)
      for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
          const int x = 2 * X + dx, y = 2 * Y + dy, z = 2 * Z + dz;
          if (x < f.nx && y < f.ny && z < f.nz) {
            s += __bfloat162float(in[aidx(ch, x + (int64_t)f.nx * (y + (int64_t)f.ny * z), f.n())]);
            ++cnt;
          }
        }
    out[aidx(ch, p, c.n())] = __float2bfloat16(s / cnt);
  }
}

// gin[fine] += gout[coarse] / count(coarse)
__global__ void k_pool_bwd(Grid3 f, int C, const float *__restrict__ gout, float *gin)
{
  const Grid3 c = coarse(f);
  const int64_t n = f.n() * C;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int ch = (int)(t / f.n());
    const int64_t p = t % f.n();
    const int x = (int)(p % f.nx), y = (int)((p / f.nx) % f.ny), z = (int)(p / ((int64_t)f.nx * f.ny));
    const int X = x / 2, Y = y / 2, Z = z / 2;
    const int cx = (2 * X + 1 < f.nx) ? 2 : 1, cy = (2 * Y + 1 < f.ny) ? 2 : 1, cz = (2 * Z + 1 < f.nz) ? 2 : 1;
    gin[t] += gout[(int64_t)ch * c.n() + X + (int64_t)c.nx * (Y + (int64_t)c.ny * Z)] / (float)(cx * cy * cz);
  }
}

// nearest-neighbour upsampling coarse -> fine
__global__ void k_up(Grid3 f, int C, const __nv_bfloat16 *__restrict__ in, __nv_bfloat16 *out)
{
  const Grid3 c = coarse(f);
  const int64_t n = f.n() * C;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int ch = (int)(t / f.n());
    const int64_t p = t % f.n();
    const int x = (int)(p % f.nx), y = (int)((p / f.nx) % f.ny), z = (int)(p / ((int64_t)f.nx * f.ny));
    out[aidx(ch, p, f.n())] = in[aidx(ch, x / 2 + (int64_t)c.nx * (y / 2 + (int64_t)c.ny * (z / 2)), c.n())];
  }
}

// gin[coarse] = sum of gout over its fine children
__global__ void k_up_bwd(Grid3 f, int C, const float *__restrict__ gout, float *gin)
{
  const Grid3 c = coarse(f);
  const int64_t n = c.n() * C;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int ch = (int)(t / c.n());
    const int64_t p = t % c.n();
    const int X = (int)(p % c.nx), Y = (int)((p / c.nx) % c.ny), Z = (int)(p / ((int64_t)c.nx * c.ny));
    float s = 0.f;
    for (int dz = 0; dz < 2; ++dz)
      for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) {
          const int x = 2 * X + dx, y = 2 * Y + dy, z = 2 * Z + dz;
          if (x < f.nx && y < f.ny && z < f.nz)
            s += gout[(int64_t)ch * f.n() + x + (int64_t)f.nx * (y + (int64_t)f.ny * z)];
        }
    gin[t] = s;
  }
}

// g[c][p] *= (y[c][p] > 0) for C channels of np points (y chunked, g planar)
__global__ void k_relu_mask(int64_t np, int C, const __nv_bfloat16 *__restrict__ y, float *g)
{
  const int64_t n = np * C;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    if (!(__bfloat162float(y[aidx((int)(t / np), t % np, np)]) > 0.f)) g[t] = 0.f;
}

__global__ void k_add_inplace(int64_t n, float *a, const float *__restrict__ b)
{
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    a[t] += b[t];
}

__global__ void k_f32_to_bf16(int64_t n, const float *__restrict__ a, __nv_bfloat16 *b)
{
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
    b[t] = __float2bfloat16(a[t]);
}

// planar FP32 [C][np] -> chunked BF16 [ceil(C/8)][np][8], pad channels zero
__global__ void k_f32_to_chunked(int64_t np, int C, const float *__restrict__ a, __nv_bfloat16 *b)
{
  const int64_t n = np * pad8(C);
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(t & 7) + 8 * (int)(t / (8 * np));
    const int64_t p = (t >> 3) % np;
    b[t] = __float2bfloat16(c < C ? a[(int64_t)c * np + p] : 0.f);
  }
}

// loss = mean (y - target)^2 ; g = 2 (y - target) / n
__global__ void k_mse(int64_t n, const float *__restrict__ y, const float *__restrict__ target,
                      float *g, double *partials, unsigned *counter, double *loss)
{
  double v[1] = {0.0};
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const float d = y[t] - target[t];
    if (g) g[t] = 2.f * d / (float)n;
    v[0] += (double)d * d;
  }
  double tot[1];
  if (grid_sum<1>(v, partials, counter, tot)) *loss = tot[0] / (double)n;
}

__global__ void k_adam(int64_t n, float *p, const float *__restrict__ g, float *m, float *v, float lr,
                       float b1, float b2, float eps, float c1, float c2, __nv_bfloat16 *pb)
{
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
    const float gt = g[t];
    const float mt = b1 * m[t] + (1.f - b1) * gt;
    const float vt = b2 * v[t] + (1.f - b2) * gt * gt;
    m[t] = mt;
    v[t] = vt;
    const float np = p[t] - lr * (mt / c1) / (sqrtf(vt / c2) + eps);
    p[t] = np;
    pb[t] = __float2bfloat16(np);
  }
}

int grid1d(int64_t n) { return (int)std::min<int64_t>((n + 255) / 256, 148 * 16); }

}  // namespace

// ---------------------------------------------------------------------------
// the network
// ---------------------------------------------------------------------------
struct ConvL {
  int ci, co;
  int64_t woff, boff;  // offsets into the parameter vector
};

struct mpdg_unet {
  cudaStream_t stream = nullptr;
  Grid3 g[4];
  ConvL L[15];
  int64_t n_params = 0;
  float *p = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
  __nv_bfloat16 *pb = nullptr;
  uint4 *wpk = nullptr;       // weights packed for the tensor-core convolution
  int64_t wpk_off[15] = {};   // per layer, in uint4
  uint4 *wpkt = nullptr;      // flipped, channel-transposed packs (the data gradient)
  int64_t wpkt_off[15] = {};
  bool use_tc_bwd = true;     // data gradients on the tensor cores
  __nv_bfloat16 *gbf = nullptr;  // an output gradient in BF16 (the tensor cores' input)
  float *zero_bias = nullptr;    // 64 zeros
  bool wpk_dirty = true;      // pb changed since the last packing
  bool use_tc = true;         // forward convolutions on the tensor cores
  bool training = false;      // forward keeps what the backward pass reads
  bool ups_valid = false;     // u2, u1, u0 hold the upsampled decoder inputs
  // raised by a tensor-core convolution whose wait expired: page-locked mapped host memory
  // (tc_err is its device address), read by the host without a synchronisation
  int *tc_err = nullptr, *tc_err_host = nullptr;
  int sm_count = 148;
  int64_t step = 0;
  // activations (BF16) and gradients (FP32)
  std::vector<void *> owned;
  __nv_bfloat16 *x0, *a0, *e0, *p0, *a1, *e1, *p1, *a2, *e2, *p2, *a3, *e3, *u2, *s2, *d2, *u1, *s1,
    *d1, *u0, *s0, *d0;
  float *y;
  float *gA, *gB, *gC, *gE0, *gE1, *gE2;  // gradient scratch
  double *partials, *lossd;
  unsigned *counter;
};

namespace {

enum { E0A, E0B, E1A, E1B, E2A, E2B, E3A, E3B, D2A, D2B, D1A, D1B, D0A, D0B, OUT };
const int kCi[15] = {3, 16, 16, 32, 32, 48, 48, 64, 64, 48, 48, 32, 32, 16, 16};
const int kCo[15] = {16, 16, 32, 32, 48, 48, 64, 64, 48, 48, 32, 32, 16, 16, 1};
const int kLevel[15] = {0, 0, 1, 1, 2, 2, 3, 3, 2, 2, 1, 1, 0, 0, 0};  // the grid of each layer

uint64_t mix(uint64_t x)
{
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

template <typename TI, typename TO, bool RELU, bool ADD, bool MASK, bool FLIP>
int conv(mpdg_unet *u, Grid3 g, int Ci, int Co, const TI *in, const __nv_bfloat16 *w,
         const float *bias, const __nv_bfloat16 *add, const __nv_bfloat16 *mask, TO *out)
{
  const int tiles = ((g.nx + TX - 1) / TX) * ((g.ny + TY - 1) / TY) * ((g.nz + TZ - 1) / TZ);
  dim3 grid(tiles, (Co + COB - 1) / COB);
  k_conv3d<TI, TO, RELU, ADD, MASK, FLIP><<<grid, TP, 0, u->stream>>>(g, Ci, Co, in, w, bias, add,
                                                                      mask, out);
  NNCU(cudaGetLastError());
  return MPDG_OK;
}

int wgrad(mpdg_unet *u, Grid3 g, int l, const __nv_bfloat16 *in, const float *gout)
{
  const ConvL &L = u->L[l];
  const int tiles = ((g.nx + TX - 1) / TX) * ((g.ny + TY - 1) / TY) * ((g.nz + TZ - 1) / TZ);
  dim3 grid(tiles, (L.co + COB - 1) / COB, (L.ci + CIB - 1) / CIB);
  k_conv3d_wgrad<<<grid, COB * CIB, 0, u->stream>>>(g, L.ci, L.co, in, gout, u->grad + L.woff,
                                              u->grad + L.boff);
  NNCU(cudaGetLastError());
  return MPDG_OK;
}

const __nv_bfloat16 *W(mpdg_unet *u, int l) { return u->pb + u->L[l].woff; }
const float *B(mpdg_unet *u, int l) { return u->p + u->L[l].boff; }

int npad_of(int co) { return (co + 15) / 16 * 16; }
int cg_of(int ci) { return (ci + 15) / 16; }

int pack_weights(mpdg_unet *u)
{
  for (int l = 0; l < 15; ++l) {
    const int ci = u->L[l].ci, co = u->L[l].co;
    nn_tc::k_pack_weights<<<64, 256, 0, u->stream>>>(ci, co, cg_of(ci), npad_of(co), W(u, l),
                                                     u->wpk + u->wpk_off[l]);
    if (u->wpkt)
      nn_tc::k_pack_weights_t<<<64, 256, 0, u->stream>>>(ci, co, cg_of(co), npad_of(ci), W(u, l),
                                                         u->wpkt + u->wpkt_off[l]);
  }
  NNCU(cudaGetLastError());
  u->wpk_dirty = false;
  return MPDG_OK;
}

template <int NPAD, bool RELU, bool ADD, typename TO>
int tc_launch(mpdg_unet *u, Grid3 g, int ci, int co, const uint4 *wp, const float *bias,
              const __nv_bfloat16 *in, const __nv_bfloat16 *add, TO *out, const Grid3 *up_from)
{
  auto k = nn_tc::k_conv3d_tc<NPAD, RELU, ADD, TO>;
  static size_t attr_smem = 0;  // the attribute is kept at the request of the launch, so
                                // that the occupancy query sees the real footprint
  nn_tc::ConvArgs a;
  a.nx = g.nx;
  a.ny = g.ny;
  a.nz = g.nz;
  a.ci = ci;
  a.co = co;
  a.cg = cg_of(a.ci);
  a.taps_per_stage = nn_tc::smem_bytes(a.cg, NPAD, 27) <= 200 * 1024 ? 27 : 9;
  a.up = up_from != nullptr;
  a.sx = up_from ? up_from->nx : g.nx;
  a.sy = up_from ? up_from->ny : g.ny;
  a.sz = up_from ? up_from->nz : g.nz;
  a.in = in;
  a.wp = wp;
  a.bias = bias;
  a.add = add;
  a.out = out;
  a.err = u->tc_err;
  const size_t smem = nn_tc::smem_bytes(a.cg, NPAD, a.taps_per_stage);
  if (smem != attr_smem) {
    NNCU(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr_smem = smem;
  }
  // resident CTAs per SM from registers, shared memory, threads and tensor-memory columns
  static int per_sm_regs = 0, smem_sm = 0, smem_rsv = 0, static_smem = 0;
  if (per_sm_regs == 0) {
    cudaFuncAttributes fa;
    NNCU(cudaFuncGetAttributes(&fa, k));
    int dev = 0;
    NNCU(cudaGetDevice(&dev));
    NNCU(cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    NNCU(cudaDeviceGetAttribute(&smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev));
    static_smem = (int)fa.sharedSizeBytes;
    per_sm_regs = 65536 / (((fa.numRegs + 7) / 8 * 8) * nn_tc::kThreads);
  }
  int per_sm = std::min(per_sm_regs, smem_sm / ((int)smem + static_smem + smem_rsv));
  per_sm = std::min(per_sm, 2048 / nn_tc::kThreads);
  per_sm = std::max(1, std::min(per_sm, 512 / nn_tc::tmem_cols(NPAD)));
  const int64_t tiles = (int64_t)((g.nx + nn_tc::TCX - 1) / nn_tc::TCX) *
                        ((g.ny + nn_tc::TCY - 1) / nn_tc::TCY) * g.nz;
  const int grid = (int)std::min<int64_t>(tiles, (int64_t)per_sm * u->sm_count);
  k<<<grid, nn_tc::kThreads, smem, u->stream>>>(a);
  NNCU(cudaGetLastError());
  return MPDG_OK;
}

template <int NPAD, bool RELU, bool ADD, typename TO>
int conv_tc_t(mpdg_unet *u, int l, Grid3 g, const __nv_bfloat16 *in, const __nv_bfloat16 *add,
              TO *out, const Grid3 *up_from)
{
  return tc_launch<NPAD, RELU, ADD, TO>(u, g, u->L[l].ci, u->L[l].co, u->wpk + u->wpk_off[l],
                                        B(u, l), in, add, out, up_from);
}

template <bool RELU, bool ADD, typename TO>
int conv_tc(mpdg_unet *u, int l, Grid3 g, const __nv_bfloat16 *in, const __nv_bfloat16 *add,
            TO *out, const Grid3 *up_from = nullptr)
{
  if (u->wpk_dirty) NNTRY(pack_weights(u));
  switch (npad_of(u->L[l].co)) {
  case 16: return conv_tc_t<16, RELU, ADD, TO>(u, l, g, in, add, out, up_from);
  case 32: return conv_tc_t<32, RELU, ADD, TO>(u, l, g, in, add, out, up_from);
  case 48: return conv_tc_t<48, RELU, ADD, TO>(u, l, g, in, add, out, up_from);
  case 64: return conv_tc_t<64, RELU, ADD, TO>(u, l, g, in, add, out, up_from);
  default: return nn_fail(MPDG_ERR_INVALID_ARGUMENT, "tensor-core convolution: Cout > 64");
  }
}

// conv + relu (activation out, BF16)
int conv_relu(mpdg_unet *u, int l, Grid3 g, const __nv_bfloat16 *in, __nv_bfloat16 *out,
              const __nv_bfloat16 *add = nullptr)
{
  if (u->use_tc)
    return add ? conv_tc<true, true>(u, l, g, in, add, out)
               : conv_tc<true, false>(u, l, g, in, (const __nv_bfloat16 *)nullptr, out);
  if (add)
    return conv<__nv_bfloat16, __nv_bfloat16, true, true, false, false>(u, g, u->L[l].ci, u->L[l].co, in, W(u, l), B(u, l), add, nullptr, out);
  return conv<__nv_bfloat16, __nv_bfloat16, true, false, false, false>(u, g, u->L[l].ci, u->L[l].co, in, W(u, l), B(u, l), nullptr, nullptr, out);
}

// gin = (W^T * gout) [* (mask > 0)] on the tensor cores: gout rounded to BF16, convolved with
// the flipped, channel-transposed weights (FP32 accumulation and output), then masked
int dgrad_tc(mpdg_unet *u, int l, Grid3 g, const float *gout, float *gin,
             const __nv_bfloat16 *mask)
{
  if (u->wpk_dirty) NNTRY(pack_weights(u));
  const int ci = u->L[l].ci, co = u->L[l].co;
  const int64_t n = g.n();
  k_f32_to_chunked<<<grid1d((int64_t)pad8(co) * n), 256, 0, u->stream>>>(n, co, gout, u->gbf);
  NNCU(cudaGetLastError());
  const uint4 *wp = u->wpkt + u->wpkt_off[l];
  int rc;
  switch (npad_of(ci)) {
  case 16: rc = tc_launch<16, false, false, float>(u, g, co, ci, wp, u->zero_bias, u->gbf, nullptr, gin, nullptr); break;
  case 32: rc = tc_launch<32, false, false, float>(u, g, co, ci, wp, u->zero_bias, u->gbf, nullptr, gin, nullptr); break;
  case 48: rc = tc_launch<48, false, false, float>(u, g, co, ci, wp, u->zero_bias, u->gbf, nullptr, gin, nullptr); break;
  case 64: rc = tc_launch<64, false, false, float>(u, g, co, ci, wp, u->zero_bias, u->gbf, nullptr, gin, nullptr); break;
  default: return nn_fail(MPDG_ERR_INVALID_ARGUMENT, "tensor-core data gradient: Cin > 64");
  }
  NNTRY(rc);
  if (mask) {
    k_relu_mask<<<grid1d((int64_t)ci * n), 256, 0, u->stream>>>(n, ci, mask, gin);
    NNCU(cudaGetLastError());
  }
  return MPDG_OK;
}

// gin = (W^T * gout) [* (mask > 0)]
int dgrad(mpdg_unet *u, int l, Grid3 g, const float *gout, float *gin, const __nv_bfloat16 *mask)
{
  if (u->use_tc && u->use_tc_bwd) return dgrad_tc(u, l, g, gout, gin, mask);
  if (mask)
    return conv<float, float, false, false, true, true>(u, g, u->L[l].co, u->L[l].ci, gout, W(u, l), nullptr, nullptr, mask, gin);
  return conv<float, float, false, false, false, true>(u, g, u->L[l].co, u->L[l].ci, gout, W(u, l), nullptr, nullptr, nullptr, gin);
}

// the error flag of the tensor-core convolutions, read (and cleared) without a synchronisation:
// a forward's expired wait is reported by the next call that checks
int check_tc_err(mpdg_unet *u)
{
  if (u->tc_err_host && *(volatile int *)u->tc_err_host) {
    *(volatile int *)u->tc_err_host = 0;
    return nn_fail(MPDG_ERR_CUDA, "tensor-core convolution: wait for the MMAs expired");
  }
  return MPDG_OK;
}

int forward(mpdg_unet *u)
{
  const Grid3 *g = u->g;
  auto pool = [&](Grid3 f, int C, const __nv_bfloat16 *in, __nv_bfloat16 *out) -> int {
    k_pool<<<grid1d(coarse(f).n() * C), 256, 0, u->stream>>>(f, C, in, out);
    NNCU(cudaGetLastError());
    return MPDG_OK;
  };
  auto up = [&](Grid3 f, int C, const __nv_bfloat16 *in, __nv_bfloat16 *out) -> int {
    k_up<<<grid1d(f.n() * C), 256, 0, u->stream>>>(f, C, in, out);
    NNCU(cudaGetLastError());
    return MPDG_OK;
  };
  NNTRY(conv_relu(u, E0A, g[0], u->x0, u->a0));
  NNTRY(conv_relu(u, E0B, g[0], u->a0, u->e0));
  NNTRY(pool(g[0], 16, u->e0, u->p0));
  NNTRY(conv_relu(u, E1A, g[1], u->p0, u->a1));
  NNTRY(conv_relu(u, E1B, g[1], u->a1, u->e1));
  NNTRY(pool(g[1], 32, u->e1, u->p1));
  NNTRY(conv_relu(u, E2A, g[2], u->p1, u->a2));
  NNTRY(conv_relu(u, E2B, g[2], u->a2, u->e2));
  NNTRY(pool(g[2], 48, u->e2, u->p2));
  NNTRY(conv_relu(u, E3A, g[3], u->p2, u->a3));
  NNTRY(conv_relu(u, E3B, g[3], u->a3, u->e3));
  // decoder: with the tensor-core path the upsampling is fused into the halo load of
  // the next convolution (the upsampled tensors are then formed only for training)
  u->ups_valid = !u->use_tc || u->training;
  if (u->use_tc) {
    if (u->training) NNTRY(up(g[2], 64, u->e3, u->u2));
    NNTRY((conv_tc<true, true>(u, D2A, g[2], u->e3, u->e2, u->s2, &g[3])));
    NNTRY(conv_relu(u, D2B, g[2], u->s2, u->d2));
    if (u->training) NNTRY(up(g[1], 48, u->d2, u->u1));
    NNTRY((conv_tc<true, true>(u, D1A, g[1], u->d2, u->e1, u->s1, &g[2])));
    NNTRY(conv_relu(u, D1B, g[1], u->s1, u->d1));
    if (u->training) NNTRY(up(g[0], 32, u->d1, u->u0));
    NNTRY((conv_tc<true, true>(u, D0A, g[0], u->d1, u->e0, u->s0, &g[1])));
    NNTRY(conv_relu(u, D0B, g[0], u->s0, u->d0));
    return conv_tc<false, false>(u, OUT, g[0], u->d0, (const __nv_bfloat16 *)nullptr, u->y);
  }
  NNTRY(up(g[2], 64, u->e3, u->u2));
  NNTRY(conv_relu(u, D2A, g[2], u->u2, u->s2, u->e2));
  NNTRY(conv_relu(u, D2B, g[2], u->s2, u->d2));
  NNTRY(up(g[1], 48, u->d2, u->u1));
  NNTRY(conv_relu(u, D1A, g[1], u->u1, u->s1, u->e1));
  NNTRY(conv_relu(u, D1B, g[1], u->s1, u->d1));
  NNTRY(up(g[0], 32, u->d1, u->u0));
  NNTRY(conv_relu(u, D0A, g[0], u->u0, u->s0, u->e0));
  NNTRY(conv_relu(u, D0B, g[0], u->s0, u->d0));
  return conv<__nv_bfloat16, float, false, false, false, false>(u, g[0], 16, 1, u->d0, W(u, OUT), B(u, OUT), nullptr, nullptr, u->y);
}

// gradients of sum(gy * y) with respect to the parameters (after forward)
int backward(mpdg_unet *u, const float *gy)
{
  const Grid3 *g = u->g;
  if (!u->ups_valid) {  // an inference forward fused the upsampling: form its outputs now
    k_up<<<grid1d(g[2].n() * 64), 256, 0, u->stream>>>(g[2], 64, u->e3, u->u2);
    k_up<<<grid1d(g[1].n() * 48), 256, 0, u->stream>>>(g[1], 48, u->d2, u->u1);
    k_up<<<grid1d(g[0].n() * 32), 256, 0, u->stream>>>(g[0], 32, u->d1, u->u0);
    NNCU(cudaGetLastError());
    u->ups_valid = true;
  }
  NNCU(cudaMemsetAsync(u->grad, 0, sizeof(float) * u->n_params, u->stream));
  float *gA = u->gA, *gB = u->gB, *gC = u->gC;
  auto relu_mask = [&](Grid3 gr, int C, const __nv_bfloat16 *y, float *gg) -> int {
    k_relu_mask<<<grid1d(gr.n() * C), 256, 0, u->stream>>>(gr.n(), C, y, gg);
    NNCU(cudaGetLastError());
    return MPDG_OK;
  };
  auto addi = [&](int64_t n, float *a, const float *b) -> int {
    k_add_inplace<<<grid1d(n), 256, 0, u->stream>>>(n, a, b);
    NNCU(cudaGetLastError());
    return MPDG_OK;
  };
  auto up_bwd = [&](Grid3 f, int C, const float *go, float *gi) -> int {
    k_up_bwd<<<grid1d(coarse(f).n() * C), 256, 0, u->stream>>>(f, C, go, gi);
    NNCU(cudaGetLastError());
    return MPDG_OK;
  };
  auto pool_bwd = [&](Grid3 f, int C, const float *go, float *gi) -> int {
    k_pool_bwd<<<grid1d(f.n() * C), 256, 0, u->stream>>>(f, C, go, gi);
    NNCU(cudaGetLastError());
    return MPDG_OK;
  };
  // output layer: y = W d0 + b
  NNTRY(wgrad(u, g[0], OUT, u->d0, gy));
  NNTRY(dgrad(u, OUT, g[0], gy, gA, u->d0));            // gA: pre-relu of d0
  NNTRY(wgrad(u, g[0], D0B, u->s0, gA));
  NNTRY(dgrad(u, D0B, g[0], gA, gB, u->s0));            // gB: pre-relu of s0
  NNTRY(wgrad(u, g[0], D0A, u->u0, gB));
  NNCU(cudaMemcpyAsync(u->gE0, gB, sizeof(float) * 16 * g[0].n(), cudaMemcpyDeviceToDevice, u->stream));
  NNTRY(dgrad(u, D0A, g[0], gB, gC, nullptr));          // gC: d u0 (32 @ g0)
  NNTRY(up_bwd(g[0], 32, gC, gA));                      // gA: d d1 (32 @ g1)
  NNTRY(relu_mask(g[1], 32, u->d1, gA));
  NNTRY(wgrad(u, g[1], D1B, u->s1, gA));
  NNTRY(dgrad(u, D1B, g[1], gA, gB, u->s1));
  NNTRY(wgrad(u, g[1], D1A, u->u1, gB));
  NNCU(cudaMemcpyAsync(u->gE1, gB, sizeof(float) * 32 * g[1].n(), cudaMemcpyDeviceToDevice, u->stream));
  NNTRY(dgrad(u, D1A, g[1], gB, gC, nullptr));          // d u1 (48 @ g1)
  NNTRY(up_bwd(g[1], 48, gC, gA));                      // d d2 (48 @ g2)
  NNTRY(relu_mask(g[2], 48, u->d2, gA));
  NNTRY(wgrad(u, g[2], D2B, u->s2, gA));
  NNTRY(dgrad(u, D2B, g[2], gA, gB, u->s2));
  NNTRY(wgrad(u, g[2], D2A, u->u2, gB));
  NNCU(cudaMemcpyAsync(u->gE2, gB, sizeof(float) * 48 * g[2].n(), cudaMemcpyDeviceToDevice, u->stream));
  NNTRY(dgrad(u, D2A, g[2], gB, gC, nullptr));          // d u2 (64 @ g2)
  NNTRY(up_bwd(g[2], 64, gC, gA));                      // d e3 (64 @ g3)
  NNTRY(relu_mask(g[3], 64, u->e3, gA));
  NNTRY(wgrad(u, g[3], E3B, u->a3, gA));
  NNTRY(dgrad(u, E3B, g[3], gA, gB, u->a3));
  NNTRY(wgrad(u, g[3], E3A, u->p2, gB));
  NNTRY(dgrad(u, E3A, g[3], gB, gC, nullptr));          // d p2 (48 @ g3)
  NNTRY(pool_bwd(g[2], 48, gC, u->gE2));                // d e2 += pool^T
  NNTRY(relu_mask(g[2], 48, u->e2, u->gE2));
  NNTRY(wgrad(u, g[2], E2B, u->a2, u->gE2));
  NNTRY(dgrad(u, E2B, g[2], u->gE2, gB, u->a2));
  NNTRY(wgrad(u, g[2], E2A, u->p1, gB));
  NNTRY(dgrad(u, E2A, g[2], gB, gC, nullptr));          // d p1 (32 @ g2)
  NNTRY(pool_bwd(g[1], 32, gC, u->gE1));
  NNTRY(relu_mask(g[1], 32, u->e1, u->gE1));
  NNTRY(wgrad(u, g[1], E1B, u->a1, u->gE1));
  NNTRY(dgrad(u, E1B, g[1], u->gE1, gB, u->a1));
  NNTRY(wgrad(u, g[1], E1A, u->p0, gB));
  NNTRY(dgrad(u, E1A, g[1], gB, gC, nullptr));          // d p0 (16 @ g1)
  NNTRY(pool_bwd(g[0], 16, gC, u->gE0));
  NNTRY(relu_mask(g[0], 16, u->e0, u->gE0));
  NNTRY(wgrad(u, g[0], E0B, u->a0, u->gE0));
  NNTRY(dgrad(u, E0B, g[0], u->gE0, gB, u->a0));
  NNTRY(wgrad(u, g[0], E0A, u->x0, gB));
  (void)addi;
  return MPDG_OK;
}

int ualloc(mpdg_unet *u, void **p, size_t bytes)
{
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) return nn_fail(MPDG_ERR_OUT_OF_MEMORY, "cudaMalloc (unet)");
  u->owned.push_back(*p);
  return MPDG_OK;
}

}  // namespace

extern "C" const char *mpdg_unet_last_error(void) { return g_nn_err.c_str(); }

extern "C" int mpdg_unet_create(int nx, int ny, int nz, uint64_t seed, mpdg_unet **out)
{
  if (!out || nx < 8 || ny < 8 || nz < 8) return nn_fail(MPDG_ERR_INVALID_ARGUMENT, "grid must be >= 8^3");
  mpdg_unet *u = new mpdg_unet();
  u->g[0] = {nx, ny, nz};
  for (int l = 1; l < 4; ++l) u->g[l] = coarse(u->g[l - 1]);
  int64_t off = 0;
  for (int l = 0; l < 15; ++l) {
    u->L[l].ci = kCi[l];
    u->L[l].co = kCo[l];
    u->L[l].woff = off;
    off += (int64_t)kCi[l] * kCo[l] * 27;
    u->L[l].boff = off;
    off += kCo[l];
  }
  u->n_params = off;
  auto fail_free = [&](int rc) {
    for (void *p : u->owned) cudaFree(p);
    if (u->tc_err_host) cudaFreeHost(u->tc_err_host);
    delete u;
    return rc;
  };
  const int64_t n0 = u->g[0].n(), n1 = u->g[1].n(), n2 = u->g[2].n(), n3 = u->g[3].n();
  struct A { __nv_bfloat16 **p; int64_t n; } acts[] = {
    {&u->x0, 8 * n0}, {&u->a0, 16 * n0}, {&u->e0, 16 * n0}, {&u->p0, 16 * n1}, {&u->a1, 32 * n1},
    {&u->e1, 32 * n1}, {&u->p1, 32 * n2}, {&u->a2, 48 * n2}, {&u->e2, 48 * n2}, {&u->p2, 48 * n3},
    {&u->a3, 64 * n3}, {&u->e3, 64 * n3}, {&u->u2, 64 * n2}, {&u->s2, 48 * n2}, {&u->d2, 48 * n2},
    {&u->u1, 48 * n1}, {&u->s1, 32 * n1}, {&u->d1, 32 * n1}, {&u->u0, 32 * n0}, {&u->s0, 16 * n0},
    {&u->d0, 16 * n0}};
  int rc;
  for (auto &a : acts)
    if ((rc = ualloc(u, (void **)a.p, sizeof(__nv_bfloat16) * a.n)) != MPDG_OK) return fail_free(rc);
  const int64_t gmax = std::max(std::max(32 * n0, 48 * n1), std::max(64 * n2, 64 * n3));
  float **fb[] = {&u->y, &u->gA, &u->gB, &u->gC};
  const int64_t fsz[] = {n0, gmax, gmax, gmax};
  for (int i = 0; i < 4; ++i)
    if ((rc = ualloc(u, (void **)fb[i], sizeof(float) * fsz[i])) != MPDG_OK) return fail_free(rc);
  if ((rc = ualloc(u, (void **)&u->gE0, sizeof(float) * 16 * n0)) != MPDG_OK ||
      (rc = ualloc(u, (void **)&u->gE1, sizeof(float) * 32 * n1)) != MPDG_OK ||
      (rc = ualloc(u, (void **)&u->gE2, sizeof(float) * 48 * n2)) != MPDG_OK ||
      (rc = ualloc(u, (void **)&u->p, sizeof(float) * u->n_params)) != MPDG_OK ||
      (rc = ualloc(u, (void **)&u->grad, sizeof(float) * u->n_params)) != MPDG_OK ||
      (rc = ualloc(u, (void **)&u->m, sizeof(float) * u->n_params)) != MPDG_OK ||
      (rc = ualloc(u, (void **)&u->v, sizeof(float) * u->n_params)) != MPDG_OK ||
      (rc = ualloc(u, (void **)&u->pb, sizeof(__nv_bfloat16) * u->n_params)) != MPDG_OK ||
      (rc = ualloc(u, (void **)&u->partials, sizeof(double) * 148 * 16)) != MPDG_OK ||
      (rc = ualloc(u, (void **)&u->lossd, sizeof(double) * 2)) != MPDG_OK ||
      (rc = ualloc(u, (void **)&u->counter, sizeof(unsigned) * 4)) != MPDG_OK)
    return fail_free(rc);
  if (cudaHostAlloc((void **)&u->tc_err_host, sizeof(int), cudaHostAllocMapped) != cudaSuccess)
    return fail_free(nn_fail(MPDG_ERR_OUT_OF_MEMORY, "cudaHostAlloc (unet)"));
  *u->tc_err_host = 0;
  if (cudaHostGetDevicePointer((void **)&u->tc_err, u->tc_err_host, 0) != cudaSuccess)
    return fail_free(nn_fail(MPDG_ERR_CUDA, "cudaHostGetDevicePointer (unet)"));
  int64_t wtot = 0;
  for (int l = 0; l < 15; ++l) {
    u->wpk_off[l] = wtot;
    wtot += (int64_t)27 * cg_of(kCi[l]) * 2 * npad_of(kCo[l]);
  }
  if ((rc = ualloc(u, (void **)&u->wpk, sizeof(uint4) * wtot)) != MPDG_OK) return fail_free(rc);
  int64_t wtot_t = 0, gbf_n = 0;
  for (int l = 0; l < 15; ++l) {
    u->wpkt_off[l] = wtot_t;
    wtot_t += (int64_t)27 * cg_of(kCo[l]) * 2 * npad_of(kCi[l]);
    gbf_n = std::max(gbf_n, (int64_t)pad8(kCo[l]) * u->g[kLevel[l]].n());  // an output gradient
  }
  if ((rc = ualloc(u, (void **)&u->wpkt, sizeof(uint4) * wtot_t)) != MPDG_OK ||
      (rc = ualloc(u, (void **)&u->gbf, sizeof(__nv_bfloat16) * gbf_n)) != MPDG_OK ||
      (rc = ualloc(u, (void **)&u->zero_bias, sizeof(float) * 64)) != MPDG_OK)
    return fail_free(rc);
  cudaMemset(u->zero_bias, 0, sizeof(float) * 64);
  {
    const char *e = getenv("MPDG_UNET_TC");
    u->use_tc = !(e && e[0] == '0');
    const char *eb = getenv("MPDG_UNET_TC_BWD");
    u->use_tc_bwd = !(eb && eb[0] == '0');
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&u->sm_count, cudaDevAttrMultiProcessorCount, dev);
  }
  // He-uniform initialisation from a counter hash; output layer scaled by 0.1
  std::vector<float> h(u->n_params, 0.f);
  for (int l = 0; l < 15; ++l) {
    const double bound = std::sqrt(6.0 / (27.0 * kCi[l])) * (l == OUT ? 0.1 : 1.0);
    for (int64_t i = 0; i < (int64_t)kCi[l] * kCo[l] * 27; ++i) {
      const uint64_t r = mix(seed * 0x2545F4914F6CDD1DULL + (uint64_t)(u->L[l].woff + i));
      h[u->L[l].woff + i] = (float)(bound * (2.0 * ((r >> 11) * (1.0 / 9007199254740992.0)) - 1.0));
    }
  }
  cudaMemcpy(u->p, h.data(), sizeof(float) * u->n_params, cudaMemcpyHostToDevice);
  cudaMemset(u->m, 0, sizeof(float) * u->n_params);
  cudaMemset(u->v, 0, sizeof(float) * u->n_params);
  cudaMemset(u->counter, 0, sizeof(unsigned) * 4);
  k_f32_to_bf16<<<grid1d(u->n_params), 256>>>(u->n_params, u->p, u->pb);
  if (cudaDeviceSynchronize() != cudaSuccess) return fail_free(nn_fail(MPDG_ERR_CUDA, "unet init"));
  *out = u;
  return MPDG_OK;
}

extern "C" int mpdg_unet_destroy(mpdg_unet *u)
{
  if (!u) return MPDG_OK;
  if (u->stream) cudaStreamSynchronize(u->stream);
  for (void *p : u->owned) cudaFree(p);
  if (u->tc_err_host) cudaFreeHost(u->tc_err_host);
  delete u;
  return MPDG_OK;
}

extern "C" int mpdg_unet_set_stream(mpdg_unet *u, void *stream)
{
  if (!u) return nn_fail(MPDG_ERR_INVALID_ARGUMENT, "null network");
  u->stream = (cudaStream_t)stream;
  return MPDG_OK;
}

extern "C" int mpdg_unet_dims(const mpdg_unet *u, int dims[3])
{
  if (!u || !dims) return nn_fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  dims[0] = u->g[0].nx;
  dims[1] = u->g[0].ny;
  dims[2] = u->g[0].nz;
  return MPDG_OK;
}

extern "C" int mpdg_unet_n_params(const mpdg_unet *u, int64_t *n)
{
  if (!u || !n) return nn_fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  *n = u->n_params;
  return MPDG_OK;
}

extern "C" int mpdg_unet_get_params(mpdg_unet *u, float *dst)
{
  if (!u || !dst) return nn_fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  NNCU(cudaMemcpyAsync(dst, u->p, sizeof(float) * u->n_params, cudaMemcpyDeviceToDevice, u->stream));
  return MPDG_OK;
}

extern "C" int mpdg_unet_set_params(mpdg_unet *u, const float *src)
{
  if (!u || !src) return nn_fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  NNCU(cudaMemcpyAsync(u->p, src, sizeof(float) * u->n_params, cudaMemcpyDeviceToDevice, u->stream));
  k_f32_to_bf16<<<grid1d(u->n_params), 256, 0, u->stream>>>(u->n_params, u->p, u->pb);
  NNCU(cudaGetLastError());
  u->wpk_dirty = true;
  return MPDG_OK;
}

// input: 3 x n0 FP32 (device), output: n0 FP32 (device)
extern "C" int mpdg_unet_forward(mpdg_unet *u, const float *input, float *output)
{
  if (!u || !input) return nn_fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  NNTRY(check_tc_err(u));  // raised by an earlier forward's convolutions
  const int64_t n0 = u->g[0].n();
  k_f32_to_chunked<<<grid1d(8 * n0), 256, 0, u->stream>>>(n0, 3, input, u->x0);
  NNCU(cudaGetLastError());
  NNTRY(forward(u));
  if (output) NNCU(cudaMemcpyAsync(output, u->y, sizeof(float) * n0, cudaMemcpyDeviceToDevice, u->stream));
  return MPDG_OK;
}

// gradient of sum(grad_output * y) w.r.t. the parameters, written to grad_params
// (device, n_params FP32); needs a preceding forward on the same input
extern "C" int mpdg_unet_backward(mpdg_unet *u, const float *grad_output, float *grad_params)
{
  if (!u || !grad_output) return nn_fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  NNTRY(backward(u, grad_output));
  if (grad_params)
    NNCU(cudaMemcpyAsync(grad_params, u->grad, sizeof(float) * u->n_params, cudaMemcpyDeviceToDevice, u->stream));
  return MPDG_OK;
}

// one Adam step on the MSE between the output and target; loss returned on the host
extern "C" int mpdg_unet_train_step(mpdg_unet *u, const float *input, const float *target, float lr,
                                    double *loss)
{
  if (!u || !input || !target) return nn_fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  const int64_t n0 = u->g[0].n();
  u->training = true;
  const int frc = mpdg_unet_forward(u, input, nullptr);
  u->training = false;
  NNTRY(frc);
  float *gy = u->gC;  // reuse scratch for dL/dy (copied before backward overwrites gC)
  k_mse<<<grid1d(n0), 256, 0, u->stream>>>(n0, u->y, target, gy, u->partials, u->counter, u->lossd);
  NNCU(cudaGetLastError());
  float *gy2 = u->gE0;  // gE0 is first written after the output layer's gradients are taken
  NNCU(cudaMemcpyAsync(u->y, gy, sizeof(float) * n0, cudaMemcpyDeviceToDevice, u->stream));
  (void)gy2;
  NNTRY(backward(u, u->y));
  ++u->step;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)u->step), c2 = 1.f - powf(b2, (float)u->step);
  k_adam<<<grid1d(u->n_params), 256, 0, u->stream>>>(u->n_params, u->p, u->grad, u->m, u->v, lr, b1,
                                                      b2, 1e-8f, c1, c2, u->pb);
  NNCU(cudaGetLastError());
  u->wpk_dirty = true;
  if (loss) {
    double l = 0.0;
    NNCU(cudaMemcpyAsync(&l, u->lossd, sizeof(double), cudaMemcpyDeviceToHost, u->stream));
    NNCU(cudaStreamSynchronize(u->stream));
    *loss = l;
    NNTRY(check_tc_err(u));
  }
  return MPDG_OK;
}

// MSE of the current output against target (after forward), on the host
extern "C" int mpdg_unet_loss(mpdg_unet *u, const float *target, double *loss)
{
  if (!u || !target || !loss) return nn_fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  const int64_t n0 = u->g[0].n();
  k_mse<<<grid1d(n0), 256, 0, u->stream>>>(n0, u->y, target, nullptr, u->partials, u->counter, u->lossd);
  NNCU(cudaGetLastError());
  NNCU(cudaMemcpyAsync(loss, u->lossd, sizeof(double), cudaMemcpyDeviceToHost, u->stream));
  NNCU(cudaStreamSynchronize(u->stream));
  return MPDG_OK;
}
