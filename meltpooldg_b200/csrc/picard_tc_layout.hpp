// Layout constants and the G matrices of the tensor-core Picard operator (cell_kernels_tc.cuh),
// shared by the kernel and the host code that builds them (CUDA translation units only).
#pragma once

#include <stdint.h>

#include <cstring>

#include "fe_tables.hpp"

namespace mpdg {
namespace optc {

constexpr int kBX = 8, kBY = 4, kBZ = 4;                                  // cells per brick
constexpr int kGroups = 2;                  // warpgroups per CTA, one brick each
constexpr int kThreads = 128 * kGroups;
constexpr uint32_t kColsPerGroup = 256;    // tensor-memory columns of one warpgroup
constexpr uint32_t kTmemCols = kColsPerGroup * kGroups;
constexpr int kGFloats = 256 * 64;         // one matrix: G^T (first GEMM) or G (second)
constexpr size_t kGBytes = sizeof(float) * kGFloats;  // 65536
constexpr size_t kSmem = 2 * kGBytes;  // G^T and G
static_assert(kSmem <= 227 * 1024, "shared-memory plan");

// G^T for the first GEMM (N = 256 rows j, K = 64 columns i) and G for the second (N = 64 rows
// i, K = 256 columns j), both in the no-swizzle K-major canonical layout (8-row core matrices
// of 16 B rows; LBO = 128 B between 4-element K chunks; SBO between 8-row groups: 2048 B for
// G^T, 8192 B for G)
__host__ __device__ constexpr int gmat_offset(int j, int i)
{
  return (j >> 3) * 512 + (i >> 2) * 32 + (j & 7) * 4 + (i & 3);
}
__host__ __device__ constexpr int gmat2_offset(int i, int j)
{
  return (i >> 3) * 2048 + (j >> 2) * 32 + (i & 7) * 4 + (j & 3);
}

// TF32 x TF32 -> FP32, M = 128, N = n, B K-major (an MN-major TF32 B operand in the
// no-swizzle layout gave zero products on this hardware, so both matrices are stored K-major)
__host__ __device__ constexpr uint32_t idesc_tf32_m128(int n)
{
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24);
}

// round to the nearest TF32 value (10 mantissa bits), ties to even; finite inputs
__host__ __device__ inline float round_tf32(float x)
{
#ifdef __CUDA_ARCH__
  uint32_t b = __float_as_uint(x);
#else
  uint32_t b;
  std::memcpy(&b, &x, 4);
#endif
  b += 0xFFFu + ((b >> 13) & 1u);
  b &= ~0x1FFFu;
#ifdef __CUDA_ARCH__
  return __uint_as_float(b);
#else
  float r;
  std::memcpy(&r, &b, 4);
  return r;
#endif
}

// G^T then G (2 x kGFloats) in the shared-memory layouts above, entries rounded to TF32
inline void build_gmat(float *g)
{
  const Tables1D t = make_tables(4);
  double S[4][4], Sd[4][4];
  for (int q = 0; q < 4; ++q)
    for (int i = 0; i < 4; ++i) {
      S[q][i] = t.A[kS][q][i];
      double s = 0.0;
      for (int m = 0; m < 4; ++m) s += t.A[kD][q][m] * t.A[kS][m][i];
      Sd[q][i] = s;
    }
  for (int c = 0; c < 4; ++c)
    for (int q = 0; q < 64; ++q)
      for (int i = 0; i < 64; ++i) {
        const int qx = q & 3, qy = (q >> 2) & 3, qz = q >> 4;
        const int ix = i & 3, iy = (i >> 2) & 3, iz = i >> 4;
        const double v = (c == 0 ? Sd[qx][ix] : S[qx][ix]) * (c == 1 ? Sd[qy][iy] : S[qy][iy]) *
                         (c == 2 ? Sd[qz][iz] : S[qz][iz]);
        const float r = round_tf32((float)v);
        g[gmat_offset(64 * c + q, i)] = r;
        g[kGFloats + gmat2_offset(i, 64 * c + q)] = r;
      }
}

}  // namespace optc
}  // namespace mpdg
