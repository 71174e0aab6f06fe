// FP32 Picard operator of the multigrid fine level on the 5th-generation tensor cores
// (tcgen05, kind::tf32), FE_Q(3) on a uniform box mesh.
//
// The operator is v = G^T diag(f) G u per cell, with G the 256 x 64 matrix that maps the 64
// nodal values of a cell to its reference gradients and values at the 64 Gauss points,
//   rows j = c * 64 + q, c = 0..2: d/dxi_c (Sd x S x S, S x Sd x S, S x S x Sd), c = 3: S x S x S,
// (S: GLL shape values at the Gauss points, Sd: their derivatives) and f the point factors:
// k(q) w_q det(J) / h_c^2 for the gradients, rho c_p / dt w_q det(J) for the values. For a brick
// of 8 x 4 x 4 = 128 cells this is two GEMMs with M = 128 cells:
//   D1 (128 x 256) = U (128 x 64) * G^T          (A = U in tensor memory, B = G in shared memory)
//   V  (128 x 64)  = (f o D1) (128 x 256) * G    (A = the scaled D1 in tensor memory)
// G^T and G are stored once per CTA in shared memory, both K-major in the no-swizzle canonical
// UMMA layout (picard_tc_layout.hpp; 64 KB each).
//
// Tensor memory: 256 columns per brick pipeline, U [0, 64), D1 half [64, 192), V [192, 256).
// D1 is formed in two halves (x, y gradients; z gradient and values) so that it fits:
//   GEMM1a -> x, y fluxes in place -> GEMM2a (V =) -> GEMM1b -> z flux, mass -> GEMM2b (V +=).
// A CTA runs two such pipelines (warpgroups, one brick each, named barriers), so the memory
// phases of one overlap the MMAs of the other, sharing the two matrices.
// Thread t owns cell t of the brick (accumulator lane t): it gathers its cell's 64 nodal values
// from src (constrained DoFs read as zero; the next brick's rows and conductivities are
// prefetched into L2 while this one computes), writes its U row, scales its D1 row, reads its V
// row and adds it into dst with global reductions (constrained rows skipped), as the CUDA-core
// kernel scatters. Operands are rounded to TF32 (cvt.rna); accumulation is FP32.
//
// Waits on the MMA-completion barrier are bounded; on expiry the kernel raises *err (and stops
// the solver state, when given), frees its tensor memory and returns.
#pragma once

#include <stdint.h>

#include "cell_kernels.cuh"
#include "picard_tc_layout.hpp"

namespace mpdg {
namespace optc {

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t desc_noswizzle(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// bounded wait on the MMA-completion barrier; each try suspends the thread for up to 2 us (a
// hint to the hardware) instead of spinning, so waiting warps leave the issue slots to the other
// brick pipeline; at most 2^20 tries
__device__ __forceinline__ bool wait_bar(uint32_t bar, uint32_t parity)
{
  for (int it = 0; it < (1 << 20); ++it) {
    uint32_t done;
    asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(bar), "r"(parity), "r"(2000u)
      : "memory");
    if (done) return true;
  }
  return false;
}

// D (tensor memory) [+]= A (tensor memory, K = 8 columns) * B (shared-memory descriptor)
__device__ __forceinline__ void mma_tf32(uint32_t d, uint32_t a, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
  asm volatile(
    "{\n\t.reg .pred p;\n\t"
    "setp.ne.b32 p, %4, 0;\n\t"
    "tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n\t}"
    ::"r"(d), "r"(a), "l"(bdesc), "r"(idesc), "r"(accumulate)
    : "memory");
}

__device__ __forceinline__ void commit(uint32_t bar)
{
  asm volatile(
    "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
    : "memory");
}

// 16 columns of this thread's lane; the registers are valid after tmem_wait_ld()
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16])
{
  asm volatile(
    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
    "%12, %13, %14, %15}, [%16];"
    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
      "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
      "=r"(r[14]), "=r"(r[15])
    : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld()
{
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// FP32 -> TF32, round to nearest (ties away), one instruction
__device__ __forceinline__ float to_tf32(float x)
{
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float (&v)[16])
{
  asm volatile(
    "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, "
    "%12, %13, %14, %15, %16};" ::"r"(taddr),
    "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
    "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
    "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
    "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
    "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
    "r"(__float_as_uint(v[15]))
    : "memory");
}

__device__ __forceinline__ void before_sync()
{
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void after_sync()
{
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// named barrier of one warpgroup (ids 1, 2; 0 is __syncthreads)
__device__ __forceinline__ void group_sync(int g)
{
  asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory");
}
__device__ __forceinline__ bool group_and(int g, bool v)
{
  uint32_t r;
  asm volatile(
    "{\n\t.reg .pred p, q;\n\t"
    "setp.ne.u32 p, %1, 0;\n\t"
    "bar.red.and.pred q, %2, 128, p;\n\t"
    "selp.u32 %0, 1, 0, q;\n\t}"
    : "=r"(r)
    : "r"((uint32_t)v), "r"(1 + g)
    : "memory");
  return r != 0;
}

// a cell that touches a Dirichlet face (its gather masks and its scatter skips those rows)
__device__ __forceinline__ bool cell_on_dirichlet(const MeshDims &d, int cx, int cy, int cz)
{
  return ((d.dmask & 1) && cx == 0) || ((d.dmask & 2) && cx == d.m[0] - 1) ||
         ((d.dmask & 4) && cy == 0) || ((d.dmask & 8) && cy == d.m[1] - 1) ||
         ((d.dmask & 16) && cz == 0) || ((d.dmask & 32) && cz == d.m[2] - 1);
}

}  // namespace optc

// a.dst += A_picard a.src (constrained rows skipped, constrained columns read as zero);
// LAW 3 (conductivity field a.kq), uniform box, FE_Q(3) (n = 4); requires a.fin == FIN_NONE.
// Two warpgroups per CTA, each an independent brick pipeline with its own 256 tensor-memory
// columns and barrier; they share G^T and G in shared memory.
template <int n>
__global__ void __launch_bounds__(optc::kThreads, 1)
  k_vmult_picard_tc(CellArgs<float> a, const float4 *__restrict__ gmat, int *err)
{
  static_assert(n == 4, "FE_Q(3) only");
  using namespace optc;
  if (a.st && a.st->done) return;
  extern __shared__ __align__(128) unsigned char smem_tc[];
  __shared__ __align__(8) uint64_t mbar[kGroups];
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, grp = tid >> 7, lt = tid & 127, warp = tid >> 5;
  const int wi = warp & 3;
  const MeshDims &d = a.d;
  const int nbx = (d.m[0] + kBX - 1) / kBX, nby = (d.m[1] + kBY - 1) / kBY;
  const int nbz = (d.m[2] + kBZ - 1) / kBZ;
  const int64_t n_bricks = (int64_t)nbx * nby * nbz;
  const int64_t sy = d.nd[0], sz = (int64_t)d.nd[0] * d.nd[1];
  const uint32_t bar = smem_addr(&mbar[grp]);

  if (lt == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_addr(&tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  for (int i = tid; i < 2 * kGFloats / 4; i += kThreads)
    reinterpret_cast<float4 *>(smem_tc)[i] = gmat[i];
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  before_sync();
  __syncthreads();
  after_sync();
  const uint32_t tbase = tmem_slot + kColsPerGroup * grp;
  const uint32_t lane_off = (uint32_t)(32 * wi) << 16;
  const uint32_t tU = tbase, tD1 = tbase + 64, tV = tbase + 192;
  const uint32_t g1_a = smem_addr(smem_tc), g2_a = smem_addr(smem_tc + kGBytes);
  constexpr uint32_t ID1 = idesc_tf32_m128(128), ID2 = idesc_tf32_m128(64);

  // this thread's cell within a brick
  const int tx = lt & 7, ty = (lt >> 3) & 3, tz = lt >> 5;
  const float cmass = a.m.idt * (a.m.rho_l * a.m.cp_l) * a.g.detJ;
  const float cx0 = a.g.Gd[0], cy0 = a.g.Gd[1], cz0 = a.g.Gd[2];
  float w1[4];
#pragma unroll
  for (int e = 0; e < 4; ++e) w1[e] = cw<float>(w_off(4) + e);
  uint32_t phase = 0;
  bool ok = true;
  const int64_t b_step = (int64_t)gridDim.x * kGroups;

  for (int64_t b = (int64_t)blockIdx.x * kGroups + grp; b < n_bricks && ok; b += b_step) {
    const int bx = (int)(b % nbx), by = (int)((b / nbx) % nby);
    const int bz = (int)(b / ((int64_t)nbx * nby));
    const int cx = bx * kBX + tx, cy = by * kBY + ty, cz = bz * kBZ + tz;
    const bool active = cx < d.m[0] && cy < d.m[1] && cz < d.m[2];
    const bool masked = active && cell_on_dirichlet(d, cx, cy, cz);
    const int64_t cell = active ? cx + (int64_t)d.m[0] * (cy + (int64_t)d.m[1] * cz) : 0;
    const int64_t node0 = 3 * cx + sy * (3 * cy) + sz * (3 * cz);  // the cell's first DoF

    // the next brick's rows and conductivities into L2 while this one computes
    if (b + b_step < n_bricks) {
      const int64_t nb = b + b_step;
      const int ncx = (int)(nb % nbx) * kBX + tx, ncy = (int)((nb / nbx) % nby) * kBY + ty;
      const int ncz = (int)(nb / ((int64_t)nbx * nby)) * kBZ + tz;
      if (ncx < d.m[0] && ncy < d.m[1] && ncz < d.m[2]) {
        const float *kn = a.kq + 64 * (ncx + (int64_t)d.m[0] * (ncy + (int64_t)d.m[1] * ncz));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(kn));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(kn + 32));
        if (tx == 0 || tx == 4) {  // 4 cells' x-extent (13 nodes) per 64-byte line pair
          const float *np = a.src + 3 * ncx + sy * (3 * ncy) + sz * (3 * ncz);
          const bool far = 3 * ncx + 12 < d.nd[0];  // the row's 13th node exists
#pragma unroll
          for (int r = 0; r < 16; ++r) {
            const float *rp = np + sy * (r & 3) + sz * (r >> 2);
            asm volatile("prefetch.global.L2 [%0];" ::"l"(rp));
            if (far) asm volatile("prefetch.global.L2 [%0];" ::"l"(rp + 12));
          }
        }
      }
    }

    // conductivity x quadrature weight at the cell's points (q = qx + 4 (qy + 4 qz))
    float kw[64];
    {
      const float4 *kp = reinterpret_cast<const float4 *>(a.kq + cell * 64);
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (active) v = __ldg(kp + r);
        const int q = 4 * r;
        const float wyz = w1[(q >> 2) & 3] * w1[q >> 4];
        kw[q + 0] = v.x * (w1[0] * wyz);
        kw[q + 1] = v.y * (w1[1] * wyz);
        kw[q + 2] = v.z * (w1[2] * wyz);
        kw[q + 3] = v.w * (w1[3] * wyz);
      }
    }
    // U row (DoF i = ix + 4 (iy + 4 iz)) gathered from src into tensor memory
#pragma unroll
    for (int iz = 0; iz < 4; ++iz) {
      float r[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int64_t off = node0 + (e & 3) + sy * (e >> 2) + sz * iz;
        float v = 0.f;
        if (active) v = __ldg(a.src + off);
        if (masked && constrained(d, 3 * cx + (e & 3), 3 * cy + (e >> 2), 3 * cz + iz)) v = 0.f;
        r[e] = to_tf32(v);
      }
      tmem_st16(tU + lane_off + 16 * iz, r);
    }
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    before_sync();
    group_sync(grp);
    after_sync();
    if (lt == 0) {  // GEMM1a: x and y gradients (rows 0..127 of G^T)
#pragma unroll
      for (int kk = 0; kk < 8; ++kk)
        mma_tf32(tD1, tU + 8 * kk, desc_noswizzle(g1_a + 256u * kk, 128u, 2048u), ID1, kk > 0);
      commit(bar);
    }
    ok = group_and(grp, wait_bar(bar, phase));
    phase ^= 1u;
    if (!ok) break;
    after_sync();
    // x and y fluxes in place
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      uint32_t rx[16], ry[16];
      tmem_ld16(tD1 + lane_off + 16 * c, rx);
      tmem_ld16(tD1 + lane_off + 64 + 16 * c, ry);
      tmem_wait_ld();
      float gx[16], gy[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        gx[e] = to_tf32(kw[16 * c + e] * (cx0 * __uint_as_float(rx[e])));
        gy[e] = to_tf32(kw[16 * c + e] * (cy0 * __uint_as_float(ry[e])));
      }
      tmem_st16(tD1 + lane_off + 16 * c, gx);
      tmem_st16(tD1 + lane_off + 64 + 16 * c, gy);
    }
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    before_sync();
    group_sync(grp);
    after_sync();
    if (lt == 0) {  // GEMM2a: V = F_xy G_xy (K steps j = 0..127 of G)
#pragma unroll
      for (int kk = 0; kk < 16; ++kk)
        mma_tf32(tV, tD1 + 8 * kk, desc_noswizzle(g2_a + 256u * kk, 128u, 8192u), ID2, kk > 0);
      commit(bar);
    }
    ok = group_and(grp, wait_bar(bar, phase));
    phase ^= 1u;
    if (!ok) break;
    after_sync();
    if (lt == 0) {  // GEMM1b: z gradient and values (rows 128..255), over the consumed D1 half
#pragma unroll
      for (int kk = 0; kk < 8; ++kk)
        mma_tf32(tD1, tU + 8 * kk, desc_noswizzle(g1_a + 32768u + 256u * kk, 128u, 2048u), ID1,
                 kk > 0);
      commit(bar);
    }
    ok = group_and(grp, wait_bar(bar, phase));
    phase ^= 1u;
    if (!ok) break;
    after_sync();
    // z flux and the mass term in place
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      uint32_t rz[16], rv[16];
      tmem_ld16(tD1 + lane_off + 16 * c, rz);
      tmem_ld16(tD1 + lane_off + 64 + 16 * c, rv);
      tmem_wait_ld();
      float gz[16], gv[16];
#pragma unroll
      for (int e = 0; e < 16; ++e) {
        const int q = 16 * c + e;
        gz[e] = to_tf32(kw[q] * (cz0 * __uint_as_float(rz[e])));
        gv[e] = to_tf32((cmass * (w1[q & 3] * w1[(q >> 2) & 3] * w1[q >> 4])) *
                        __uint_as_float(rv[e]));
      }
      tmem_st16(tD1 + lane_off + 16 * c, gz);
      tmem_st16(tD1 + lane_off + 64 + 16 * c, gv);
    }
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
    before_sync();
    group_sync(grp);
    after_sync();
    if (lt == 0) {  // GEMM2b: V += F_zv G_zv (K steps j = 128..255 of G)
#pragma unroll
      for (int kk = 0; kk < 16; ++kk)
        mma_tf32(tV, tD1 + 8 * kk, desc_noswizzle(g2_a + 256u * (16 + kk), 128u, 8192u), ID2, 1u);
      commit(bar);
    }
    ok = group_and(grp, wait_bar(bar, phase));
    phase ^= 1u;
    if (!ok) break;
    after_sync();
    // scatter the cell's V row into dst (reductions; constrained rows skipped)
#pragma unroll
    for (int iz = 0; iz < 4; ++iz) {
      uint32_t v[16];
      tmem_ld16(tV + lane_off + 16 * iz, v);
      tmem_wait_ld();
      if (active) {
#pragma unroll
        for (int e = 0; e < 16; ++e) {
          if (masked && constrained(d, 3 * cx + (e & 3), 3 * cy + (e >> 2), 3 * cz + iz)) continue;
          atomicAdd(a.dst + node0 + (e & 3) + sy * (e >> 2) + sz * iz, __uint_as_float(v[e]));
        }
      }
    }
    // every V read is done before the next brick's GEMM2a overwrites it
    before_sync();
    group_sync(grp);
    after_sync();
  }
  if (!ok && lt == 0) {
    *(volatile int *)err = 1;  // page-locked host memory: a plain store
    if (a.st) {
      a.st->status = MPDG_ERR_CUDA;
      a.st->done = 2;
    }
  }
  before_sync();
  __syncthreads();
  after_sync();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_slot),
                 "r"(kTmemCols)
                 : "memory");
}

}  // namespace mpdg
