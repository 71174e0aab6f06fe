// Forward 3x3x3 convolution of the guess network on the 5th-generation tensor
// cores (tcgen05, sm_100a): implicit GEMM with M = 128 output points, N = the
// output channels (padded to 16/32/48/64), K = 27 taps x the input channels.
//
// No im2col: a CTA stages the halo of its 8 x 16 x 1 output tile for all input
// channels in shared memory as 8-channel chunks, [chunk][hz][hy][hx] x 16 bytes (one
// 16-byte load per point and chunk from the channel-chunked activations),
// which is the canonical no-swizzle K-major UMMA layout for ANY tap shift: the 8
// rows of a core matrix are 8 consecutive x points (16 bytes apart), row groups
// are the 16 y rows (stride 16 * 10 bytes), the two K halves of a 16-channel
// step are consecutive chunks. So the A descriptor of tap (dx, dy, dz) just
// points at halo point (dx, dy, dz), and a tile is 27 x ceil(Ci / 16) MMAs of
// 128 x N x 16 issued by one thread into one FP32 accumulator in tensor memory.
// The weights are packed once per update into the matching B layout
// [tap][16-channel group][K half][Cout][8] and kept in shared memory for the
// whole persistent CTA when they fit (else streamed 9 taps at a time). The
// epilogue reads the accumulator with tcgen05.ld (one output point per thread),
// adds bias and the skip input, applies ReLU and stores the BF16 activations channel-chunked
// ([C/8][points][8], one 16-byte vector per point and chunk; FP32 outputs planar [C][points]).
//
// Waits on the MMA-completion barrier are bounded; on expiry the kernel raises
// *err, skips its stores, frees its tensor memory and returns.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace nn_tc {

constexpr int TCX = 8, TCY = 16;  // output tile (M = 128 rows, row = x + 8 y)
constexpr int THX = TCX + 2, THY = TCY + 2, THZ = 3, THP = THX * THY * THZ;  // 540 halo points
constexpr int kThreads = 128;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// shared-memory matrix descriptor: no swizzle, K-major; lbo = bytes between the two
// 8-element K halves of a 16-element step, sbo = bytes between 8-row groups
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: BF16 x BF16 -> FP32, A and B K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t idesc_bf16_m128(int n)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((128u >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
  for (int it = 0; it < (1 << 22); ++it) {
    uint32_t done;
    asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
    if (done) return true;
  }
  return false;
}

struct ConvArgs {
  int nx, ny, nz;
  int ci, co;
  int cg;              // 16-channel groups of the input
  int taps_per_stage;  // 27: weights resident in shared memory; 9: streamed
  int up;              // input is the coarse grid (sx, sy, sz), read nearest-neighbour
  int sx, sy, sz;
  const __nv_bfloat16 *in;  // [ci][points] (of the coarse grid when up)
  const uint4 *wp;          // packed weights [27][cg][2][npad] x 8 BF16
  const float *bias;        // [co]
  const __nv_bfloat16 *add; // [co][points] (skip input added before ReLU) or null
  void *out;                // [co][points], BF16 or FP32
  int *err;
};

__host__ __device__ constexpr int tmem_cols(int npad) { return npad <= 32 ? 32 : 64; }
__host__ __device__ inline size_t smem_bytes(int cg, int npad, int taps)
{
  return (size_t)16 * ((size_t)2 * cg * THP + (size_t)taps * cg * 2 * npad);
}

template <int NPAD, bool RELU, bool ADD, typename TO>
__global__ void __launch_bounds__(kThreads, 1) k_conv3d_tc(ConvArgs a)
{
  static_assert(NPAD % 16 == 0 && NPAD >= 16 && NPAD <= 64, "N = 16, 32, 48, 64");
  static_assert(!(ADD && sizeof(TO) == 4), "the skip input is added to BF16 activations only");
  constexpr uint32_t TCOLS = tmem_cols(NPAD);
  constexpr uint32_t IDESC = idesc_bf16_m128(NPAD);
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nchunk = 2 * a.cg;
  uint4 *halo = reinterpret_cast<uint4 *>(smem);  // [nchunk][THP]
  uint4 *wsm = halo + nchunk * THP;               // [taps][cg][2][NPAD]
  const int64_t np = (int64_t)a.nx * a.ny * a.nz;
  const int tiles_x = (a.nx + TCX - 1) / TCX, tiles_y = (a.ny + TCY - 1) / TCY;
  const int64_t n_tiles = (int64_t)tiles_x * tiles_y * a.nz;
  const uint32_t bar = smem_u32(&mbar);

  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                   smem_u32(&tmem_slot)),
                 "r"(TCOLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;

  const int wstage = a.taps_per_stage * a.cg * 2 * NPAD;  // uint4 per weight stage
  const bool resident = a.taps_per_stage == 27;
  if (resident)
    for (int i = tid; i < wstage; i += kThreads) wsm[i] = a.wp[i];
  const uint32_t halo_a = smem_u32(halo), w_a = smem_u32(wsm);
  // activations are channel-chunked, [C/8][points][8] BF16: one 16-byte vector per point and
  // 8-channel chunk (chunks past ceil(Ci/8) are zero)
  const uint4 *src = reinterpret_cast<const uint4 *>(a.in);
  const int64_t snp = a.up ? (int64_t)a.sx * a.sy * a.sz : np;  // input plane size
  uint32_t phase = 0;
  bool ok = true;

  for (int64_t tile = blockIdx.x; tile < n_tiles && ok; tile += gridDim.x) {
    const int bx = (int)(tile % tiles_x) * TCX;
    const int by = (int)((tile / tiles_x) % tiles_y) * TCY;
    const int bz = (int)(tile / ((int64_t)tiles_x * tiles_y));
    // halo of all input channels, zero outside the grid and above ci; UNROLL items
    // per thread and pass so that 8 * UNROLL independent loads are in flight
    constexpr int UNROLL = 4;
    const int nitems = nchunk * THP;
    for (int base = 0; base < nitems; base += UNROLL * kThreads) {
      uint32_t w4[UNROLL][4];
#pragma unroll
      for (int u = 0; u < UNROLL; ++u) {
        w4[u][0] = w4[u][1] = w4[u][2] = w4[u][3] = 0u;
        const int i = base + u * kThreads + tid;
        const int c = i / THP, hp = i - c * THP;
        const int hx = hp % THX, hy = (hp / THX) % THY, hz = hp / (THX * THY);
        const int gx = bx + hx - 1, gy = by + hy - 1, gz = bz + hz - 1;
        if (i < nitems && 8 * c < a.ci && gx >= 0 && gx < a.nx && gy >= 0 && gy < a.ny && gz >= 0 &&
            gz < a.nz) {
          // the input lives on the grid itself or, with a.up, on the coarse grid it is
          // nearest-neighbour upsampled from
          const int64_t gp = a.up ? (gx >> 1) + (int64_t)a.sx * ((gy >> 1) + (int64_t)a.sy * (gz >> 1))
                                  : gx + (int64_t)a.nx * (gy + (int64_t)a.ny * gz);
          const uint4 v = __ldg(src + (int64_t)c * snp + gp);
          w4[u][0] = v.x;
          w4[u][1] = v.y;
          w4[u][2] = v.z;
          w4[u][3] = v.w;
        }
      }
#pragma unroll
      for (int u = 0; u < UNROLL; ++u) {
        const int i = base + u * kThreads + tid;
        if (i < nitems) halo[i] = make_uint4(w4[u][0], w4[u][1], w4[u][2], w4[u][3]);
      }
    }
    for (int t0 = 0; t0 < 27; t0 += a.taps_per_stage) {
      if (!resident) {
        const uint4 *ws = a.wp + (int64_t)t0 * a.cg * 2 * NPAD;
        for (int i = tid; i < wstage; i += kThreads) wsm[i] = ws[i];
      }
      // generic-proxy shared stores -> visible to the tensor core (async proxy)
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (tid == 0) {
        for (int tl = 0; tl < a.taps_per_stage; ++tl) {
          const int tap = t0 + tl;
          const int dx = tap % 3, dy = (tap / 3) % 3, dz = tap / 9;
          for (int g = 0; g < a.cg; ++g) {
            const uint32_t aaddr =
              halo_a + 16u * (uint32_t)(2 * g * THP + dx + THX * (dy + THY * dz));
            const uint32_t baddr = w_a + 16u * (uint32_t)((tl * a.cg + g) * 2 * NPAD);
            const uint64_t ad = umma_desc(aaddr, 16u * THP, 16u * THX);
            const uint64_t bd = umma_desc(baddr, 16u * NPAD, 128u);
            const uint32_t accumulate = (tap | g) != 0 ? 1u : 0u;
            asm volatile(
              "{\n\t.reg .pred p;\n\t"
              "setp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
              ::"r"(tmem), "l"(ad), "l"(bd), "r"(IDESC), "r"(accumulate)
              : "memory");
          }
        }
        asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
          : "memory");
      }
      // the MMAs read the halo and the weight stage: wait before either is rewritten
      const bool done = mbar_wait(bar, phase);
      phase ^= 1u;
      ok = __syncthreads_and(done) != 0;
      if (!ok) break;
    }
    if (!ok) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = 32 * warp + lane;  // accumulator lane = tile row
    const int x = bx + (row & 7), y = by + (row >> 3);
    const bool inside = x < a.nx && y < a.ny;
    const int64_t p = x + (int64_t)a.nx * (y + (int64_t)a.ny * bz);
#pragma unroll
    for (int c0 = 0; c0 < NPAD; c0 += 8) {
      uint32_t r[8];
      asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7])
        : "r"(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (inside && c0 < a.co) {
        if constexpr (sizeof(TO) == 4) {
          // FP32 outputs (the network's output, data gradients) are planar [C][points]
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            const int co = c0 + j;
            if (co < a.co) {
              float v = __uint_as_float(r[j]) + a.bias[co];
              if (RELU) v = fmaxf(v, 0.f);
              reinterpret_cast<float *>(a.out)[(int64_t)co * np + p] = v;
            }
          }
        } else {
          // BF16 activations: the chunk's 8 channels as one 16-byte vector (zero past Co)
          uint4 sk = make_uint4(0u, 0u, 0u, 0u);
          if (ADD) sk = __ldg(reinterpret_cast<const uint4 *>(a.add) + (int64_t)(c0 >> 3) * np + p);
          const __nv_bfloat16 *skh = reinterpret_cast<const __nv_bfloat16 *>(&sk);
          uint32_t o4[4];
#pragma unroll
          for (int j = 0; j < 8; j += 2) {
            float v[2];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int co = c0 + j + e;
              v[e] = 0.f;
              if (co < a.co) {
                v[e] = __uint_as_float(r[j + e]) + a.bias[co];
                if (ADD) v[e] += __bfloat162float(skh[j + e]);
                if (RELU) v[e] = fmaxf(v[e], 0.f);
              }
            }
            const __nv_bfloat162 h2 = __floats2bfloat162_rn(v[0], v[1]);
            o4[j >> 1] = *reinterpret_cast<const uint32_t *>(&h2);
          }
          reinterpret_cast<uint4 *>(a.out)[(int64_t)(c0 >> 3) * np + p] =
            make_uint4(o4[0], o4[1], o4[2], o4[3]);
        }
      }
    }
    // every accumulator read is done before the next tile's first MMA overwrites it
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
  }
  if (!ok && tid == 0) *(volatile int *)a.err = 1;  // page-locked host memory: a plain store
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS)
                 : "memory");
}

// w[co][ci][27] (BF16) -> [27][cg][2][npad] x 8 BF16, zero-padded channels
__global__ void k_pack_weights(int ci, int co, int cg, int npad, const __nv_bfloat16 *__restrict__ w,
                               uint4 *wp)
{
  const int64_t n = (int64_t)27 * cg * 2 * npad;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int o = (int)(i % npad);
    const int half = (int)((i / npad) % 2);
    const int g = (int)((i / (2 * npad)) % cg);
    const int tap = (int)(i / ((int64_t)2 * npad * cg));
    const unsigned short *ws = reinterpret_cast<const unsigned short *>(w);
    uint32_t v4[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int c = 16 * g + 8 * half + e;
      const uint32_t v = (o < co && c < ci) ? (uint32_t)ws[((int64_t)o * ci + c) * 27 + tap] : 0u;
      v4[e >> 1] |= v << (16 * (e & 1));
    }
    wp[i] = make_uint4(v4[0], v4[1], v4[2], v4[3]);
  }
}

// The data gradient of a convolution is the convolution of the output gradient with the
// flipped, channel-transposed weights: gin[c] = sum_o sum_tap w[o][c][tap] gout[o](x - shift(tap))
// = conv(gout, w')[c] with w'[c][o][26 - tap] = w[o][c][tap]. Packs w' (ci' = co, co' = ci) in the
// layout of k_pack_weights.
__global__ void k_pack_weights_t(int ci, int co, int cg, int npad, const __nv_bfloat16 *__restrict__ w,
                                 uint4 *wp)
{
  // cg = 16-channel groups of co (the transposed input), npad = ci padded (its output)
  const int64_t n = (int64_t)27 * cg * 2 * npad;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int c = (int)(i % npad);  // output channel of the transposed convolution
    const int half = (int)((i / npad) % 2);
    const int g = (int)((i / (2 * npad)) % cg);
    const int tap = (int)(i / ((int64_t)2 * npad * cg));
    const unsigned short *ws = reinterpret_cast<const unsigned short *>(w);
    uint32_t v4[4] = {0u, 0u, 0u, 0u};
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      const int o = 16 * g + 8 * half + e;  // input channel of the transposed convolution
      const uint32_t v = (c < ci && o < co) ? (uint32_t)ws[((int64_t)o * ci + c) * 27 + (26 - tap)] : 0u;
      v4[e >> 1] |= v << (16 * (e & 1));
    }
    wp[i] = make_uint4(v4[0], v4[1], v4[2], v4[3]);
  }
}

}  // namespace nn_tc
