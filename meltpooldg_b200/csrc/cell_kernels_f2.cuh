// Packed-pair FP32 operator kernel (n = p + 1 <= 4), opt-in (MPDG_FP32_PACKED=1).
//
// Same register-resident plane layout as k_vmult2, but every group of n lanes
// processes TWO cells at once: cell A in the low and cell B in the high half of
// a float2. Every sweep, pointwise and layout-switch operation is then one
// packed instruction for both cells (sm_100 FFMA2 / FADD2 / FMUL2 and 64-bit
// shared-memory accesses), which halves the issue count of the FP32 kernel; the
// register and shared-memory footprint per lane equals that of the FP64 kernel.
// Cells A = 2c and B = 2c + 1 are x-neighbours in the same row whenever the row
// has an even number of cells; then the DoFs of their common face are summed in
// registers and scattered with one atomic instead of two.
//
// Supported coefficient laws: 0 (constant k), 1 (k = k0 + k1 T with its tangent),
// 3 (conductivity field at the q-points, the Picard operator of the
// preconditioner). The liquid-solid law runs on the scalar kernel.
#pragma once

#include "cell_kernels_v2.cuh"

namespace mpdg {

static __constant__ float2 c_tab_f2[kTabSize];  // c_tab_f with every entry duplicated

struct F2 {
  float2 v;
  F2() = default;
  __device__ __forceinline__ F2(float s) : v(make_float2(s, s)) {}
  __device__ __forceinline__ F2(float2 x) : v(x) {}
  __device__ __forceinline__ F2(float a, float b) : v(make_float2(a, b)) {}
};
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b)
{
  return F2(__ffma2_rn(b.v, make_float2(-1.f, -1.f), a.v));
}
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return F2(__fmul2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 fma(F2 a, F2 b, F2 c) { return F2(__ffma2_rn(a.v, b.v, c.v)); }
template <> __device__ __forceinline__ F2 ctab<F2>(int i) { return F2(c_tab_f2[i]); }

// nodal-grid offset of plane K = p cz + t of a cell, and its corner indices
__device__ __forceinline__ int64_t cell_plane_base(const MeshDims &d, int64_t cell, int t, int &I0,
                                                   int &J0, int &K)
{
  const int cx = (int)(cell % d.m[0]);
  const int cy = (int)((cell / d.m[0]) % d.m[1]);
  const int cz = (int)(cell / ((int64_t)d.m[0] * d.m[1]));
  I0 = d.p * cx;
  J0 = d.p * cy;
  K = d.p * cz + t;
  return (int64_t)d.nd[0] * (J0 + (int64_t)d.nd[1] * K) + I0;
}

template <int n>
__device__ __forceinline__ void gather_pair(const MeshDims &d, int64_t bA, int64_t bB,
                                            const PlaneMask &mA, const PlaneMask &mB, bool masked,
                                            const float *__restrict__ g, F2 (&P)[n][n], bool actA,
                                            bool actB)
{
#pragma unroll
  for (int j = 0; j < n; ++j) {
    const int64_t r = (int64_t)d.nd[0] * j;
#pragma unroll
    for (int i = 0; i < n; ++i) {
      float a = 0.f, b = 0.f;
      if (actA) {
        a = __ldg(g + bA + r + i);
        if (masked && mA.template at<n>(i, j)) a = 0.f;
      }
      if (actB) {
        b = __ldg(g + bB + r + i);
        if (masked && mB.template at<n>(i, j)) b = 0.f;
      }
      P[j][i] = F2(a, b);
    }
  }
}

template <int n, int GEO>
__device__ __forceinline__ void geo_pair(const GeoParams<float> &g, int64_t cA, int64_t cB, int qi,
                                         int qj, int qk, F2 &jxw, F2 G[6])
{
  if (GEO == 0) {
    const float w = cw<float>(w_off(n) + qi) * cw<float>(w_off(n) + qj) * cw<float>(w_off(n) + qk);
    jxw = F2(g.detJ * w);
    G[0] = F2(g.Gd[0] * w);
    G[3] = F2(g.Gd[1] * w);
    G[5] = F2(g.Gd[2] * w);
  } else {
    constexpr int npt = n * n * n;
    const int q = qi + n * (qj + n * qk);
    const float *a = g.q + cA * 7 * npt + q;
    const float *b = g.q + cB * 7 * npt + q;
    jxw = F2(__ldg(a), __ldg(b));
#pragma unroll
    for (int t = 0; t < 6; ++t) G[t] = F2(__ldg(a + (1 + t) * npt), __ldg(b + (1 + t) * npt));
  }
}

template <int GEO>
__device__ __forceinline__ void apply_G2(const F2 G[6], F2 a, F2 b, F2 c, F2 &x, F2 &y, F2 &z)
{
  if (GEO == 0) {
    x = G[0] * a;
    y = G[3] * b;
    z = G[5] * c;
  } else {
    x = fma(G[2], c, fma(G[1], b, G[0] * a));
    y = fma(G[4], c, fma(G[3], b, G[1] * a));
    z = fma(G[5], c, fma(G[4], b, G[2] * a));
  }
}

template <int n, int GEO, int LAW>
__global__ void __launch_bounds__(32 * kV2Warps) k_vmult2p(CellArgs<float> a)
{
  static_assert(LAW == 0 || LAW == 1 || LAW == 3, "packed kernel: laws 0, 1, 3");
  constexpr int CW = v2_cells_per_warp<n>();  // lane groups per warp (two cells each)
  constexpr int CS = v2_cell_stride<n>();
  constexpr bool TDEP = LAW == 1;
  if (a.st && a.st->done) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int cw_ = lane / n, t = lane % n;
  const bool lane_ok = cw_ < CW;
  F2 *wbuf = reinterpret_cast<F2 *>(smem_raw) + (size_t)warp * (v2_smem_per_warp<n, F2, LAW>() / sizeof(F2));
  F2 *bufA = wbuf + cw_ * CS;
  F2 *bufB = wbuf + (CW + 1) * CS + cw_ * CS;
  F2 *coef = wbuf + 2 * (CW + 1) * CS;  // [4][n*n][32] (law 1), thread-private columns
  const MeshDims &d = a.d;
  double dot = 0.0;
  const int64_t n_pairs = (a.n_cells + 1) / 2;
  const int64_t n_groups = (n_pairs + CW - 1) / CW;
  for (int64_t grp = (int64_t)blockIdx.x * kV2Warps + warp; grp < n_groups;
       grp += (int64_t)gridDim.x * kV2Warps) {
    const int64_t pc = grp * CW + cw_;
    const bool actA = lane_ok && 2 * pc < a.n_cells;
    const bool actB = lane_ok && 2 * pc + 1 < a.n_cells;
    const int64_t cA = actA ? 2 * pc : 0, cB = actB ? 2 * pc + 1 : 0;
    int I0a, J0a, Ka, I0b, J0b, Kb;
    const int64_t bA = cell_plane_base(d, cA, t, I0a, J0a, Ka);
    const int64_t bB = cell_plane_base(d, cB, t, I0b, J0b, Kb);
    const PlaneMask mA(d, I0a, J0a, Ka, d.p), mB(d, I0b, J0b, Kb, d.p);
    const bool adjacent = actB && bB == bA + d.p;  // shared face i = n-1 (A) / i = 0 (B)

    F2 Pu[n][n];
    gather_pair<n>(d, bA, bB, mA, mB, true, a.src, Pu, actA, actB);
    F2 Pt[n][n];
    if (TDEP) gather_pair<n>(d, bA, bB, mA, mB, false, a.Tl, Pt, actA, actB);

    // L2 prefetch of the next pair group's rows (and geometry / conductivity)
    {
      const int64_t npc = pc + (int64_t)gridDim.x * kV2Warps * CW;
      if (lane_ok && 2 * npc < a.n_cells) {
        int i0, j0, k0;
        const int64_t na = cell_plane_base(d, 2 * npc, t, i0, j0, k0);
        prefetch_plane<n>(a.src, na, d.nd[0]);
        if (TDEP) prefetch_plane<n>(a.Tl, na, d.nd[0]);
        if (2 * npc + 1 < a.n_cells) {
          const int64_t nb = cell_plane_base(d, 2 * npc + 1, t, i0, j0, k0);
          if (nb != na + d.p) {
            prefetch_plane<n>(a.src, nb, d.nd[0]);
            if (TDEP) prefetch_plane<n>(a.Tl, nb, d.nd[0]);
          }
        }
        constexpr int npt = n * n * n;
        if (LAW == 3) {
          const char *kq = reinterpret_cast<const char *>(a.kq + 2 * npc * npt);
          for (int off = t * 128; off < 2 * npt * 4; off += n * 128)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(kq + off));
        }
        if (GEO == 1) {
          const char *gq = reinterpret_cast<const char *>(a.g.q + 2 * npc * 7 * npt);
          constexpr int bytes = 2 * 7 * npt * 4;
          for (int off = t * 128; off < bytes; off += n * 128)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(gq + off));
        }
      }
    }

    if (TDEP) {
      F2 (&P)[n][n] = Pt;
      F2 Dx[n][n];
      psweep_b<n, kS, false>(P, P);
      psweep_a<n, kS, false>(P, P);
      psweep_b<n, kD, false>(P, Dx);
      F2 Tq[n][n], Tx[n][n];
      z_to_x2<n>(P, Dx, Tq, Tx, bufA, bufB, t);
      psweep_a<n, kS, false>(Tq, Tq);
      psweep_a<n, kS, false>(Tx, Tx);
      F2 Ty[n][n], Tz[n][n];
      psweep_b<n, kD, false>(Tq, Ty);
      psweep_a<n, kD, false>(Tq, Tz);
      const F2 k0(a.m.k_l), k1(a.m.k1);
#pragma unroll
      for (int k = 0; k < n; ++k)
#pragma unroll
        for (int j = 0; j < n; ++j) {
          const int pt = k * n + j;
          coef[(0 * n * n + pt) * 32 + lane] = fma(k1, Tq[k][j], k0);
          coef[(1 * n * n + pt) * 32 + lane] = k1 * Tx[k][j];
          coef[(2 * n * n + pt) * 32 + lane] = k1 * Ty[k][j];
          coef[(3 * n * n + pt) * 32 + lane] = k1 * Tz[k][j];
        }
    }

    F2 U[n][n], Ux[n][n];
    {
      F2 Dx[n][n];
      psweep_b<n, kS, false>(Pu, Pu);
      psweep_a<n, kS, false>(Pu, Pu);
      psweep_b<n, kD, false>(Pu, Dx);
      z_to_x2<n>(Pu, Dx, U, Ux, bufA, bufB, t);
    }
    psweep_a<n, kS, false>(U, U);
    psweep_a<n, kS, false>(Ux, Ux);
    F2 Uy[n][n], Uz[n][n];
    psweep_b<n, kD, false>(U, Uy);
    psweep_a<n, kD, false>(U, Uz);

    const F2 cval(a.m.idt * (a.m.rho_l * a.m.cp_l));
#pragma unroll
    for (int k = 0; k < n; ++k)
#pragma unroll
      for (int j = 0; j < n; ++j) {
        F2 jxw, G[6];
        geo_pair<n, GEO>(a.g, cA, cB, t, j, k, jxw, G);
        const F2 uu = U[k][j];
        F2 f0, f1, f2;
        if (TDEP) {
          const int pt = k * n + j;
          const F2 kk = coef[(0 * n * n + pt) * 32 + lane];
          f0 = fma(kk, Ux[k][j], coef[(1 * n * n + pt) * 32 + lane] * uu);
          f1 = fma(kk, Uy[k][j], coef[(2 * n * n + pt) * 32 + lane] * uu);
          f2 = fma(kk, Uz[k][j], coef[(3 * n * n + pt) * 32 + lane] * uu);
        } else {
          F2 kk;
          if (LAW == 3) {
            const int q = t + n * (j + n * k);
            kk = F2(actA ? __ldg(a.kq + cA * (n * n * n) + q) : 0.f,
                    actB ? __ldg(a.kq + cB * (n * n * n) + q) : 0.f);
          } else {
            kk = F2(a.m.k_l);
          }
          f0 = kk * Ux[k][j];
          f1 = kk * Uy[k][j];
          f2 = kk * Uz[k][j];
        }
        F2 F0, F1, F2_;
        apply_G2<GEO>(G, f0, f1, f2, F0, F1, F2_);
        U[k][j] = cval * uu * jxw;
        Ux[k][j] = F0;
        Uy[k][j] = F1;
        Uz[k][j] = F2_;
      }

    psweep_b<n, kDT, true>(Uy, U);
    psweep_a<n, kDT, true>(Uz, U);
    psweep_a<n, kST, false>(U, U);
    psweep_a<n, kST, false>(Ux, Ux);
    F2 W[n][n], Wx[n][n];
    x_to_z2<n>(U, Ux, W, Wx, bufA, bufB, t);
    psweep_b<n, kDT, true>(Wx, W);
    psweep_b<n, kST, false>(W, W);
    psweep_a<n, kST, false>(W, W);

    // scatter: cell A (with cell B's first column folded in when they share it), then B
    const bool want_dot = a.fin != FIN_NONE;
    if (actA) {
#pragma unroll
      for (int j = 0; j < n; ++j) {
        const int64_t row = bA + (int64_t)d.nd[0] * j;
#pragma unroll
        for (int i = 0; i < n; ++i) {
          if (mA.template at<n>(i, j)) continue;
          float w = W[j][i].v.x;
          if (i == n - 1 && adjacent) w += W[j][0].v.y;
          atomic_add(a.dst + row + i, w);
          if (want_dot) dot += (double)__ldg(a.src + row + i) * (double)w;
        }
      }
    }
    if (actB) {
#pragma unroll
      for (int j = 0; j < n; ++j) {
        const int64_t row = bB + (int64_t)d.nd[0] * j;
#pragma unroll
        for (int i = 0; i < n; ++i) {
          if (i == 0 && adjacent) continue;
          if (mB.template at<n>(i, j)) continue;
          const float w = W[j][i].v.y;
          atomic_add(a.dst + row + i, w);
          if (want_dot) dot += (double)__ldg(a.src + row + i) * (double)w;
        }
      }
    }
  }
  if (a.fin != FIN_NONE) {
    double v[1] = {dot}, tot[1];
    if (grid_sum<1>(v, a.partials, a.counter, tot)) {
      if (a.extra_dot) tot[0] += *a.extra_dot;
      if (a.fin == FIN_STORE) {
        *a.out = tot[0];
      } else {
        SolverState *s = a.st;
        s->pAp = tot[0];
        if (!(tot[0] > 0.0) || !isfinite(tot[0])) {
          s->done = 2;
          s->status = 5;
        } else {
          s->alpha = s->rz / tot[0];
        }
      }
    }
  }
}

}  // namespace mpdg
