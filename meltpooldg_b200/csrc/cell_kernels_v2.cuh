// Register-resident cell kernel for the operator application (n = p + 1 <= 5).
//
// Layout: every cell gets n threads of one warp (32/n cells per warp); thread t
// holds one 2D plane of the cell's n^3 tensor in registers:
//   Z-layout  thread t holds P[j][i] = u(i, j, k = t)   (x and y in registers)
//   X-layout  thread t holds Q[k][j] = u(i = t, j, k)   (y and z in registers)
// so x/y contractions run on Z-planes and y/z contractions on X-planes without
// touching shared memory. Switching layouts goes through a per-cell shared
// buffer buf[k][j][i] (plane stride n^2+1, cell stride = 4 mod 16 doubles),
// which keeps both the plane-wise writes and the strided reads free of bank
// conflicts. A cell never spans two warps, so __syncwarp is the only barrier.
//
// Operator application per cell (TDEP = temperature-dependent law):
//   T_lin: gather Z, S_x S_y, copy D_x, Z->X (2 planes), S_z (2), D_y, D_z
//          -> per-point coefficients k, dk dT/dxi_d (staged in a thread-private
//             interleaved shared area: the same thread writes and reads them)
//   u:     gather Z (masked), S_x S_y, copy D_x, Z->X (2), S_z (2), D_y, D_z
//   q-op:  val = c u JxW, f = G (k grad u + dk u grad T)   (pointwise, X)
//   integ: t = val + D_y^T f_y + D_z^T f_z, S_z^T t, S_z^T f_x, X->Z (2),
//          w = t + D_x^T f_x, S_x^T, S_y^T, atomic scatter of plane t
// i.e. 21 1D sweeps and 6 layout switches per cell for k(T), 14 and 4 without.
#pragma once

#include "cell_kernels.cuh"

namespace mpdg {

template <int n> __host__ __device__ constexpr int v2_cells_per_warp() { return 32 / n; }
template <int n> __host__ __device__ constexpr int v2_plane_stride() { return n * n + 1; }
template <int n> __host__ __device__ constexpr int v2_cell_stride()
{
  int s = n * v2_plane_stride<n>();
  while (s % 16 != 4) ++s;
  return s;
}
template <int LAW> __host__ __device__ constexpr int v2_ncoef()
{
  return (LAW == 1) ? 4 : (LAW == 2 ? 5 : (LAW == 8 ? 1 : 0));
}
constexpr int kV2Warps = 2;  // warps per CTA
template <int n, typename T, int LAW> __host__ __device__ constexpr size_t v2_smem_per_warp()
{
  return sizeof(T) * ((size_t)2 * (v2_cells_per_warp<n>() + 1) * v2_cell_stride<n>() +
                      (size_t)v2_ncoef<LAW>() * n * n * 32);
}
template <int n, typename T, int LAW> __host__ __device__ constexpr size_t v2_smem()
{
  return kV2Warps * v2_smem_per_warp<n, T, LAW>();
}

// 1D contraction of matrix `kind` along the second index of A[a][b] for every a
// (B may alias A).
template <int n, int kind, bool add, typename T>
__device__ __forceinline__ void psweep_b(const T (&A)[n][n], T (&B)[n][n])
{
  constexpr int h = n / 2;
  constexpr int off = tab_off(n, kind);
  constexpr int sym = kind_sym(kind);
#pragma unroll
  for (int a = 0; a < n; ++a) {
    T x[n];
#pragma unroll
    for (int i = 0; i < n; ++i) x[i] = A[a][i];
    T e[h], o[h];
#pragma unroll
    for (int l = 0; l < h; ++l) {
      e[l] = x[l] + x[n - 1 - l];
      o[l] = x[l] - x[n - 1 - l];
    }
#pragma unroll
    for (int q = 0; q < h + (n & 1); ++q) {
      T E = (n & 1) ? ctab<T>(off + 2 * n * h + q) * x[h] : ctab<T>(off + q * h) * e[0];
      T O = ctab<T>(off + n * h + q * h) * o[0];
#pragma unroll
      for (int l = (n & 1) ? 0 : 1; l < h; ++l) E = fma(ctab<T>(off + q * h + l), e[l], E);
#pragma unroll
      for (int l = 1; l < h; ++l) O = fma(ctab<T>(off + n * h + q * h + l), o[l], O);
      if (q < h) {
        const T y0 = E + O, y1 = sym > 0 ? E - O : O - E;
        B[a][q] = add ? B[a][q] + y0 : y0;
        B[a][n - 1 - q] = add ? B[a][n - 1 - q] + y1 : y1;
      } else {
        B[a][q] = add ? B[a][q] + (E + O) : (E + O);
      }
    }
  }
}

// 1D contraction along the first index of A[a][b] for every b (B may alias A).
template <int n, int kind, bool add, typename T>
__device__ __forceinline__ void psweep_a(const T (&A)[n][n], T (&B)[n][n])
{
  constexpr int h = n / 2;
  constexpr int off = tab_off(n, kind);
  constexpr int sym = kind_sym(kind);
#pragma unroll
  for (int b = 0; b < n; ++b) {
    T x[n];
#pragma unroll
    for (int i = 0; i < n; ++i) x[i] = A[i][b];
    T e[h], o[h];
#pragma unroll
    for (int l = 0; l < h; ++l) {
      e[l] = x[l] + x[n - 1 - l];
      o[l] = x[l] - x[n - 1 - l];
    }
#pragma unroll
    for (int q = 0; q < h + (n & 1); ++q) {
      T E = (n & 1) ? ctab<T>(off + 2 * n * h + q) * x[h] : ctab<T>(off + q * h) * e[0];
      T O = ctab<T>(off + n * h + q * h) * o[0];
#pragma unroll
      for (int l = (n & 1) ? 0 : 1; l < h; ++l) E = fma(ctab<T>(off + q * h + l), e[l], E);
#pragma unroll
      for (int l = 1; l < h; ++l) O = fma(ctab<T>(off + n * h + q * h + l), o[l], O);
      if (q < h) {
        const T y0 = E + O, y1 = sym > 0 ? E - O : O - E;
        B[q][b] = add ? B[q][b] + y0 : y0;
        B[n - 1 - q][b] = add ? B[n - 1 - q][b] + y1 : y1;
      } else {
        B[q][b] = add ? B[q][b] + (E + O) : (E + O);
      }
    }
  }
}

// Layout switches through the per-cell shared buffer buf[k][j][i].
// Z -> X: thread t writes plane k = t, then reads column i = t.
template <int n, typename T>
__device__ __forceinline__ void z_to_x1(const T (&A)[n][n], T (&QA)[n][n], T *ba, int t)
{
  constexpr int PS = v2_plane_stride<n>();
#pragma unroll
  for (int j = 0; j < n; ++j)
#pragma unroll
    for (int i = 0; i < n; ++i) ba[t * PS + j * n + i] = A[j][i];
  __syncwarp();
#pragma unroll
  for (int k = 0; k < n; ++k)
#pragma unroll
    for (int j = 0; j < n; ++j) QA[k][j] = ba[k * PS + j * n + t];
  __syncwarp();
}

template <int n, typename T>
__device__ __forceinline__ void z_to_x2(const T (&A)[n][n], const T (&B)[n][n], T (&QA)[n][n],
                                        T (&QB)[n][n], T *ba, T *bb, int t)
{
  constexpr int PS = v2_plane_stride<n>();
#pragma unroll
  for (int j = 0; j < n; ++j)
#pragma unroll
    for (int i = 0; i < n; ++i) {
      ba[t * PS + j * n + i] = A[j][i];
      bb[t * PS + j * n + i] = B[j][i];
    }
  __syncwarp();
#pragma unroll
  for (int k = 0; k < n; ++k)
#pragma unroll
    for (int j = 0; j < n; ++j) {
      QA[k][j] = ba[k * PS + j * n + t];
      QB[k][j] = bb[k * PS + j * n + t];
    }
  __syncwarp();
}

// X -> Z: thread t writes column i = t, then reads plane k = t.
template <int n, typename T>
__device__ __forceinline__ void x_to_z2(const T (&QA)[n][n], const T (&QB)[n][n], T (&A)[n][n],
                                        T (&B)[n][n], T *ba, T *bb, int t)
{
  constexpr int PS = v2_plane_stride<n>();
#pragma unroll
  for (int k = 0; k < n; ++k)
#pragma unroll
    for (int j = 0; j < n; ++j) {
      ba[k * PS + j * n + t] = QA[k][j];
      bb[k * PS + j * n + t] = QB[k][j];
    }
  __syncwarp();
#pragma unroll
  for (int j = 0; j < n; ++j)
#pragma unroll
    for (int i = 0; i < n; ++i) {
      A[j][i] = ba[t * PS + j * n + i];
      B[j][i] = bb[t * PS + j * n + i];
    }
  __syncwarp();
}

// Dirichlet test of the DoFs of plane K of cell (I0, J0): face flags per row, the
// x faces only at i = 0 and i = n - 1.
struct PlaneMask {
  bool plane, xlo, xhi, ylo, yhi;
  __device__ __forceinline__ PlaneMask(const MeshDims &d, int I0, int J0, int K, int p)
  {
    plane = ((d.dmask & 16) && K == 0) || ((d.dmask & 32) && K == d.nd[2] - 1);
    xlo = (d.dmask & 1) && I0 == 0;
    xhi = (d.dmask & 2) && I0 + p == d.nd[0] - 1;
    ylo = (d.dmask & 4) && J0 == 0;
    yhi = (d.dmask & 8) && J0 + p == d.nd[1] - 1;
  }
  template <int n>
  __device__ __forceinline__ bool at(int i, int j) const
  {
    return plane || (j == 0 && ylo) || (j == n - 1 && yhi) || (i == 0 && xlo) ||
           (i == n - 1 && xhi);
  }
};

// L2 prefetch of the n rows (n values each) of plane K of a cell
template <int n, typename T>
__device__ __forceinline__ void prefetch_plane(const T *g, int64_t base, int nd0)
{
#pragma unroll
  for (int j = 0; j < n; ++j) {
    const T *row = g + base + (int64_t)nd0 * j;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(row));
    if ((reinterpret_cast<uintptr_t>(row) & 127) + n * sizeof(T) > 128)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(row + n - 1));
  }
}

// gather plane k = K of a cell (Z-layout), optionally masked
template <int n, typename T>
__device__ __forceinline__ void gather_plane(const MeshDims &d, int64_t base, const PlaneMask &pm,
                                             bool masked, const T *__restrict__ g, T (&P)[n][n],
                                             bool active)
{
#pragma unroll
  for (int j = 0; j < n; ++j) {
    const int64_t row = base + (int64_t)d.nd[0] * j;
#pragma unroll
    for (int i = 0; i < n; ++i) {
      T v = T(0);
      if (active) {
        v = __ldg(g + row + i);
        if (masked && pm.template at<n>(i, j)) v = T(0);
      }
      P[j][i] = v;
    }
  }
}

// GPRE (deformed meshes, where the 7 x n^2 factors of a thread's points fit the registers): the
// per-point geometry is loaded when the cell group starts, so its loads overlap the gathers and
// the evaluation sweeps instead of stalling the quadrature-point loop
// ROWS (FP32 Picard operator at p = 3): the operand is in the cell-row layout, in which the n = 4
// nodes of a cell's x-row are one aligned float4 and a node shared by x-neighbours is stored in
// both cells' rows (cell_row_index below); a plane is then gathered with 4 vector loads instead
// of 16 scalar ones. The result is scattered into the lexicographic dst as usual; no src.dst
// partial (the host passes FIN_NONE).
template <int n, typename T, int GEO, int LAW, bool GPRE = false, bool ROWS = false>
__global__ void __launch_bounds__(32 * kV2Warps) k_vmult2(CellArgs<T> a)
{
  static_assert(!ROWS || (n == 4 && sizeof(T) == 4 && LAW == 3), "cell rows: FP32 Picard, p = 3");
  constexpr int CW = v2_cells_per_warp<n>();
  constexpr int CS = v2_cell_stride<n>();
  constexpr int NCOEF = v2_ncoef<LAW>();
  // LAW 3: conductivity field k(q), no tangent; LAW 4: coefficient fields a.cf; LAW 6: the
  // tangent coefficient fields of LAW 5 built at the linearisation point (8 per point); LAW 8:
  // the Picard operator of the linear-k law with k(T_lin(q)) interpolated from the gathered
  // T_lin (k is affine in T, so this is the conductivity field of LAW 3 without storing it)
  constexpr bool TDEP = LAW == 1 || LAW == 2;
  constexpr bool TLIN = TDEP || LAW == 8;
  if (a.st && a.st->done) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int cw = lane / n, t = lane % n;
  const bool lane_ok = cw < CW;
  T *wbuf = reinterpret_cast<T *>(smem_raw) + (size_t)warp * (v2_smem_per_warp<n, T, LAW>() / sizeof(T));
  T *bufA = wbuf + cw * CS;                     // idle lanes use the spare slot cw == CW
  T *bufB = wbuf + (CW + 1) * CS + cw * CS;
  T *coef = wbuf + 2 * (CW + 1) * CS;           // [NCOEF][n*n][32], thread-private columns
  const MeshDims &d = a.d;
  double dot = 0.0;
  const int64_t n_groups = (a.n_cells + CW - 1) / CW;
  for (int64_t grp = (int64_t)blockIdx.x * kV2Warps + warp; grp < n_groups;
       grp += (int64_t)gridDim.x * kV2Warps) {
    const int64_t cell = grp * CW + cw;
    const bool active = lane_ok && cell < a.n_cells;
    const int64_t cc = active ? cell : 0;
    const int cx = (int)(cc % d.m[0]);
    const int cy = (int)((cc / d.m[0]) % d.m[1]);
    const int cz = (int)(cc / ((int64_t)d.m[0] * d.m[1]));
    const int I0 = d.p * cx, J0 = d.p * cy, K = d.p * cz + t;
    const int64_t base = (int64_t)d.nd[0] * (J0 + (int64_t)d.nd[1] * K) + I0;
    const PlaneMask pm(d, I0, J0, K, d.p);

    // both gathers first so their latencies overlap
    T Pu[n][n];
    if constexpr (ROWS) {
      const int64_t RS = 4 * (int64_t)d.m[0];
      const int64_t rb = ((int64_t)K * d.nd[1] + J0) * RS + 4 * cx;
#pragma unroll
      for (int j = 0; j < n; ++j) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (active) v = __ldg(reinterpret_cast<const float4 *>(a.src + rb + RS * j));
        Pu[j][0] = pm.template at<n>(0, j) ? T(0) : v.x;
        Pu[j][1] = pm.template at<n>(1, j) ? T(0) : v.y;
        Pu[j][2] = pm.template at<n>(2, j) ? T(0) : v.z;
        Pu[j][3] = pm.template at<n>(3, j) ? T(0) : v.w;
      }
    } else {
      gather_plane<n>(d, base, pm, true, a.src, Pu, active);
    }
    T gpre[GPRE ? 7 : 1][GPRE ? n : 1][GPRE ? n : 1];
    if constexpr (GPRE && GEO == 1) {
      constexpr int npt = n * n * n;
      const T *gb = a.g.q + cc * 7 * npt + t;
#pragma unroll
      for (int f = 0; f < 7; ++f)
#pragma unroll
        for (int k = 0; k < n; ++k)
#pragma unroll
          for (int j = 0; j < n; ++j) gpre[f][k][j] = active ? __ldg(gb + f * npt + n * (j + n * k)) : T(0);
    }
    T Pt[n][n];
    if (TLIN) gather_plane<n>(d, base, pm, false, a.Tl, Pt, active);

    // L2 prefetch of the next group's rows (and geometry) while this one computes
    {
      const int64_t ncell = cell + (int64_t)gridDim.x * kV2Warps * CW;
      if (lane_ok && ncell < a.n_cells) {
        const int ncx = (int)(ncell % d.m[0]);
        const int ncy = (int)((ncell / d.m[0]) % d.m[1]);
        const int ncz = (int)(ncell / ((int64_t)d.m[0] * d.m[1]));
        const int64_t nbase =
          (int64_t)d.nd[0] * (d.p * ncy + (int64_t)d.nd[1] * (d.p * ncz + t)) + d.p * ncx;
        // (cell rows: the vector gathers measured faster without the operand's and the
        // conductivity's prefetch)
        if (!ROWS) prefetch_plane<n>(a.src, nbase, d.nd[0]);
        if (TLIN) prefetch_plane<n>(a.Tl, nbase, d.nd[0]);
        if (LAW == 3 && !ROWS) {
          const char *kq = reinterpret_cast<const char *>(a.kq + ncell * (n * n * n));
          for (int off = t * 128; off < n * n * n * 4; off += n * 128)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(kq + off));
        }
        if (LAW == 4 || LAW == 6 || LAW == 7) {
          constexpr int nf = LAW == 4 ? 5 : (LAW == 6 ? 8 : 4);
          constexpr int bytes = nf * n * n * n * (int)sizeof(T);
          const char *cf = reinterpret_cast<const char *>(a.cf + ncell * nf * (n * n * n));
          for (int off = t * 128; off < bytes; off += n * 128)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(cf + off));
        }
        if (GEO == 1) {
          constexpr int npt = n * n * n;
          const char *gq = reinterpret_cast<const char *>(a.g.q + ncell * 7 * npt);
          constexpr int bytes = 7 * npt * (int)sizeof(T);
          for (int off = t * 128; off < bytes; off += n * 128)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(gq + off));
        }
      }
    }

    if (LAW == 8) {
      // ---- linearisation point: values at the q-points -> k(T_lin) (thread-private columns)
      T (&P)[n][n] = Pt;
      psweep_b<n, kS, false>(P, P);
      psweep_a<n, kS, false>(P, P);
      T Tq[n][n];
      z_to_x1<n>(P, Tq, bufA, t);
      psweep_a<n, kS, false>(Tq, Tq);
#pragma unroll
      for (int k = 0; k < n; ++k)
#pragma unroll
        for (int j = 0; j < n; ++j) {
          T rhocp, kk, drhocp, dk;
          mat_eval<1>(a.m, Tq[k][j], rhocp, kk, drhocp, dk);
          coef[(k * n + j) * 32 + lane] = kk;
        }
    }
    if (TDEP) {
      // ---- linearisation point: values and reference gradients at the q-points
      T (&P)[n][n] = Pt;
      T Dx[n][n];
      psweep_b<n, kS, false>(P, P);
      psweep_a<n, kS, false>(P, P);
      psweep_b<n, kD, false>(P, Dx);
      T Tq[n][n], Tx[n][n];
      z_to_x2<n>(P, Dx, Tq, Tx, bufA, bufB, t);
      psweep_a<n, kS, false>(Tq, Tq);
      psweep_a<n, kS, false>(Tx, Tx);
      T Ty[n][n], Tz[n][n];
      psweep_b<n, kD, false>(Tq, Ty);
      psweep_a<n, kD, false>(Tq, Tz);
      T To[n][n];
      if (LAW == 2 && a.m.need_told) {
        gather_plane<n>(d, base, pm, false, a.To, P, active);
        psweep_b<n, kS, false>(P, P);
        psweep_a<n, kS, false>(P, P);
        z_to_x1<n>(P, To, bufA, t);
        psweep_a<n, kS, false>(To, To);
      }
#pragma unroll
      for (int k = 0; k < n; ++k)
#pragma unroll
        for (int j = 0; j < n; ++j) {
          T rhocp, kk, drhocp, dk;
          mat_eval<LAW>(a.m, Tq[k][j], rhocp, kk, drhocp, dk);
          const int pt = k * n + j;
          coef[(0 * n * n + pt) * 32 + lane] = kk;
          coef[(1 * n * n + pt) * 32 + lane] = dk * Tx[k][j];
          coef[(2 * n * n + pt) * 32 + lane] = dk * Ty[k][j];
          coef[(3 * n * n + pt) * 32 + lane] = dk * Tz[k][j];
          if (LAW == 2) {
            T c = a.m.idt * rhocp;
            if (a.m.need_told) c += a.m.idt * drhocp * (Tq[k][j] - To[k][j]);
            coef[(4 * n * n + pt) * 32 + lane] = c;
          }
        }
    }

    // ---- operand: values and reference gradients at the q-points
    T U[n][n], Ux[n][n];
    {
      T Dx[n][n];
      psweep_b<n, kS, false>(Pu, Pu);
      psweep_a<n, kS, false>(Pu, Pu);
      psweep_b<n, kD, false>(Pu, Dx);
      z_to_x2<n>(Pu, Dx, U, Ux, bufA, bufB, t);
    }
    psweep_a<n, kS, false>(U, U);
    psweep_a<n, kS, false>(Ux, Ux);
    T Uy[n][n], Uz[n][n];
    psweep_b<n, kD, false>(U, Uy);
    psweep_a<n, kD, false>(U, Uz);

    // ---- quadrature-point operation (tangent_local_cell_operation)
#pragma unroll
    for (int k = 0; k < n; ++k)
#pragma unroll
      for (int j = 0; j < n; ++j) {
        T jxw, G[6];
        if constexpr (GPRE && GEO == 1) {
          jxw = gpre[0][k][j];
#pragma unroll
          for (int f = 0; f < 6; ++f) G[f] = gpre[1 + f][k][j];
        } else {
          geo_at<n, GEO>(a.g, cc, t, j, k, jxw, G);
        }
        const T uu = U[k][j];
        T kk, cval;
        T f0, f1, f2;
        T val = T(0);
        if (LAW == 4) {
          // rho_cp u / dt + rho_cp v.grad(u), and the flux k grad(u), from the fields
          constexpr int npt = n * n * n;
          const T *cf = a.cf + cc * 5 * npt + t + n * (j + n * k);
          kk = __ldg(cf + npt);
          val = a.m.idt * __ldg(cf) * uu + __ldg(cf + 2 * npt) * Ux[k][j] +
                __ldg(cf + 3 * npt) * Uy[k][j] + __ldg(cf + 4 * npt) * Uz[k][j];
          f0 = kk * Ux[k][j];
          f1 = kk * Uy[k][j];
          f2 = kk * Uz[k][j];
          cval = T(0);
        } else if (LAW == 7) {
          // linear-k tangent from its fields: flux k(T_lin) grad(u) + k1 grad(T_lin) u
          constexpr int npt = n * n * n;
          const T *cf = a.cf + cc * 4 * npt + t + n * (j + n * k);
          kk = __ldg(cf);
          f0 = kk * Ux[k][j] + __ldg(cf + npt) * uu;
          f1 = kk * Uy[k][j] + __ldg(cf + 2 * npt) * uu;
          f2 = kk * Uz[k][j] + __ldg(cf + 3 * npt) * uu;
          cval = a.m.idt * (a.m.rho_l * a.m.cp_l);
        } else if (LAW == 6) {
          // c u + rho_cp b.grad(u), flux k grad(u) + dk grad(T_lin) u
          constexpr int npt = n * n * n;
          const T *cf = a.cf + cc * 8 * npt + t + n * (j + n * k);
          kk = __ldg(cf + npt);
          val = __ldg(cf) * uu + __ldg(cf + 2 * npt) * Ux[k][j] + __ldg(cf + 3 * npt) * Uy[k][j] +
                __ldg(cf + 4 * npt) * Uz[k][j];
          f0 = kk * Ux[k][j] + __ldg(cf + 5 * npt) * uu;
          f1 = kk * Uy[k][j] + __ldg(cf + 6 * npt) * uu;
          f2 = kk * Uz[k][j] + __ldg(cf + 7 * npt) * uu;
          cval = T(0);
        } else if (TDEP) {
          const int pt = k * n + j;
          kk = coef[(0 * n * n + pt) * 32 + lane];
          f0 = kk * Ux[k][j] + coef[(1 * n * n + pt) * 32 + lane] * uu;
          f1 = kk * Uy[k][j] + coef[(2 * n * n + pt) * 32 + lane] * uu;
          f2 = kk * Uz[k][j] + coef[(3 * n * n + pt) * 32 + lane] * uu;
          cval = LAW == 2 ? coef[(4 * n * n + pt) * 32 + lane] : a.m.idt * (a.m.rho_l * a.m.cp_l);
        } else {
          if (LAW == 3)
            kk = (T)__ldg(a.kq + cc * (n * n * n) + t + n * (j + n * k));
          else if (LAW == 8)
            kk = coef[(k * n + j) * 32 + lane];
          else
            kk = a.m.k_l;
          f0 = kk * Ux[k][j];
          f1 = kk * Uy[k][j];
          f2 = kk * Uz[k][j];
          cval = a.m.idt * (a.m.rho_l * a.m.cp_l);
        }
        T F0, F1, F2;
        apply_G<GEO>(G, f0, f1, f2, F0, F1, F2);
        U[k][j] = (LAW == 4 || LAW == 6) ? val : cval * uu * jxw;
        Ux[k][j] = F0;
        Uy[k][j] = F1;
        Uz[k][j] = F2;
      }

    // ---- integration
    psweep_b<n, kDT, true>(Uy, U);
    psweep_a<n, kDT, true>(Uz, U);
    psweep_a<n, kST, false>(U, U);
    psweep_a<n, kST, false>(Ux, Ux);
    T W[n][n], Wx[n][n];
    x_to_z2<n>(U, Ux, W, Wx, bufA, bufB, t);
    psweep_b<n, kDT, true>(Wx, W);
    psweep_b<n, kST, false>(W, W);
    psweep_a<n, kST, false>(W, W);

    // ---- scatter (constrained rows skipped) and the optional src.dst partial
    if (active) {
      const bool want_dot = !ROWS && a.fin != FIN_NONE;
#pragma unroll
      for (int j = 0; j < n; ++j) {
        const int64_t row = base + (int64_t)d.nd[0] * j;
#pragma unroll
        for (int i = 0; i < n; ++i) {
          const bool c = pm.template at<n>(i, j);
          if (!c) atomic_add(a.dst + row + i, W[j][i]);
          if (want_dot && !c) dot += (double)__ldg(a.src + row + i) * (double)W[j][i];
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

// Conductivity at the quadrature points, kq[cell][q] = k(T_lin(x_q)) in FP32,
// for the coefficient-field (Picard) operator of the FP32 preconditioner.
template <int n, int LAW>
__global__ void __launch_bounds__(32 * kV2Warps) k_conductivity_q(CellArgs<double> a, float *kq)
{
  using T = double;
  constexpr int CW = v2_cells_per_warp<n>();
  constexpr int CS = v2_cell_stride<n>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int cw = lane / n, t = lane % n;
  const bool lane_ok = cw < CW;
  T *bufA = reinterpret_cast<T *>(smem_raw) + (size_t)warp * (CW + 1) * CS + cw * CS;
  const MeshDims &d = a.d;
  const int64_t n_groups = (a.n_cells + CW - 1) / CW;
  for (int64_t grp = (int64_t)blockIdx.x * kV2Warps + warp; grp < n_groups;
       grp += (int64_t)gridDim.x * kV2Warps) {
    const int64_t cell = grp * CW + cw;
    const bool active = lane_ok && cell < a.n_cells;
    const int64_t cc = active ? cell : 0;
    const int cx = (int)(cc % d.m[0]);
    const int cy = (int)((cc / d.m[0]) % d.m[1]);
    const int cz = (int)(cc / ((int64_t)d.m[0] * d.m[1]));
    const int I0 = d.p * cx, J0 = d.p * cy, K = d.p * cz + t;
    const int64_t base = (int64_t)d.nd[0] * (J0 + (int64_t)d.nd[1] * K) + I0;
    const PlaneMask pm(d, I0, J0, K, d.p);
    T P[n][n], Q[n][n];
    gather_plane<n>(d, base, pm, false, a.Tl, P, active);
    psweep_b<n, kS, false>(P, P);
    psweep_a<n, kS, false>(P, P);
    z_to_x1<n>(P, Q, bufA, t);
    psweep_a<n, kS, false>(Q, Q);
    if (active) {
#pragma unroll
      for (int k = 0; k < n; ++k)
#pragma unroll
        for (int j = 0; j < n; ++j) {
          T rhocp, kk, drhocp, dk;
          mat_eval<LAW>(a.m, Q[k][j], rhocp, kk, drhocp, dk);
          kq[cc * (n * n * n) + t + n * (j + n * k)] = (float)kk;
        }
    }
  }
}

// Diagonal of the FP32 Picard operator (conductivity field kq at the q-points, no
// dk/dT term): diag_i = sum_q c JxW phi_i^2 + grad phi_i^T (kq G) grad phi_i, sum-
// factorised with the element-wise products P = S o S, Q = D o D, R = S o D of the 1D
// value and collocation-derivative matrices (transposed tables kPT, kQT, kRT):
// contraction along z and y on X-layout planes, along x on Z-layout planes.
//   A_PP = P_z C0 + Q_z Gzz   A_PQ = P_z Gyy   A_QP = P_z Gxx
//   X_P = P_y A_PP + Q_y A_PQ   X_Q = P_y A_QP   W = P_x X_P + Q_x X_Q
// plus on deformed cells the cross terms (2 kq Gxy ... in R products):
//   A_PR = R_z Gyz  A_RR = P_z Gxy  A_RP = R_z Gxz
//   X_P += R_y A_PR   X_R = R_y A_RR + P_y A_RP   W += R_x X_R
// a.dst (FP32) accumulates; Dirichlet rows are skipped.
template <int n, int GEO>
__global__ void __launch_bounds__(32 * kV2Warps) k_diag_picard(CellArgs<float> a)
{
  using T = float;
  constexpr int CW = v2_cells_per_warp<n>();
  constexpr int CS = v2_cell_stride<n>();
  constexpr int npt = n * n * n;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int cw = lane / n, t = lane % n;
  const bool lane_ok = cw < CW;
  T *wbuf = reinterpret_cast<T *>(smem_raw) + (size_t)warp * 2 * (CW + 1) * CS;
  T *bufA = wbuf + cw * CS;
  T *bufB = wbuf + (CW + 1) * CS + cw * CS;
  const MeshDims &d = a.d;
  const T cval = a.m.idt * (a.m.rho_l * a.m.cp_l);
  const int64_t n_groups = (a.n_cells + CW - 1) / CW;
  for (int64_t grp = (int64_t)blockIdx.x * kV2Warps + warp; grp < n_groups;
       grp += (int64_t)gridDim.x * kV2Warps) {
    const int64_t cell = grp * CW + cw;
    const bool active = lane_ok && cell < a.n_cells;
    const int64_t cc = active ? cell : 0;
    const int cx = (int)(cc % d.m[0]);
    const int cy = (int)((cc / d.m[0]) % d.m[1]);
    const int cz = (int)(cc / ((int64_t)d.m[0] * d.m[1]));
    const int I0 = d.p * cx, J0 = d.p * cy, K = d.p * cz + t;
    const int64_t base = (int64_t)d.nd[0] * (J0 + (int64_t)d.nd[1] * K) + I0;
    const PlaneMask pm(d, I0, J0, K, d.p);
    // q-point coefficients on X-layout planes: thread t = q_x, registers [q_z][q_y]
    T APP[n][n], APQ[n][n], AQP[n][n];
    {
      T C0[n][n], Gxx[n][n], Gyy[n][n], Gzz[n][n];
#pragma unroll
      for (int k = 0; k < n; ++k)
#pragma unroll
        for (int j = 0; j < n; ++j) {
          T jxw, G[6];
          geo_at<n, GEO>(a.g, cc, t, j, k, jxw, G);
          const T kk = active ? (T)__ldg(a.kq + cc * npt + t + n * (j + n * k)) : T(0);
          C0[k][j] = active ? cval * jxw : T(0);
          Gxx[k][j] = kk * G[0];
          Gyy[k][j] = kk * G[3];
          Gzz[k][j] = kk * G[5];
        }
      psweep_a<n, kPT, false>(C0, APP);
      psweep_a<n, kQT, true>(Gzz, APP);
      psweep_a<n, kPT, false>(Gyy, APQ);
      psweep_a<n, kPT, false>(Gxx, AQP);
    }
    T XP[n][n], XQ[n][n];
    psweep_b<n, kPT, false>(APP, XP);
    psweep_b<n, kQT, true>(APQ, XP);
    psweep_b<n, kPT, false>(AQP, XQ);
    T XR[n][n];
    if (GEO == 1) {
      T Gxy[n][n], Gxz[n][n], Gyz[n][n];
#pragma unroll
      for (int k = 0; k < n; ++k)
#pragma unroll
        for (int j = 0; j < n; ++j) {
          T jxw, G[6];
          geo_at<n, GEO>(a.g, cc, t, j, k, jxw, G);
          const T kk = active ? (T)__ldg(a.kq + cc * npt + t + n * (j + n * k)) : T(0);
          Gxy[k][j] = T(2) * kk * G[1];
          Gxz[k][j] = T(2) * kk * G[2];
          Gyz[k][j] = T(2) * kk * G[4];
        }
      T A1[n][n], A2[n][n];
      psweep_a<n, kRT, false>(Gyz, A1);  // A_PR
      psweep_b<n, kRT, true>(A1, XP);
      psweep_a<n, kPT, false>(Gxy, A1);  // A_RR
      psweep_a<n, kRT, false>(Gxz, A2);  // A_RP
      psweep_b<n, kRT, false>(A1, XR);
      psweep_b<n, kPT, true>(A2, XR);
    }
    T ZP[n][n], ZQ[n][n];
    x_to_z2<n>(XP, XQ, ZP, ZQ, bufA, bufB, t);
    T W[n][n];
    psweep_b<n, kPT, false>(ZP, W);
    psweep_b<n, kQT, true>(ZQ, W);
    if (GEO == 1) {
      x_to_z2<n>(XR, XR, ZP, ZQ, bufA, bufB, t);
      psweep_b<n, kRT, true>(ZP, W);
    }
    if (active) {
#pragma unroll
      for (int j = 0; j < n; ++j) {
        const int64_t row = base + (int64_t)d.nd[0] * j;
#pragma unroll
        for (int i = 0; i < n; ++i)
          if (!pm.template at<n>(i, j)) atomicAdd(a.dst + row + i, W[j][i]);
      }
    }
  }
}

// create_rhs on register-resident planes for laws with constant rho*cp (0, 1):
// dst += -R(T) = -sum_q [ (c (T - T_old) - q_h) phi_i JxW + k(T) grad T . G grad phi_i ]
// with c = rho*cp / dt (rhs_cell_loop, heat_diffuse_operator.cpp:393-529). The value
// term is linear in the nodal values, so w = c (T - T_old) - q is formed at the gather
// and interpolated once.
template <int n, int GEO, int LAW>
__global__ void __launch_bounds__(32 * kV2Warps) k_rhs2(CellArgs<double> a)
{
  static_assert(LAW == 0 || LAW == 1, "constant rho*cp laws");
  using T = double;
  constexpr int CW = v2_cells_per_warp<n>();
  constexpr int CS = v2_cell_stride<n>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int cw = lane / n, t = lane % n;
  const bool lane_ok = cw < CW;
  T *wbuf = reinterpret_cast<T *>(smem_raw) + (size_t)warp * 2 * (CW + 1) * CS;
  T *bufA = wbuf + cw * CS;
  T *bufB = wbuf + (CW + 1) * CS + cw * CS;
  const MeshDims &d = a.d;
  const T c = a.m.idt * (a.m.rho_l * a.m.cp_l);
  const int64_t n_groups = (a.n_cells + CW - 1) / CW;
  for (int64_t grp = (int64_t)blockIdx.x * kV2Warps + warp; grp < n_groups;
       grp += (int64_t)gridDim.x * kV2Warps) {
    const int64_t cell = grp * CW + cw;
    const bool active = lane_ok && cell < a.n_cells;
    const int64_t cc = active ? cell : 0;
    const int cx = (int)(cc % d.m[0]);
    const int cy = (int)((cc / d.m[0]) % d.m[1]);
    const int cz = (int)(cc / ((int64_t)d.m[0] * d.m[1]));
    const int I0 = d.p * cx, J0 = d.p * cy, K = d.p * cz + t;
    const int64_t base = (int64_t)d.nd[0] * (J0 + (int64_t)d.nd[1] * K) + I0;
    const PlaneMask pm(d, I0, J0, K, d.p);
    T Pt[n][n], Pw[n][n];
#pragma unroll
    for (int j = 0; j < n; ++j) {
      const int64_t row = base + (int64_t)d.nd[0] * j;
#pragma unroll
      for (int i = 0; i < n; ++i) {
        T tv = T(0), w = T(0);
        if (active) {
          tv = __ldg(a.Tl + row + i);
          const T qv = a.source.on ? (T)source_at(a.source, row + i)
                                   : (a.qs ? __ldg(a.qs + row + i) : T(0));
          w = c * (tv - __ldg(a.To + row + i)) - qv;
        }
        Pt[j][i] = tv;
        Pw[j][i] = w;
      }
    }
    // T at the q-points: values and reference gradients (X-layout)
    T Fx[n][n], Fy[n][n], Fz[n][n];
    {
      T Dx[n][n], Tq[n][n];
      psweep_b<n, kS, false>(Pt, Pt);
      psweep_a<n, kS, false>(Pt, Pt);
      psweep_b<n, kD, false>(Pt, Dx);
      z_to_x2<n>(Pt, Dx, Tq, Fx, bufA, bufB, t);
      psweep_a<n, kS, false>(Tq, Tq);
      psweep_a<n, kS, false>(Fx, Fx);
      psweep_b<n, kD, false>(Tq, Fy);
      psweep_a<n, kD, false>(Tq, Fz);
      // f = -k(T) G grad T
#pragma unroll
      for (int k = 0; k < n; ++k)
#pragma unroll
        for (int j = 0; j < n; ++j) {
          T jxw, G[6];
          geo_at<n, GEO>(a.g, cc, t, j, k, jxw, G);
          T rhocp, kk, drhocp, dk;
          mat_eval<LAW>(a.m, Tq[k][j], rhocp, kk, drhocp, dk);
          T F0, F1, F2;
          apply_G<GEO>(G, kk * Fx[k][j], kk * Fy[k][j], kk * Fz[k][j], F0, F1, F2);
          Fx[k][j] = -F0;
          Fy[k][j] = -F1;
          Fz[k][j] = -F2;
        }
    }
    // w at the q-points, val = -w JxW
    T U[n][n];
    psweep_b<n, kS, false>(Pw, Pw);
    psweep_a<n, kS, false>(Pw, Pw);
    z_to_x1<n>(Pw, U, bufA, t);
    psweep_a<n, kS, false>(U, U);
#pragma unroll
    for (int k = 0; k < n; ++k)
#pragma unroll
      for (int j = 0; j < n; ++j) {
        T jxw, G[6];
        geo_at<n, GEO>(a.g, cc, t, j, k, jxw, G);
        U[k][j] = -U[k][j] * jxw;
      }
    // integration (as in k_vmult2)
    psweep_b<n, kDT, true>(Fy, U);
    psweep_a<n, kDT, true>(Fz, U);
    psweep_a<n, kST, false>(U, U);
    psweep_a<n, kST, false>(Fx, Fx);
    T W[n][n], Wx[n][n];
    x_to_z2<n>(U, Fx, W, Wx, bufA, bufB, t);
    psweep_b<n, kDT, true>(Wx, W);
    psweep_b<n, kST, false>(W, W);
    psweep_a<n, kST, false>(W, W);
    if (active) {
#pragma unroll
      for (int j = 0; j < n; ++j) {
        const int64_t row = base + (int64_t)d.nd[0] * j;
#pragma unroll
        for (int i = 0; i < n; ++i)
          if (!pm.template at<n>(i, j)) atomic_add(a.dst + row + i, W[j][i]);
      }
    }
  }
}

}  // namespace mpdg
