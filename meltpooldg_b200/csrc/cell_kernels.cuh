// Matrix-free cell kernels for the heat tangent operator on sm_100a.
//
// One CTA processes CPB cells at a time (grid-stride over cell batches); each
// cell gets n^2 threads, one per 1D line of the n^3 tensor in the current
// sweep direction. A sweep contracts every line with an n x n matrix using the
// even-odd split (coefficients are compile-time offsets into __constant__
// memory, so they enter the FMAs as constant-bank operands). Cell tensors are
// staged in shared memory between sweeps. Gather/scatter walk x-lines of the
// lexicographic DoF grid, so neighbouring cells of a CTA touch neighbouring
// memory; the scatter is a double/float atomic add into the zeroed output.
//
// The arithmetic restates deal.II FEEvaluation as MeltPoolDG uses it:
//   evaluate(values|gradients): values at QGauss(n) by three S sweeps,
//     gradients by collocation derivative sweeps D at the Gauss points;
//   q-point work of HeatDiffuseMultiPhaseOperator::tangent_local_cell_operation
//     (source/heat/heat_diffuse_operator.cpp:1029-1078) and rhs_cell_loop
//     (:481-527);
//   integrate(values|gradients): D^T sweeps accumulated, then three S^T sweeps.
//
// LAW selects the q-point coefficients: 0 constant, 1 k(T) = k_l + k1 T, 2 liquid-solid
// (both with their tangent terms at T_lin), 3 a per-q FP32 conductivity field (the Picard
// operator of the preconditioner, register-resident kernel only), 4 per-q coefficient
// fields a.cf (gas-liquid law weighted by the level-set heaviside and/or the convective
// term rho_cp v.grad, heat_diffuse_operator.cpp:499-500 and :1038-1042), 5 the liquid-solid
// law at T_lin mixed with the gas by a per-q weight, with the convective terms including
// d(rho_cp)/dT (v.grad T_lin) u (:1044-1049) (three-phase law, liquid-solid with velocity).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cell_args.cuh"
#include "fe_tables.hpp"
#include "material_law.cuh"
#include "reduce.cuh"
#include "source_eval.cuh"

namespace mpdg {

// ---------------------------------------------------------------------------
// constant tables (one copy per translation unit; uploaded by its host stub)
// ---------------------------------------------------------------------------
static __constant__ double c_tab_d[kTabSize];
static __constant__ float c_tab_f[kTabSize];
static __constant__ double c_w_d[kWSize];
static __constant__ float c_w_f[kWSize];

template <typename T> __device__ __forceinline__ T ctab(int i);
template <> __device__ __forceinline__ double ctab<double>(int i) { return c_tab_d[i]; }
template <> __device__ __forceinline__ float ctab<float>(int i) { return c_tab_f[i]; }
template <typename T> __device__ __forceinline__ T cw(int i);
template <> __device__ __forceinline__ double cw<double>(int i) { return c_w_d[i]; }
template <> __device__ __forceinline__ float cw<float>(int i) { return c_w_f[i]; }

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------

template <typename T> __device__ __forceinline__ void atomic_add(T *p, T v) { atomicAdd(p, v); }

// laws whose coefficients depend on the linearisation point T_lin
template <int LAW> __host__ __device__ constexpr bool law_tdep() { return LAW == 1 || LAW == 2 || LAW == 5; }
// laws that may need T_old (d(rho_cp)/dT (T_lin - T_old) / dt in the tangent)
template <int LAW> __host__ __device__ constexpr bool law_told() { return LAW == 2 || LAW == 5; }
// shared arrays per cell of the line-per-thread operator: u and its gradients, a temporary (Tq
// doubles as it with T_lin), T_lin's values and gradients, T_old's values
template <int LAW> __host__ __device__ constexpr int vmult_arrays()
{
  return law_tdep<LAW>() ? (law_told<LAW>() ? 9 : 8) : 5;
}

// One 1D sweep of matrix `kind` along `dir` for line `line` (0 <= line < n^2).
template <int n, int kind, int dir, bool add, typename T>
__device__ __forceinline__ void sweep(const T *in, T *out, int line)
{
  constexpr int h = n / 2;
  constexpr int st = dir == 0 ? 1 : (dir == 1 ? n : n * n);
  constexpr int off = tab_off(n, kind);
  constexpr int sym = kind_sym(kind);
  const int a = line % n, b = line / n;
  const int base = dir == 0 ? n * (a + n * b) : (dir == 1 ? a + n * n * b : a + n * b);
  T x[n];
#pragma unroll
  for (int i = 0; i < n; ++i) x[i] = in[base + i * st];
  T e[h], o[h];
#pragma unroll
  for (int l = 0; l < h; ++l) {
    e[l] = x[l] + x[n - 1 - l];
    o[l] = x[l] - x[n - 1 - l];
  }
#pragma unroll
  for (int q = 0; q < h + (n & 1); ++q) {
    T E, O;
    if (n & 1)
      E = ctab<T>(off + 2 * n * h + q) * x[h];
    else
      E = ctab<T>(off + q * h) * e[0];
    O = ctab<T>(off + n * h + q * h) * o[0];
#pragma unroll
    for (int l = (n & 1) ? 0 : 1; l < h; ++l) E = fma(ctab<T>(off + q * h + l), e[l], E);
#pragma unroll
    for (int l = 1; l < h; ++l) O = fma(ctab<T>(off + n * h + q * h + l), o[l], O);
    if (q < h) {
      const T y0 = E + O;
      const T y1 = sym > 0 ? E - O : O - E;
      if (add) {
        out[base + q * st] += y0;
        out[base + (n - 1 - q) * st] += y1;
      } else {
        out[base + q * st] = y0;
        out[base + (n - 1 - q) * st] = y1;
      }
    } else {
      const T y0 = E + O;
      if (add)
        out[base + q * st] += y0;
      else
        out[base + q * st] = y0;
    }
  }
}

// values (3 S sweeps) of u into vq, using t1, t2 as temporaries; u is preserved
template <int n, typename T>
__device__ __forceinline__ void eval_values(const T *u, T *t1, T *t2, T *vq, int line)
{
  sweep<n, kS, 0, false>(u, t1, line);
  __syncthreads();
  sweep<n, kS, 1, false>(t1, t2, line);
  __syncthreads();
  sweep<n, kS, 2, false>(t2, vq, line);
  __syncthreads();
}

template <int n, typename T>
__device__ __forceinline__ void eval_gradients(const T *vq, T *dx, T *dy, T *dz, int line)
{
  sweep<n, kD, 0, false>(vq, dx, line);
  sweep<n, kD, 1, false>(vq, dy, line);
  sweep<n, kD, 2, false>(vq, dz, line);
  __syncthreads();
}

// v = S^T S^T S^T (v + D_x^T fx + D_y^T fy + D_z^T fz); fx and t1 are clobbered
template <int n, typename T>
__device__ __forceinline__ void integrate(T *v, T *fx, const T *fy, const T *fz, T *t1, int line)
{
  sweep<n, kDT, 0, true>(fx, v, line);
  __syncthreads();
  sweep<n, kDT, 1, true>(fy, v, line);
  __syncthreads();
  sweep<n, kDT, 2, true>(fz, v, line);
  __syncthreads();
  sweep<n, kST, 2, false>(v, t1, line);
  __syncthreads();
  sweep<n, kST, 1, false>(t1, fx, line);
  __syncthreads();
  sweep<n, kST, 0, false>(fx, v, line);
  __syncthreads();
}

template <int n, typename T>
__device__ __forceinline__ void gather_xline(const MeshDims &d, int64_t row, int I0, int J, int K,
                                             bool masked, const T *__restrict__ g, T *x,
                                             bool active)
{
#pragma unroll
  for (int i = 0; i < n; ++i) {
    T v = T(0);
    if (active) {
      v = __ldg(g + row + i);
      if (masked && constrained(d, I0 + i, J, K)) v = T(0);
    }
    x[i] = v;
  }
}

// geometry of point (qi,qj,qk) of a cell; G has 6 comps (diagonal for GEO == 0)
template <int n, int GEO, typename T>
__device__ __forceinline__ void geo_at(const GeoParams<T> &g, int64_t cell, int qi, int qj, int qk,
                                       T &jxw, T G[6])
{
  if (GEO == 0) {
    const T w = cw<T>(w_off(n) + qi) * cw<T>(w_off(n) + qj) * cw<T>(w_off(n) + qk);
    jxw = g.detJ * w;
    G[0] = g.Gd[0] * w;
    G[1] = T(0);
    G[2] = T(0);
    G[3] = g.Gd[1] * w;
    G[4] = T(0);
    G[5] = g.Gd[2] * w;
  } else {
    constexpr int npt = n * n * n;
    const int q = qi + n * (qj + n * qk);
    const T *base = g.q + cell * 7 * npt + q;
    jxw = __ldg(base);
#pragma unroll
    for (int t = 0; t < 6; ++t) G[t] = __ldg(base + (1 + t) * npt);
  }
}

template <int GEO, typename T>
__device__ __forceinline__ void apply_G(const T G[6], T a, T b, T c, T &x, T &y, T &z)
{
  if (GEO == 0) {
    x = G[0] * a;
    y = G[3] * b;
    z = G[5] * c;
  } else {
    x = G[0] * a + G[1] * b + G[2] * c;
    y = G[1] * a + G[3] * b + G[4] * c;
    z = G[2] * a + G[4] * b + G[5] * c;
  }
}

// L2 prefetch of the next batch of a line-per-thread kernel: this thread's x-line of each
// given vector and, cooperatively over the block, the batch's contiguous per-cell blocks of
// per-q data (nper values per q-point), so the next batch's gathers and q-point loads hit L2
// instead of stalling on DRAM (the long-scoreboard stall of the q-point loop).
template <int n, typename T>
__device__ __forceinline__ void prefetch_next_batch(const MeshDims &d, int64_t n_cells,
                                                    int64_t next_batch, int cl, int j, int k,
                                                    const T *v0, const T *v1, const T *perq,
                                                    int nper)
{
  constexpr int n3 = n * n * n, CPB = cells_per_block(n);
  const int64_t first = next_batch * CPB;
  if (first >= n_cells) return;
  const int64_t ncell = first + cl;
  if (ncell < n_cells) {
    const int ncx = (int)(ncell % d.m[0]);
    const int ncy = (int)((ncell / d.m[0]) % d.m[1]);
    const int ncz = (int)(ncell / ((int64_t)d.m[0] * d.m[1]));
    const int64_t nrow =
      (int64_t)d.nd[0] * ((d.p * ncy + j) + (int64_t)d.nd[1] * (d.p * ncz + k)) + d.p * ncx;
    for (const T *v : {v0, v1}) {
      if (!v) continue;
      asm volatile("prefetch.global.L2 [%0];" ::"l"(v + nrow));
      asm volatile("prefetch.global.L2 [%0];" ::"l"(v + nrow + n - 1));
    }
  }
  if (perq) {
    const int64_t last = first + CPB < n_cells ? first + CPB : n_cells;
    const char *g0 = reinterpret_cast<const char *>(perq + first * nper * n3);
    const int64_t bytes = (last - first) * nper * n3 * (int64_t)sizeof(T);
    for (int64_t off = (int64_t)threadIdx.x * 128; off < bytes; off += (int64_t)blockDim.x * 128)
      asm volatile("prefetch.global.L2 [%0];" ::"l"(g0 + off));
  }
}

// ---------------------------------------------------------------------------
// vmult: dst += J src (dst zeroed by the caller); optional src.dst dot
// ---------------------------------------------------------------------------
// PRE (deformed meshes): this batch's per-point geometry (7 values at each of the thread's n
// points) is loaded into registers when the batch starts, so those loads are in flight during
// the gather and the evaluation sweeps instead of stalling the quadrature-point loop.
template <int n, typename T, int GEO, int LAW, bool PRE = false>
__global__ void __launch_bounds__(block_threads(n)) k_vmult(CellArgs<T> a)
{
  constexpr int n2 = n * n, n3 = n2 * n, CPB = cells_per_block(n);
  constexpr bool TDEP = law_tdep<LAW>();
  static_assert(!PRE || GEO == 1, "the geometry preload is for per-point geometry");
  // shared arrays per cell: the sweeps' temporaries alias arrays that are free at that time
  // (gx, gy while values are interpolated, the gathered T_lin in gz, Tq after the q-point loop)
  constexpr int NF = vmult_arrays<LAW>();
  if (a.st && a.st->done) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  const int cl = threadIdx.x / n2, line = threadIdx.x % n2;
  T *u = sm + cl * NF * n3, *gx = u + n3, *gy = u + 2 * n3, *gz = u + 3 * n3;
  T *t1 = u + 4 * n3;  // integration temporary without the T_lin arrays
  T *Tq = u + 4 * n3, *Tx = u + 5 * n3, *Ty = u + 6 * n3, *Tz = u + 7 * n3, *Toq = u + 8 * n3;
  const MeshDims &d = a.d;
  double dot = 0.0;
  const int64_t n_batches = (a.n_cells + CPB - 1) / CPB;
  for (int64_t batch = blockIdx.x; batch < n_batches; batch += gridDim.x) {
    const int64_t cell = batch * CPB + cl;
    const bool active = cell < a.n_cells;
    const int64_t cc = active ? cell : 0;
    const int cx = (int)(cc % d.m[0]);
    const int cy = (int)((cc / d.m[0]) % d.m[1]);
    const int cz = (int)(cc / ((int64_t)d.m[0] * d.m[1]));
    const int j = line % n, k = line / n;
    const int I0 = d.p * cx, J = d.p * cy + j, K = d.p * cz + k;
    const int64_t row = (int64_t)d.nd[0] * (J + (int64_t)d.nd[1] * K) + I0;
    T gpre[PRE ? n : 1][7];
    T fpre[(PRE && LAW == 7) ? n : 1][4];
    if (PRE) {
      const T *gb = a.g.q + cc * 7 * n3 + line;
#pragma unroll
      for (int r = 0; r < n; ++r)
#pragma unroll
        for (int c = 0; c < 7; ++c) gpre[r][c] = __ldg(gb + c * n3 + n2 * r);
      if (LAW == 7) {
        const T *fb = a.cf + cc * 4 * n3 + line;
#pragma unroll
        for (int r = 0; r < n; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c) fpre[r][c] = __ldg(fb + c * n3 + n2 * r);
      }
    }
    // the geometry, or the coefficient fields of LAW 4/5, dominate a batch's q-point loads
    if (GEO == 1)
      prefetch_next_batch<n>(d, a.n_cells, batch + gridDim.x, cl, j, k, a.src,
                             TDEP ? a.Tl : nullptr, a.g.q, 7);
    else
      prefetch_next_batch<n>(d, a.n_cells, batch + gridDim.x, cl, j, k, a.src,
                             TDEP ? a.Tl : nullptr, (LAW == 4 || LAW == 5) ? a.cf : nullptr, 5);
    T xs[n];
    gather_xline<n>(d, row, I0, J, K, true, a.src, xs, active);
#pragma unroll
    for (int i = 0; i < n; ++i) u[i + n * line] = xs[i];
    if (TDEP) {
      T xt[n];
      if (law_told<LAW>() && a.m.need_told) {
        gather_xline<n>(d, row, I0, J, K, false, a.To, xt, active);
#pragma unroll
        for (int i = 0; i < n; ++i) Tq[i + n * line] = xt[i];
      }
      gather_xline<n>(d, row, I0, J, K, false, a.Tl, xt, active);
#pragma unroll
      for (int i = 0; i < n; ++i) gz[i + n * line] = xt[i];
    }
    __syncthreads();
    if (TDEP) {
      // T_lin values + gradients: gz -> (S) -> Tq; old values first if needed
      if (law_told<LAW>() && a.m.need_told) {
        eval_values<n>(Tq, gx, gy, Toq, line);
      }
      eval_values<n>(gz, gx, gy, Tq, line);
      eval_gradients<n>(Tq, Tx, Ty, Tz, line);
    }
    eval_values<n>(u, gx, gy, u, line);  // values overwrite the gathered nodal values
    eval_gradients<n>(u, gx, gy, gz, line);
    // quadrature-point operation (tangent_local_cell_operation)
#pragma unroll
    for (int r = 0; r < n; ++r) {
      const int q = line + n2 * r;
      const int qi = q % n, qj = (q / n) % n, qk = q / n2;
      T jxw, G[6];
      if (PRE) {
        jxw = gpre[r][0];
#pragma unroll
        for (int c = 0; c < 6; ++c) G[c] = gpre[r][1 + c];
      } else {
        geo_at<n, GEO>(a.g, cc, qi, qj, qk, jxw, G);
      }
      T rhocp, kk, drhocp, dk;
      const T uu = u[q];
      T val, b0 = T(0), b1 = T(0), b2 = T(0);
      if (LAW == 5) {
        const T *cf = a.cf + cc * 5 * n3 + q;
        mat_eval_w(a.m, Tq[q], __ldg(cf), rhocp, kk, drhocp, dk);
        b0 = __ldg(cf + 2 * n3);
        b1 = __ldg(cf + 3 * n3);
        b2 = __ldg(cf + 4 * n3);
      } else if (LAW == 4) {
        const T *cf = a.cf + cc * 5 * n3 + q;
        kk = __ldg(cf + n3);
        rhocp = drhocp = dk = T(0);
        val = a.m.idt * __ldg(cf) * uu + __ldg(cf + 2 * n3) * gx[q] + __ldg(cf + 3 * n3) * gy[q] +
              __ldg(cf + 4 * n3) * gz[q];
      } else if (LAW == 7) {
        // linear-k tangent from its fields: k(T_lin) and k1 dT_lin/dxi_d at the point
        T fk, fd[3];
        if (PRE) {
          fk = fpre[r][0];
#pragma unroll
          for (int c = 0; c < 3; ++c) fd[c] = fpre[r][1 + c];
        } else {
          const T *cf = a.cf + cc * 4 * n3 + q;
          fk = __ldg(cf);
#pragma unroll
          for (int c = 0; c < 3; ++c) fd[c] = __ldg(cf + (1 + c) * n3);
        }
        kk = fk;
        rhocp = a.m.rho_l * a.m.cp_l;
        drhocp = dk = T(0);
        b0 = fd[0];
        b1 = fd[1];
        b2 = fd[2];
      } else {
        mat_eval<LAW>(a.m, TDEP ? Tq[q] : T(0), rhocp, kk, drhocp, dk);
      }
      T cval = a.m.idt * rhocp;
      T f0 = kk * gx[q], f1 = kk * gy[q], f2 = kk * gz[q];
      if (LAW == 7) {
        f0 += b0 * uu;
        f1 += b1 * uu;
        f2 += b2 * uu;
      }
      if (TDEP) {
        if (law_told<LAW>() && a.m.need_told) cval += a.m.idt * drhocp * (Tq[q] - Toq[q]);
        f0 += dk * Tx[q] * uu;
        f1 += dk * Ty[q] * uu;
        f2 += dk * Tz[q] * uu;
      }
      if (LAW == 5)  // rho_cp b.grad(u) + d(rho_cp)/dT (b.grad T) u, b = JxW J^-1 v
        val = cval * uu * jxw + rhocp * (b0 * gx[q] + b1 * gy[q] + b2 * gz[q]) +
              drhocp * (b0 * Tx[q] + b1 * Ty[q] + b2 * Tz[q]) * uu;
      u[q] = (LAW == 4 || LAW == 5) ? val : cval * uu * jxw;
      T F0, F1, F2;
      apply_G<GEO>(G, f0, f1, f2, F0, F1, F2);
      gx[q] = F0;
      gy[q] = F1;
      gz[q] = F2;
    }
    __syncthreads();
    integrate<n>(u, gx, gy, gz, t1, line);
    // scatter the x-line (skip constrained rows) and accumulate src.dst
    if (active) {
#pragma unroll
      for (int i = 0; i < n; ++i) {
        const T r = u[i + n * line];
        if (!constrained(d, I0 + i, J, K)) atomic_add(a.dst + row + i, r);
        dot += (double)xs[i] * (double)r;
      }
    }
    __syncthreads();
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
          s->status = 5;  // breakdown
        } else {
          s->alpha = s->rz / tot[0];
        }
      }
    }
  }
}

// ---------------------------------------------------------------------------
// create_rhs: dst += -R(T)   (rhs_cell_loop, heat_diffuse_operator.cpp:393-529)
// ---------------------------------------------------------------------------
template <int n, int GEO, int LAW>
__global__ void __launch_bounds__(block_threads(n)) k_rhs(CellArgs<double> a)
{
  using T = double;
  constexpr int n2 = n * n, n3 = n2 * n, CPB = cells_per_block(n);
  constexpr int NF = 9;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  const int cl = threadIdx.x / n2, line = threadIdx.x % n2;
  T *u = sm + cl * NF * n3, *t1 = u + n3, *t2 = u + 2 * n3, *gx = u + 3 * n3, *gy = u + 4 * n3,
    *gz = u + 5 * n3, *Toq = u + 6 * n3, *Sq = u + 7 * n3, *tq = u + 8 * n3;
  const MeshDims &d = a.d;
  const int64_t n_batches = (a.n_cells + CPB - 1) / CPB;
  for (int64_t batch = blockIdx.x; batch < n_batches; batch += gridDim.x) {
    const int64_t cell = batch * CPB + cl;
    const bool active = cell < a.n_cells;
    const int64_t cc = active ? cell : 0;
    const int cx = (int)(cc % d.m[0]);
    const int cy = (int)((cc / d.m[0]) % d.m[1]);
    const int cz = (int)(cc / ((int64_t)d.m[0] * d.m[1]));
    const int j = line % n, k = line / n;
    const int I0 = d.p * cx, J = d.p * cy + j, K = d.p * cz + k;
    const int64_t row = (int64_t)d.nd[0] * (J + (int64_t)d.nd[1] * K) + I0;
    T x[n];
    gather_xline<n>(d, row, I0, J, K, false, a.Tl, x, active);
#pragma unroll
    for (int i = 0; i < n; ++i) u[i + n * line] = x[i];
    gather_xline<n>(d, row, I0, J, K, false, a.To, x, active);
#pragma unroll
    for (int i = 0; i < n; ++i) Toq[i + n * line] = x[i];
    if (a.source.on) {
#pragma unroll
      for (int i = 0; i < n; ++i) x[i] = active ? source_at(a.source, row + i) : T(0);
    } else if (a.qs) {
      gather_xline<n>(d, row, I0, J, K, false, a.qs, x, active);
    } else {
#pragma unroll
      for (int i = 0; i < n; ++i) x[i] = T(0);
    }
#pragma unroll
    for (int i = 0; i < n; ++i) Sq[i + n * line] = x[i];
    __syncthreads();
    eval_values<n>(Toq, t1, t2, Toq, line);
    eval_values<n>(Sq, t1, t2, Sq, line);
    eval_values<n>(u, t1, t2, tq, line);
    eval_gradients<n>(tq, gx, gy, gz, line);
#pragma unroll
    for (int r = 0; r < n; ++r) {
      const int q = line + n2 * r;
      const int qi = q % n, qj = (q / n) % n, qk = q / n2;
      T jxw, G[6];
      geo_at<n, GEO>(a.g, cc, qi, qj, qk, jxw, G);
      T rhocp, kk, drhocp, dk, valw;
      if (LAW == 5) {
        const T *cf = a.cf + cc * 5 * n3 + q;
        mat_eval_w(a.m, tq[q], __ldg(cf), rhocp, kk, drhocp, dk);
        valw = (a.m.idt * rhocp * (tq[q] - Toq[q]) - Sq[q]) * jxw +
               rhocp * (__ldg(cf + 2 * n3) * gx[q] + __ldg(cf + 3 * n3) * gy[q] +
                        __ldg(cf + 4 * n3) * gz[q]);
      } else if (LAW == 4) {
        // rho_cp (T - T_old) / dt - q + rho_cp grad(T).v, times JxW
        const T *cf = a.cf + cc * 5 * n3 + q;
        kk = __ldg(cf + n3);
        valw = a.m.idt * __ldg(cf) * (tq[q] - Toq[q]) - Sq[q] * jxw +
               __ldg(cf + 2 * n3) * gx[q] + __ldg(cf + 3 * n3) * gy[q] + __ldg(cf + 4 * n3) * gz[q];
      } else {
        mat_eval<LAW>(a.m, tq[q], rhocp, kk, drhocp, dk);
        valw = (a.m.idt * rhocp * (tq[q] - Toq[q]) - Sq[q]) * jxw;
      }
      T F0, F1, F2;
      apply_G<GEO>(G, kk * gx[q], kk * gy[q], kk * gz[q], F0, F1, F2);
      u[q] = -valw;
      gx[q] = -F0;
      gy[q] = -F1;
      gz[q] = -F2;
    }
    __syncthreads();
    integrate<n>(u, gx, gy, gz, t1, line);
    if (active) {
#pragma unroll
      for (int i = 0; i < n; ++i)
        if (!constrained(d, I0 + i, J, K)) atomic_add(a.dst + row + i, u[i + n * line]);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// diagonal (MatrixFreeTools::compute_diagonal of the same local operation),
// closed form: diag_i = sum_q c0 phi_i^2 + grad phi_i^T kG grad phi_i
//                      + dk phi_i grad phi_i^T G grad T_lin,
// sum-factorised with the element-wise product matrices PT, QT, RT.
// ---------------------------------------------------------------------------
template <int n, int GEO, int LAW>
__global__ void __launch_bounds__(block_threads(n)) k_diag(CellArgs<double> a)
{
  using T = double;
  constexpr int n2 = n * n, n3 = n2 * n, CPB = cells_per_block(n);
  constexpr bool TDEP = law_tdep<LAW>();
  constexpr int NF = 16;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  const int cl = threadIdx.x / n2, line = threadIdx.x % n2;
  T *f = sm + cl * NF * n3;
  T *C0 = f, *Gxx = f + n3, *Gxy = f + 2 * n3, *Gxz = f + 3 * n3, *Gyy = f + 4 * n3,
    *Gyz = f + 5 * n3, *Gzz = f + 6 * n3, *Bx = f + 7 * n3, *By = f + 8 * n3, *Bz = f + 9 * n3;
  T *A = f + 10 * n3, *B = f + 11 * n3, *X = f + 12 * n3, *Y = f + 13 * n3, *W = f + 14 * n3,
    *Tq = f + 15 * n3;
  // T_lin gradients live in Bx..Bz until they are turned into B coefficients
  const MeshDims &d = a.d;
  const int64_t n_batches = (a.n_cells + CPB - 1) / CPB;
  for (int64_t batch = blockIdx.x; batch < n_batches; batch += gridDim.x) {
    const int64_t cell = batch * CPB + cl;
    const bool active = cell < a.n_cells;
    const int64_t cc = active ? cell : 0;
    const int cx = (int)(cc % d.m[0]);
    const int cy = (int)((cc / d.m[0]) % d.m[1]);
    const int cz = (int)(cc / ((int64_t)d.m[0] * d.m[1]));
    const int j = line % n, k = line / n;
    const int I0 = d.p * cx, J = d.p * cy + j, K = d.p * cz + k;
    const int64_t row = (int64_t)d.nd[0] * (J + (int64_t)d.nd[1] * K) + I0;
    if (TDEP) {
      T x[n];
      gather_xline<n>(d, row, I0, J, K, false, a.Tl, x, active);
#pragma unroll
      for (int i = 0; i < n; ++i) A[i + n * line] = x[i];
      if (law_told<LAW>() && a.m.need_told) {
        gather_xline<n>(d, row, I0, J, K, false, a.To, x, active);
#pragma unroll
        for (int i = 0; i < n; ++i) W[i + n * line] = x[i];
      }
      __syncthreads();
      if (law_told<LAW>() && a.m.need_told) eval_values<n>(W, X, Y, C0, line);  // T_old values -> C0
      eval_values<n>(A, X, Y, Tq, line);
      eval_gradients<n>(Tq, Bx, By, Bz, line);
    }
#pragma unroll
    for (int r = 0; r < n; ++r) {
      const int q = line + n2 * r;
      const int qi = q % n, qj = (q / n) % n, qk = q / n2;
      T jxw, G[6];
      geo_at<n, GEO>(a.g, cc, qi, qj, qk, jxw, G);
      T rhocp, kk, drhocp, dk;
      const T *cf = (LAW == 4 || LAW == 5) ? a.cf + cc * 5 * n3 + q : nullptr;
      if (LAW == 4) {
        kk = __ldg(cf + n3);
        rhocp = drhocp = dk = T(0);
      } else if (LAW == 5) {
        mat_eval_w(a.m, Tq[q], __ldg(cf), rhocp, kk, drhocp, dk);
      } else {
        mat_eval<LAW>(a.m, TDEP ? Tq[q] : T(0), rhocp, kk, drhocp, dk);
      }
      T cval = LAW == 4 ? T(0) : a.m.idt * rhocp;
      if (TDEP && law_told<LAW>() && a.m.need_told) cval += a.m.idt * drhocp * (Tq[q] - C0[q]);
      C0[q] = LAW == 4 ? a.m.idt * __ldg(cf) : cval * jxw;
      if (LAW == 5)  // d(rho_cp)/dT (b.grad T_lin) u is a mass-like term
        C0[q] += drhocp * (__ldg(cf + 2 * n3) * Bx[q] + __ldg(cf + 3 * n3) * By[q] +
                           __ldg(cf + 4 * n3) * Bz[q]);
      Gxx[q] = kk * G[0];
      Gxy[q] = T(2) * kk * G[1];
      Gxz[q] = T(2) * kk * G[2];
      Gyy[q] = kk * G[3];
      Gyz[q] = T(2) * kk * G[4];
      Gzz[q] = kk * G[5];
      if (TDEP) {
        T b0, b1, b2;
        const T t0 = Bx[q], t1v = By[q], t2v = Bz[q];
        b0 = G[0] * t0 + G[1] * t1v + G[2] * t2v;
        b1 = G[1] * t0 + G[3] * t1v + G[4] * t2v;
        b2 = G[2] * t0 + G[4] * t1v + G[5] * t2v;
        Bx[q] = dk * b0;
        By[q] = dk * b1;
        Bz[q] = dk * b2;
        if (LAW == 5) {  // convection: phi_i rho_cp (JxW J^-1 v).grad_ref(phi_i)
          Bx[q] += rhocp * __ldg(cf + 2 * n3);
          By[q] += rhocp * __ldg(cf + 3 * n3);
          Bz[q] += rhocp * __ldg(cf + 4 * n3);
        }
      } else if (LAW == 4) {
        // convection: phi_i (JxW rho_cp J^-1 v).grad_ref(phi_i)
        Bx[q] = __ldg(cf + 2 * n3);
        By[q] = __ldg(cf + 3 * n3);
        Bz[q] = __ldg(cf + 4 * n3);
      } else {
        Bx[q] = T(0);
        By[q] = T(0);
        Bz[q] = T(0);
      }
    }
    __syncthreads();
    // (x,y) = (P,P): z: P C0 + Q Gzz + R Bz
    sweep<n, kPT, 2, false>(C0, A, line);
    __syncthreads();
    sweep<n, kQT, 2, true>(Gzz, A, line);
    __syncthreads();
    sweep<n, kRT, 2, true>(Bz, A, line);
    __syncthreads();
    sweep<n, kPT, 1, false>(A, X, line);
    __syncthreads();
    // (P,Q): z P Gyy, y Q
    sweep<n, kPT, 2, false>(Gyy, A, line);
    __syncthreads();
    sweep<n, kQT, 1, true>(A, X, line);
    __syncthreads();
    // (P,R): z R Gyz + P By, y R
    sweep<n, kRT, 2, false>(Gyz, A, line);
    __syncthreads();
    sweep<n, kPT, 2, true>(By, A, line);
    __syncthreads();
    sweep<n, kRT, 1, true>(A, X, line);
    __syncthreads();
    sweep<n, kPT, 0, false>(X, W, line);
    __syncthreads();
    // (Q,P): z P Gxx, y P, x Q
    sweep<n, kPT, 2, false>(Gxx, A, line);
    __syncthreads();
    sweep<n, kPT, 1, false>(A, B, line);
    __syncthreads();
    sweep<n, kQT, 0, true>(B, W, line);
    __syncthreads();
    // (R,R): z P Gxy, y R ; (R,P): z R Gxz + P Bx, y P ; x R
    sweep<n, kPT, 2, false>(Gxy, A, line);
    __syncthreads();
    sweep<n, kRT, 1, false>(A, Y, line);
    __syncthreads();
    sweep<n, kRT, 2, false>(Gxz, A, line);
    __syncthreads();
    sweep<n, kPT, 2, true>(Bx, A, line);
    __syncthreads();
    sweep<n, kPT, 1, true>(A, Y, line);
    __syncthreads();
    sweep<n, kRT, 0, true>(Y, W, line);
    __syncthreads();
    if (active) {
#pragma unroll
      for (int i = 0; i < n; ++i)
        if (!constrained(d, I0 + i, J, K)) atomic_add(a.dst + row + i, W[i + n * line]);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Tangent coefficient fields of the LAW 5 operator at the linearisation point, built once
// per linearisation for the register-resident kernel's LAW 6: out[cell][8][n^3] =
//   c   = (rho_cp / dt + d(rho_cp)/dT (T_lin - T_old) / dt) JxW + d(rho_cp)/dT (b.grad T_lin)
//   k, rho_cp b (3), dk grad_ref T_lin (3)
// with b = JxW J^-1 v and the gas-liquid weight w from a.cf (LAW 5 layout {w, 0, b}).
// ---------------------------------------------------------------------------
template <int n, int GEO>
__global__ void __launch_bounds__(block_threads(n)) k_coef_tangent(CellArgs<double> a, double *out)
{
  using T = double;
  constexpr int n2 = n * n, n3 = n2 * n, CPB = cells_per_block(n);
  constexpr int NF = 8;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  const int cl = threadIdx.x / n2, line = threadIdx.x % n2;
  T *x = sm + cl * NF * n3, *t1 = x + n3, *t2 = x + 2 * n3, *Tq = x + 3 * n3, *Tx = x + 4 * n3,
    *Ty = x + 5 * n3, *Tz = x + 6 * n3, *To = x + 7 * n3;
  const MeshDims &d = a.d;
  const int64_t n_batches = (a.n_cells + CPB - 1) / CPB;
  for (int64_t batch = blockIdx.x; batch < n_batches; batch += gridDim.x) {
    const int64_t cell = batch * CPB + cl;
    const bool active = cell < a.n_cells;
    const int64_t cc = active ? cell : 0;
    const int cx = (int)(cc % d.m[0]);
    const int cy = (int)((cc / d.m[0]) % d.m[1]);
    const int cz = (int)(cc / ((int64_t)d.m[0] * d.m[1]));
    const int j = line % n, k = line / n;
    const int I0 = d.p * cx, J = d.p * cy + j, K = d.p * cz + k;
    const int64_t row = (int64_t)d.nd[0] * (J + (int64_t)d.nd[1] * K) + I0;
    T xv[n];
    gather_xline<n>(d, row, I0, J, K, false, a.Tl, xv, active);
#pragma unroll
    for (int i = 0; i < n; ++i) x[i + n * line] = xv[i];
    if (a.m.need_told) {
      gather_xline<n>(d, row, I0, J, K, false, a.To, xv, active);
#pragma unroll
      for (int i = 0; i < n; ++i) To[i + n * line] = xv[i];
    }
    __syncthreads();
    if (a.m.need_told) eval_values<n>(To, t1, t2, To, line);
    eval_values<n>(x, t1, t2, Tq, line);
    eval_gradients<n>(Tq, Tx, Ty, Tz, line);
    if (active) {
#pragma unroll
      for (int r = 0; r < n; ++r) {
        const int q = line + n2 * r;
        T jxw, G[6];
        geo_at<n, GEO>(a.g, cc, q % n, (q / n) % n, q / n2, jxw, G);
        const T *cf = a.cf + cc * 5 * n3 + q;
        T rhocp, kk, drhocp, dk;
        mat_eval_w(a.m, Tq[q], __ldg(cf), rhocp, kk, drhocp, dk);
        const T b0 = __ldg(cf + 2 * n3), b1 = __ldg(cf + 3 * n3), b2 = __ldg(cf + 4 * n3);
        T c = a.m.idt * rhocp;
        if (a.m.need_told) c += a.m.idt * drhocp * (Tq[q] - To[q]);
        T *o = out + cc * 8 * n3 + q;
        o[0] = c * jxw + drhocp * (b0 * Tx[q] + b1 * Ty[q] + b2 * Tz[q]);
        o[n3] = kk;
        o[2 * n3] = rhocp * b0;
        o[3 * n3] = rhocp * b1;
        o[4 * n3] = rhocp * b2;
        o[5 * n3] = dk * Tx[q];
        o[6 * n3] = dk * Ty[q];
        o[7 * n3] = dk * Tz[q];
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Tangent fields of the linear-k law at the linearisation point, built once per
// linearisation for the register-resident kernel's LAW 7: out[cell][4][n^3] =
// {k_l + k1 T_lin, k1 grad_ref T_lin} (the 7 T_lin sweeps of every LAW 1 application).
// ---------------------------------------------------------------------------
template <int n, int GEO>
__global__ void __launch_bounds__(block_threads(n)) k_coef_lineark(CellArgs<double> a, double *out)
{
  using T = double;
  constexpr int n2 = n * n, n3 = n2 * n, CPB = cells_per_block(n);
  constexpr int NF = 7;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  const int cl = threadIdx.x / n2, line = threadIdx.x % n2;
  T *x = sm + cl * NF * n3, *t1 = x + n3, *t2 = x + 2 * n3, *Tq = x + 3 * n3, *Tx = x + 4 * n3,
    *Ty = x + 5 * n3, *Tz = x + 6 * n3;
  const MeshDims &d = a.d;
  const int64_t n_batches = (a.n_cells + CPB - 1) / CPB;
  for (int64_t batch = blockIdx.x; batch < n_batches; batch += gridDim.x) {
    const int64_t cell = batch * CPB + cl;
    const bool active = cell < a.n_cells;
    const int64_t cc = active ? cell : 0;
    const int cx = (int)(cc % d.m[0]);
    const int cy = (int)((cc / d.m[0]) % d.m[1]);
    const int cz = (int)(cc / ((int64_t)d.m[0] * d.m[1]));
    const int j = line % n, k = line / n;
    const int I0 = d.p * cx, J = d.p * cy + j, K = d.p * cz + k;
    const int64_t row = (int64_t)d.nd[0] * (J + (int64_t)d.nd[1] * K) + I0;
    T xv[n];
    gather_xline<n>(d, row, I0, J, K, false, a.Tl, xv, active);
#pragma unroll
    for (int i = 0; i < n; ++i) x[i + n * line] = xv[i];
    __syncthreads();
    eval_values<n>(x, t1, t2, Tq, line);
    eval_gradients<n>(Tq, Tx, Ty, Tz, line);
    if (active) {
#pragma unroll
      for (int r = 0; r < n; ++r) {
        const int q = line + n2 * r;
        T *o = out + cc * 4 * n3 + q;
        o[0] = a.m.k_l + a.m.k1 * Tq[q];
        o[n3] = a.m.k1 * Tx[q];
        o[2 * n3] = a.m.k1 * Ty[q];
        o[3 * n3] = a.m.k1 * Tz[q];
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Values of the heaviside field H and the velocity field v (component-major, 3 x N) at the
// quadrature points, sum-factorised: cf[cell][0][q] = H (1 without a field),
// cf[cell][2 + e][q] = v_e (0 without a field); the per-point coefficient set-up then reads
// them in place.
// ---------------------------------------------------------------------------
template <int n>
__global__ void __launch_bounds__(block_threads(n)) k_field_values(CellArgs<double> a,
                                                                   const double *H,
                                                                   const double *vel,
                                                                   int64_t n_dofs, double *cf)
{
  using T = double;
  constexpr int n2 = n * n, n3 = n2 * n, CPB = cells_per_block(n);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  const int cl = threadIdx.x / n2, line = threadIdx.x % n2;
  T *u = sm + cl * 4 * n3, *t1 = u + n3, *t2 = u + 2 * n3, *vq = u + 3 * n3;
  const MeshDims &d = a.d;
  const int64_t n_batches = (a.n_cells + CPB - 1) / CPB;
  for (int64_t batch = blockIdx.x; batch < n_batches; batch += gridDim.x) {
    const int64_t cell = batch * CPB + cl;
    const bool active = cell < a.n_cells;
    const int64_t cc = active ? cell : 0;
    const int cx = (int)(cc % d.m[0]);
    const int cy = (int)((cc / d.m[0]) % d.m[1]);
    const int cz = (int)(cc / ((int64_t)d.m[0] * d.m[1]));
    const int j = line % n, k = line / n;
    const int I0 = d.p * cx, J = d.p * cy + j, K = d.p * cz + k;
    const int64_t row = (int64_t)d.nd[0] * (J + (int64_t)d.nd[1] * K) + I0;
    for (int f = 0; f < 4; ++f) {
      const double *g = f == 0 ? H : (vel ? vel + (int64_t)(f - 1) * n_dofs : nullptr);
      const int slot = f == 0 ? 0 : f + 1;
      if (!g) {
        if (active)
#pragma unroll
          for (int r = 0; r < n; ++r) cf[cc * 5 * n3 + slot * n3 + line + n2 * r] = f == 0 ? 1.0 : 0.0;
        continue;
      }
      T x[n];
      gather_xline<n>(d, row, I0, J, K, false, g, x, active);
#pragma unroll
      for (int i = 0; i < n; ++i) u[i + n * line] = x[i];
      __syncthreads();
      eval_values<n>(u, t1, t2, vq, line);
      if (active)
#pragma unroll
        for (int r = 0; r < n; ++r) cf[cc * 5 * n3 + slot * n3 + line + n2 * r] = vq[line + n2 * r];
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// L2 norm: sum over cells and q of u(q)^2 JxW (u read plain)
// ---------------------------------------------------------------------------
template <int n, int GEO>
__global__ void __launch_bounds__(block_threads(n)) k_norm(CellArgs<double> a)
{
  using T = double;
  constexpr int n2 = n * n, n3 = n2 * n, CPB = cells_per_block(n);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *sm = reinterpret_cast<T *>(smem_raw);
  const int cl = threadIdx.x / n2, line = threadIdx.x % n2;
  T *u = sm + cl * 4 * n3, *t1 = u + n3, *t2 = u + 2 * n3, *vq = u + 3 * n3;
  const MeshDims &d = a.d;
  double acc = 0.0;
  const int64_t n_batches = (a.n_cells + CPB - 1) / CPB;
  for (int64_t batch = blockIdx.x; batch < n_batches; batch += gridDim.x) {
    const int64_t cell = batch * CPB + cl;
    const bool active = cell < a.n_cells;
    const int64_t cc = active ? cell : 0;
    const int cx = (int)(cc % d.m[0]);
    const int cy = (int)((cc / d.m[0]) % d.m[1]);
    const int cz = (int)(cc / ((int64_t)d.m[0] * d.m[1]));
    const int j = line % n, k = line / n;
    const int I0 = d.p * cx, J = d.p * cy + j, K = d.p * cz + k;
    const int64_t row = (int64_t)d.nd[0] * (J + (int64_t)d.nd[1] * K) + I0;
    T x[n];
    gather_xline<n>(d, row, I0, J, K, false, a.src, x, active);
#pragma unroll
    for (int i = 0; i < n; ++i) u[i + n * line] = x[i];
    __syncthreads();
    eval_values<n>(u, t1, t2, vq, line);
    if (active) {
#pragma unroll
      for (int r = 0; r < n; ++r) {
        const int q = line + n2 * r;
        T jxw, G[6];
        geo_at<n, GEO>(a.g, cc, q % n, (q / n) % n, q / n2, jxw, G);
        acc += vq[q] * vq[q] * jxw;
      }
    }
    __syncthreads();
  }
  double v[1] = {acc}, tot[1];
  if (grid_sum<1>(v, a.partials, a.counter, tot)) *a.out = tot[0];
}

// shared-memory bytes of each kernel
template <int n, typename T, int LAW> constexpr size_t smem_vmult()
{
  return sizeof(T) * cells_per_block(n) * vmult_arrays<LAW>() * n * n * n;
}
template <int n> constexpr size_t smem_rhs() { return sizeof(double) * cells_per_block(n) * 9 * n * n * n; }
template <int n> constexpr size_t smem_diag() { return sizeof(double) * cells_per_block(n) * 16 * n * n * n; }
template <int n> constexpr size_t smem_norm() { return sizeof(double) * cells_per_block(n) * 4 * n * n * n; }
template <int n> constexpr size_t smem_coef_tangent() { return sizeof(double) * cells_per_block(n) * 8 * n * n * n; }
template <int n> constexpr size_t smem_coef_lineark() { return sizeof(double) * cells_per_block(n) * 7 * n * n * n; }

}  // namespace mpdg
