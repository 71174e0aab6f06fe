// Heat operator on a box mesh with refined cells and hanging-node constraints.
//
// The mesh: a box of coarse cells, each refined uniformly to its level, neighbouring coarse
// cells differing by one level at most (the 2:1 balance of the meshes refine_grid in
// source/utilities/amr.cpp:18-41 produces); the GPU operator takes one level for now.
// A node of a refined cell that lies on a face or an edge of an unrefined neighbour and is
// not one of its nodes hangs; its value is the neighbour's FE_Q(p) interpolant there, the
// rule of DoFTools::make_hanging_node_constraints that MeltPoolDG merges into its Dirichlet
// constraints (include/meltpooldg/utilities/constraints.hpp:111-132).
//
// The cell kernel applies the constraints inside the cell, from a per-cell code: a refined
// cell with a hanging face or edge gathers the unrefined neighbour's face or edge DoFs at the
// same local indices and interpolates them in place with the 1D child matrices
// I_s[j][a] = l_a((s + xi_j)/2), one direction at a time (lines along d on a hanging face
// normal to another direction, or on a hanging edge parallel to d); the scatter applies the
// transposes in the reverse order. One CTA of (p+1)^3 threads per cell, every sweep through
// shared memory: the first GPU form of this path, written for parity.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <initializer_list>
#include <new>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <map>
#include <mutex>
#include <vector>

#include "../../include/mpdg_heat.h"
#include "fe_tables.hpp"

int mpdg_internal_fail(int code, const char *msg);

namespace {

constexpr int kAmrMaxN = 5;  // degree <= 4
constexpr uint16_t kFineBit = 1u << 9;
constexpr int kLevelShift = 10;  // bits 10-12: the cell's refinement level
constexpr int kAmrMaxLevel = 6;

struct AmrArgs {
  const int *idx;
  const uint16_t *code;
  const uint8_t *mask;
  const double *src;
  const double *Tl;
  const double *q;  // create_rhs: the nodal heat source (nullable)
  // the linearisation point's values and reference gradients at the q-points, [cell][4][n^3],
  // built once per solve (nullable: the operator evaluates T_lin itself)
  const double *tf;
  double *dst;
  int64_t n_cells;
  double h[3];
  double cval, k0, k1;
  int tangent;
  double S[kAmrMaxN * kAmrMaxN];   // S[q][i] = l_i(x_q) at the Gauss points
  double Sd[kAmrMaxN * kAmrMaxN];  // Sd[q][i] = l_i'(x_q)
  double I[2][kAmrMaxN * kAmrMaxN];  // child interpolation I_s[j][a] = l_a((s + xi_j)/2)
  double w[kAmrMaxN];
};

int fail(int code, const std::string &msg) { return mpdg_internal_fail(code, msg.c_str()); }

#define TRY_AMR(call)              \
  do {                             \
    const int rc_ = (call);        \
    if (rc_ != MPDG_OK) return rc_; \
  } while (0)

// out[t] = sum_a M[o][a] in[line(a)], o = t's index along dir (M row-major n x n);
// transpose: sum_a M[a][o] in[line(a)]
template <int n>
__device__ __forceinline__ double line_sum(const double *M, const double *in, int t, int dir,
                                           bool transpose)
{
  const int st = dir == 0 ? 1 : (dir == 1 ? n : n * n);
  const int o = (t / st) % n;
  const int base = t - o * st;
  double v = 0.0;
#pragma unroll
  for (int a = 0; a < n; ++a) v += (transpose ? M[a * n + o] : M[o * n + a]) * in[base + a * st];
  return v;
}

// transposed line sum with the element-wise product of two 1D matrices:
// out_o = sum_a A[a][o] B[a][o] in[line(a)] (the closed-form diagonal's contractions)
template <int n>
__device__ __forceinline__ double line_sum_pp(const double *A, const double *B, const double *in,
                                              int t, int dir)
{
  const int st = dir == 0 ? 1 : (dir == 1 ? n : n * n);
  const int o = (t / st) % n;
  const int base = t - o * st;
  double v = 0.0;
#pragma unroll
  for (int a = 0; a < n; ++a) v += A[a * n + o] * B[a * n + o] * in[base + a * st];
  return v;
}

// in-place hanging interpolation of u along direction d (or its transpose)
template <int n>
__device__ __forceinline__ void hang_dir(double *u, double *tmp, int code, int d, const double *I,
                                         bool transpose, int t)
{
  const int ix[3] = {t % n, (t / n) % n, t / (n * n)};
  const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
  const int own1 = ((code >> d1) & 1) ? n - 1 : 0, own2 = ((code >> d2) & 1) ? n - 1 : 0;
  const bool f = (((code >> (3 + d1)) & 1) && ix[d1] == own1) ||
                 (((code >> (3 + d2)) & 1) && ix[d2] == own2) ||
                 (((code >> (6 + d)) & 1) && ix[d1] == own1 && ix[d2] == own2);
  tmp[t] = f ? line_sum<n>(I, u, t, d, transpose) : u[t];
  __syncthreads();
  u[t] = tmp[t];
  __syncthreads();
}

// values and reference gradients at the Gauss points of the nodal values u
template <int n>
__device__ __forceinline__ void evaluate(const AmrArgs &a, const double *u, double *val,
                                         double *gx, double *gy, double *gz, double *t1,
                                         double *t2, double *s1, double *s2, double *s3, int t)
{
  t1[t] = line_sum<n>(a.S, u, t, 0, false);
  t2[t] = line_sum<n>(a.Sd, u, t, 0, false);
  __syncthreads();
  s1[t] = line_sum<n>(a.S, t1, t, 1, false);
  s2[t] = line_sum<n>(a.Sd, t1, t, 1, false);
  s3[t] = line_sum<n>(a.S, t2, t, 1, false);
  __syncthreads();
  val[t] = line_sum<n>(a.S, s1, t, 2, false);
  gz[t] = line_sum<n>(a.Sd, s1, t, 2, false);
  gy[t] = line_sum<n>(a.S, s2, t, 2, false);
  gx[t] = line_sum<n>(a.S, s3, t, 2, false);
  __syncthreads();
}

// integration: u = S^T/Sd^T of (val, gx, gy, gz) along z, then y, then x
template <int n>
__device__ __forceinline__ void integrate_cell(const AmrArgs &a, double *u, const double *val,
                                               const double *gx, const double *gy,
                                               const double *gz, double *t1, double *t2,
                                               double *s1, double *s2, double *s3, int t)
{
  s1[t] = line_sum<n>(a.S, val, t, 2, true) + line_sum<n>(a.Sd, gz, t, 2, true);
  s2[t] = line_sum<n>(a.S, gx, t, 2, true);
  s3[t] = line_sum<n>(a.S, gy, t, 2, true);
  __syncthreads();
  t1[t] = line_sum<n>(a.S, s1, t, 1, true) + line_sum<n>(a.Sd, s3, t, 1, true);
  t2[t] = line_sum<n>(a.S, s2, t, 1, true);
  __syncthreads();
  u[t] = line_sum<n>(a.S, t1, t, 0, true) + line_sum<n>(a.Sd, t2, t, 0, true);
  __syncthreads();
}

// the cell's edge length factor 2^-level (bits 10-12 of the code; 0 for a coarse cell)
__device__ __forceinline__ double cell_size(int code)
{
  return ldexp(1.0, -((code >> kLevelShift) & 7));
}

// Apply the cell operator to the node values u (shared, overwritten with the integrated
// result, before the transposed hanging interpolation); Tv, Tx, Ty, Tz hold the linearisation
// point's values and reference gradients at the q-points when a.tangent.
template <int n>
__device__ __forceinline__ void apply_cell(const AmrArgs &a, double size, double *u,
                                           const double *Tv, const double *Tx, const double *Ty,
                                           const double *Tz, double *val, double *gx, double *gy,
                                           double *gz, double *t1, double *t2, double *s1,
                                           double *s2, double *s3, int t)
{
  evaluate<n>(a, u, val, gx, gy, gz, t1, t2, s1, s2, s3, t);
  // quadrature point t: rho_cp/dt u and the flux k grad(u) (+ k1 grad(T_lin) u)
  {
    const int qx = t % n, qy = (t / n) % n, qz = t / (n * n);
    const double hx = a.h[0] * size, hy = a.h[1] * size, hz = a.h[2] * size;
    const double jxw = a.w[qx] * a.w[qy] * a.w[qz] * hx * hy * hz;
    const double k = a.tangent ? a.k0 + a.k1 * Tv[t] : a.k0;
    double fx = k * gx[t] / hx, fy = k * gy[t] / hy, fz = k * gz[t] / hz;
    if (a.tangent) {
      fx += a.k1 * Tx[t] / hx * val[t];
      fy += a.k1 * Ty[t] / hy * val[t];
      fz += a.k1 * Tz[t] / hz * val[t];
    }
    val[t] = a.cval * val[t] * jxw;
    gx[t] = fx * jxw / hx;
    gy[t] = fy * jxw / hy;
    gz[t] = fz * jxw / hz;
  }
  __syncthreads();
  integrate_cell<n>(a, u, val, gx, gy, gz, t1, t2, s1, s2, s3, t);
}

template <int n>
__global__ void k_amr_vmult(const AmrArgs a)
{
  constexpr int n3 = n * n * n;
  __shared__ double u[n3], T[n3], tmp[n3], t1[n3], t2[n3], s1[n3], s2[n3], s3[n3];
  __shared__ double val[n3], gx[n3], gy[n3], gz[n3], Tv[n3], Tx[n3], Ty[n3], Tz[n3];
  const int t = threadIdx.x;
  for (int64_t c = blockIdx.x; c < a.n_cells; c += gridDim.x) {
    const int code = a.code[c];
    const int dof = a.idx[c * n3 + t];
    const bool hang = (code & 0x1F8) != 0;
    const double size = cell_size(code);
    const bool eval_T = a.tangent && !a.tf;
    u[t] = a.mask[dof] ? 0.0 : a.src[dof];
    if (eval_T) T[t] = a.Tl[dof];
    if (a.tangent && a.tf) {
      const double *f = a.tf + c * 4 * n3;
      Tv[t] = f[t];
      Tx[t] = f[n3 + t];
      Ty[t] = f[2 * n3 + t];
      Tz[t] = f[3 * n3 + t];
    }
    __syncthreads();
    if (hang) {
      for (int d = 0; d < 3; ++d) {
        const double *I = a.I[(code >> d) & 1];
        hang_dir<n>(u, tmp, code, d, I, false, t);
        if (eval_T) hang_dir<n>(T, tmp, code, d, I, false, t);
      }
    }
    if (eval_T) evaluate<n>(a, T, Tv, Tx, Ty, Tz, t1, t2, s1, s2, s3, t);
    apply_cell<n>(a, size, u, Tv, Tx, Ty, Tz, val, gx, gy, gz, t1, t2, s1, s2, s3, t);
    if (hang) {
      for (int d = 2; d >= 0; --d) hang_dir<n>(u, tmp, code, d, a.I[(code >> d) & 1], true, t);
    }
    if (!a.mask[dof]) atomicAdd(a.dst + dof, u[t]);
    __syncthreads();
  }
}

// the linearisation point's values and reference gradients at the q-points of every cell
// (hanging interpolation applied), [cell][4][n^3]: the operator's T_lin evaluation, once per solve
template <int n>
__global__ void k_amr_tfields(const AmrArgs a, double *tf)
{
  constexpr int n3 = n * n * n;
  __shared__ double T[n3], tmp[n3], t1[n3], t2[n3], s1[n3], s2[n3], s3[n3];
  __shared__ double Tv[n3], Tx[n3], Ty[n3], Tz[n3];
  const int t = threadIdx.x;
  for (int64_t c = blockIdx.x; c < a.n_cells; c += gridDim.x) {
    const int code = a.code[c];
    T[t] = a.Tl[a.idx[c * n3 + t]];
    __syncthreads();
    if ((code & 0x1F8) != 0)
      for (int d = 0; d < 3; ++d) hang_dir<n>(T, tmp, code, d, a.I[(code >> d) & 1], false, t);
    evaluate<n>(a, T, Tv, Tx, Ty, Tz, t1, t2, s1, s2, s3, t);
    double *f = tf + c * 4 * n3;
    f[t] = Tv[t];
    f[n3 + t] = Tx[t];
    f[2 * n3 + t] = Ty[t];
    f[3 * n3 + t] = Tz[t];
    __syncthreads();
  }
}

// diag(F^T A_e F) per cell at its gathered DoFs (distinct within a cell), by applying the
// cell operator to the cell's unit vectors (a cell on a hanging interface has no closed form)
template <int n>
__global__ void k_amr_diag(const AmrArgs a)
{
  constexpr int n3 = n * n * n;
  __shared__ double u[n3], T[n3], tmp[n3], t1[n3], t2[n3], s1[n3], s2[n3], s3[n3];
  __shared__ double val[n3], gx[n3], gy[n3], gz[n3], Tv[n3], Tx[n3], Ty[n3], Tz[n3];
  const int t = threadIdx.x;
  for (int64_t c = blockIdx.x; c < a.n_cells; c += gridDim.x) {
    const int code = a.code[c];
    const int dof = a.idx[c * n3 + t];
    const bool hang = (code & 0x1F8) != 0;
    const double size = cell_size(code);
    if (a.tangent) {
      T[t] = a.Tl[dof];
      __syncthreads();
      if (hang)
        for (int d = 0; d < 3; ++d) hang_dir<n>(T, tmp, code, d, a.I[(code >> d) & 1], false, t);
      evaluate<n>(a, T, Tv, Tx, Ty, Tz, t1, t2, s1, s2, s3, t);
    }
    double mine = 0.0;
    if (!hang) {
      // closed form: diag_i = sum_q [F0 P P P + F_x Q P P + F_y P Q P + F_z P P Q
      //                              + G_x R P P + G_y P R P + G_z P P R](q, i)
      // with P = S o S, Q = Sd o Sd, R = S o Sd (element-wise, [q][i]) along x, y, z and the
      // point factors of apply_cell: F0 = JxW rho_cp/dt, F_d = JxW k / h_d^2,
      // G_d = JxW k1 dT/dxi_d / h_d^2 (the tangent's k1 grad(T_lin) u term)
      {
        const int qx = t % n, qy = (t / n) % n, qz = t / (n * n);
        const double hx = a.h[0] * size, hy = a.h[1] * size, hz = a.h[2] * size;
        const double jxw = a.w[qx] * a.w[qy] * a.w[qz] * hx * hy * hz;
        const double k = a.tangent ? a.k0 + a.k1 * Tv[t] : a.k0;
        val[t] = jxw * a.cval;
        gx[t] = jxw * k / (hx * hx);
        gy[t] = jxw * k / (hy * hy);
        gz[t] = jxw * k / (hz * hz);
        t1[t] = a.tangent ? jxw * a.k1 * Tx[t] / (hx * hx) : 0.0;
        t2[t] = a.tangent ? jxw * a.k1 * Ty[t] / (hy * hy) : 0.0;
        s1[t] = a.tangent ? jxw * a.k1 * Tz[t] / (hz * hz) : 0.0;
      }
      __syncthreads();
      const double *S = a.S, *D = a.Sd;
      // along z: the five (x, y) matrix pairs that remain
      s2[t] = line_sum_pp<n>(S, S, val, t, 2) + line_sum_pp<n>(D, D, gz, t, 2) +
              line_sum_pp<n>(S, D, s1, t, 2);            // (P, P)
      s3[t] = line_sum_pp<n>(S, S, gx, t, 2);            // (Q, P)
      u[t] = line_sum_pp<n>(S, S, gy, t, 2);             // (P, Q)
      tmp[t] = line_sum_pp<n>(S, S, t1, t, 2);           // (R, P)
      T[t] = line_sum_pp<n>(S, S, t2, t, 2);             // (P, R)
      __syncthreads();
      // along y
      val[t] = line_sum_pp<n>(S, S, s2, t, 1) + line_sum_pp<n>(D, D, u, t, 1) +
               line_sum_pp<n>(S, D, T, t, 1);            // x: P
      gx[t] = line_sum_pp<n>(S, S, s3, t, 1);            // x: Q
      gy[t] = line_sum_pp<n>(S, S, tmp, t, 1);           // x: R
      __syncthreads();
      mine = line_sum_pp<n>(S, S, val, t, 0) + line_sum_pp<n>(D, D, gx, t, 0) +
             line_sum_pp<n>(S, D, gy, t, 0);
      __syncthreads();
    } else {
      // a cell on a hanging interface: the cell operator applied to its unit vectors
      for (int j = 0; j < n3; ++j) {
        u[t] = t == j ? 1.0 : 0.0;
        __syncthreads();
        for (int d = 0; d < 3; ++d) hang_dir<n>(u, tmp, code, d, a.I[(code >> d) & 1], false, t);
        apply_cell<n>(a, size, u, Tv, Tx, Ty, Tz, val, gx, gy, gz, t1, t2, s1, s2, s3, t);
        for (int d = 2; d >= 0; --d) hang_dir<n>(u, tmp, code, d, a.I[(code >> d) & 1], true, t);
        if (t == j) mine = u[t];
        __syncthreads();
      }
    }
    if (!a.mask[dof]) atomicAdd(a.dst + dof, mine);
    __syncthreads();
  }
}

// dst += -R(T) (create_rhs): T = a.Tl, T_old = a.src, the nodal source a.q (nullable), all
// read plain and interpolated by the hanging rule; Dirichlet rows untouched
template <int n>
__global__ void k_amr_rhs(const AmrArgs a)
{
  constexpr int n3 = n * n * n;
  __shared__ double u[n3], T[n3], tmp[n3], t1[n3], t2[n3], s1[n3], s2[n3], s3[n3];
  __shared__ double val[n3], gx[n3], gy[n3], gz[n3], To[n3], Q[n3], Tov[n3], Qv[n3];
  const int t = threadIdx.x;
  for (int64_t c = blockIdx.x; c < a.n_cells; c += gridDim.x) {
    const int code = a.code[c];
    const int dof = a.idx[c * n3 + t];
    const bool hang = (code & 0x1F8) != 0;
    const double size = cell_size(code);
    T[t] = a.Tl[dof];
    To[t] = a.src[dof];
    Q[t] = a.q ? a.q[dof] : 0.0;
    __syncthreads();
    if (hang) {
      for (int d = 0; d < 3; ++d) {
        const double *I = a.I[(code >> d) & 1];
        hang_dir<n>(T, tmp, code, d, I, false, t);
        hang_dir<n>(To, tmp, code, d, I, false, t);
        hang_dir<n>(Q, tmp, code, d, I, false, t);
      }
    }
    // values of T_old and the source at the q-points (gx.. as scratch), then T's values and
    // gradients
    evaluate<n>(a, To, Tov, gx, gy, gz, t1, t2, s1, s2, s3, t);
    evaluate<n>(a, Q, Qv, gx, gy, gz, t1, t2, s1, s2, s3, t);
    evaluate<n>(a, T, val, gx, gy, gz, t1, t2, s1, s2, s3, t);
    {
      const int qx = t % n, qy = (t / n) % n, qz = t / (n * n);
      const double hx = a.h[0] * size, hy = a.h[1] * size, hz = a.h[2] * size;
      const double jxw = a.w[qx] * a.w[qy] * a.w[qz] * hx * hy * hz;
      const double k = a.k0 + a.k1 * val[t];
      const double v = a.cval * (val[t] - Tov[t]) - Qv[t];
      val[t] = -v * jxw;
      gx[t] = -k * gx[t] / (hx * hx) * jxw;
      gy[t] = -k * gy[t] / (hy * hy) * jxw;
      gz[t] = -k * gz[t] / (hz * hz) * jxw;
    }
    __syncthreads();
    integrate_cell<n>(a, u, val, gx, gy, gz, t1, t2, s1, s2, s3, t);
    if (hang) {
      for (int d = 2; d >= 0; --d) hang_dir<n>(u, tmp, code, d, a.I[(code >> d) & 1], true, t);
    }
    if (!a.mask[dof]) atomicAdd(a.dst + dof, u[t]);
    __syncthreads();
  }
}

// vector kernels of the Krylov solve on the refined mesh (sums by block reduction and one
// atomic add per block into a device scalar)
__global__ void k_amr_dot(int64_t n, const double *__restrict__ a, const double *__restrict__ b,
                          double *out)
{
  __shared__ double red[32];
  double v = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    v += a[i] * b[i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) atomicAdd(out, v);
  }
}

// y = a x + b y (x, y may alias nothing else)
__global__ void k_amr_axpby(int64_t n, double a, const double *__restrict__ x, double b, double *y)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    y[i] = a * x[i] + b * y[i];
}

// z = D r
__global__ void k_amr_mul(int64_t n, const double *__restrict__ D, const double *__restrict__ r,
                          double *z)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    z[i] = D[i] * r[i];
}

// d <- |d| > 1e-10 ? 1/d : 1 (Dirichlet DoFs, left zero, become 1)
__global__ void k_amr_invert(int64_t n, double *d)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    d[i] = fabs(d[i]) > 1e-10 ? 1.0 / d[i] : 1.0;
}

// linear predictor (1 + r) T - r T_old, history commit T_old <- T, Dirichlet DoFs zero
__global__ void k_amr_predict(int64_t n, double r, double *T, double *To,
                              const uint8_t *__restrict__ mask)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double t = T[i], pred = (1.0 + r) * t - r * To[i];
    To[i] = t;
    T[i] = mask[i] ? 0.0 : pred;
  }
}

__global__ void k_amr_zero(int64_t n, double *p)
{
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    p[i] = 0.0;
}

}  // namespace

struct mpdg_amr {
  int p = 1, n = 2, device = -1;
  int m[3] = {0, 0, 0};
  double lo[3] = {0, 0, 0}, h[3] = {0, 0, 0};
  int64_t n_cells = 0, n_dofs = 0;
  int max_level = 0;
  std::vector<int64_t> cell_dofs;  // n_cells x n^3
  std::vector<uint16_t> codes;
  std::vector<double> dof_pos;     // n_dofs x 3, physical
  std::vector<uint8_t> mask;
  mpdg_material mat{};
  double dt = 0.0;
  bool mat_set = false;
  int *d_idx = nullptr;
  uint16_t *d_code = nullptr;
  uint8_t *d_mask = nullptr;
  // Krylov / step workspace (n_dofs each) and a device scalar for the sums
  double *w[7] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  double *d_sum = nullptr;
  double *tf = nullptr;  // tangent fields of the solve's linearisation point, [cell][4][n^3]
};

namespace {

using Key = std::array<int64_t, 3>;

Key key_of(const double *x)
{
  return {std::llround(x[0] * 67108864.0), std::llround(x[1] * 67108864.0),
          std::llround(x[2] * 67108864.0)};
}

void release(mpdg_amr *h)
{
  if (h->d_idx) cudaFree(h->d_idx);
  if (h->d_code) cudaFree(h->d_code);
  if (h->d_mask) cudaFree(h->d_mask);
  h->d_idx = nullptr;
  h->d_code = nullptr;
  h->d_mask = nullptr;
  for (double *&v : h->w) {
    if (v) cudaFree(v);
    v = nullptr;
  }
  if (h->d_sum) cudaFree(h->d_sum);
  h->d_sum = nullptr;
  if (h->tf) cudaFree(h->tf);
  h->tf = nullptr;
}

// the host description: active cells, node numbering, hanging nodes, DoFs, cell data
int build_host(mpdg_amr *h, const mpdg_mesh_desc *desc, const uint8_t *refine)
{
  const int n = h->n, n3 = n * n * n;
  const int mx = h->m[0], my = h->m[1], mz = h->m[2];
  auto level = [&](int ix, int iy, int iz) {
    return (int)refine[(size_t)ix + (size_t)mx * (iy + (size_t)my * iz)];
  };
  auto inside = [&](int ix, int iy, int iz) {
    return ix >= 0 && iy >= 0 && iz >= 0 && ix < mx && iy < my && iz < mz;
  };
  // 2:1 balance across faces, edges and vertices
  for (int iz = 0; iz < mz; ++iz)
    for (int iy = 0; iy < my; ++iy)
      for (int ix = 0; ix < mx; ++ix) {
        if (level(ix, iy, iz) > kAmrMaxLevel)
          return fail(MPDG_ERR_INVALID_ARGUMENT, "refinement level above the maximum");
        for (int dz = -1; dz <= 1; ++dz)
          for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx)
              if (inside(ix + dx, iy + dy, iz + dz) &&
                  std::abs(level(ix + dx, iy + dy, iz + dz) - level(ix, iy, iz)) > 1)
                return fail(MPDG_ERR_INVALID_ARGUMENT,
                            "neighbouring coarse cells differ by more than one level");
      }
  mpdg::Tables1D tb = mpdg::make_tables(n);
  const double *xi = tb.xl;
  // active cells: every coarse cell refined uniformly to its level
  struct Cell {
    double o[3];
    double size;
    int level;
    int64_t g[3];  // index on its level's lattice
  };
  std::vector<Cell> cells;
  std::unordered_map<int64_t, int64_t> cell_at;  // (level, lattice index) -> cell
  auto lattice_key = [](int L, int64_t gx, int64_t gy, int64_t gz) {
    return (((int64_t)L * 1048576 + gz) * 1048576 + gy) * 1048576 + gx;
  };
  for (int iz = 0; iz < mz; ++iz)
    for (int iy = 0; iy < my; ++iy)
      for (int ix = 0; ix < mx; ++ix) {
        const int L = level(ix, iy, iz), k = 1 << L;
        for (int sz = 0; sz < k; ++sz)
          for (int sy = 0; sy < k; ++sy)
            for (int sx = 0; sx < k; ++sx) {
              Cell cl{{ix + (double)sx / k, iy + (double)sy / k, iz + (double)sz / k}, 1.0 / k, L,
                      {(int64_t)ix * k + sx, (int64_t)iy * k + sy, (int64_t)iz * k + sz}};
              cell_at[lattice_key(L, cl.g[0], cl.g[1], cl.g[2])] = (int64_t)cells.size();
              cells.push_back(cl);
            }
      }
  auto find_cell = [&](int L, int64_t gx, int64_t gy, int64_t gz) -> int64_t {
    if (L < 0 || gx < 0 || gy < 0 || gz < 0) return -1;
    auto it = cell_at.find(lattice_key(L, gx, gy, gz));
    return it == cell_at.end() ? -1 : it->second;
  };
  const int64_t nc = (int64_t)cells.size();
  // nodes by position key (coarse-cell units)
  std::vector<std::pair<Key, int64_t>> ent((size_t)nc * n3);
  std::vector<double> pos((size_t)nc * n3 * 3);
  for (int64_t c = 0; c < nc; ++c)
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          const int64_t e = c * n3 + i + n * (j + n * k);
          double *x = &pos[(size_t)e * 3];
          x[0] = cells[c].o[0] + cells[c].size * xi[i];
          x[1] = cells[c].o[1] + cells[c].size * xi[j];
          x[2] = cells[c].o[2] + cells[c].size * xi[k];
          ent[(size_t)e] = {key_of(x), e};
        }
  std::sort(ent.begin(), ent.end());
  std::vector<int64_t> node_of((size_t)nc * n3);
  std::vector<int64_t> first;  // one entry per node: its first occurrence
  std::vector<Key> node_key;
  for (size_t a = 0; a < ent.size(); ++a) {
    if (a == 0 || ent[a].first != ent[a - 1].first) {
      first.push_back(ent[a].second);
      node_key.push_back(ent[a].first);
    }
    node_of[(size_t)ent[a].second] = (int64_t)first.size() - 1;
  }
  const int64_t n_nodes = (int64_t)first.size();
  // a node hangs when the coarsest cells whose closed boxes hold it (level l_min) do not have
  // it as a node; under the 2:1 balance its constraining nodes never hang
  std::vector<uint32_t> level_bits((size_t)n_nodes, 0);  // levels of the cells that have it
  for (int64_t c = 0; c < nc; ++c)
    for (int l = 0; l < n3; ++l) level_bits[(size_t)node_of[c * n3 + l]] |= 1u << cells[c].level;
  std::vector<uint8_t> hanging((size_t)n_nodes, 0);
  const double tol = 1e-9;
  for (int64_t v = 0; v < n_nodes; ++v) {
    const double *x = &pos[(size_t)first[v] * 3];
    const int bx = (int)std::floor(x[0] + tol), by = (int)std::floor(x[1] + tol),
              bz = (int)std::floor(x[2] + tol);
    int lmin = 1 << 30;
    for (int dz = 0; dz >= -1; --dz)
      for (int dy = 0; dy >= -1; --dy)
        for (int dx = 0; dx >= -1; --dx) {
          const int cx = bx + dx, cy = by + dy, cz = bz + dz;
          if (!inside(cx, cy, cz)) continue;
          if (x[0] >= cx - tol && x[0] <= cx + 1 + tol && x[1] >= cy - tol &&
              x[1] <= cy + 1 + tol && x[2] >= cz - tol && x[2] <= cz + 1 + tol)
            lmin = std::min(lmin, level(cx, cy, cz));
        }
    hanging[v] = !((level_bits[v] >> lmin) & 1u);
  }
  // DoFs: the regular nodes ordered by (z, y, x)
  std::vector<int64_t> regular;
  for (int64_t v = 0; v < n_nodes; ++v)
    if (!hanging[v]) regular.push_back(v);
  std::sort(regular.begin(), regular.end(), [&](int64_t a, int64_t b) {
    const Key &ka = node_key[a], &kb = node_key[b];
    if (ka[2] != kb[2]) return ka[2] < kb[2];
    if (ka[1] != kb[1]) return ka[1] < kb[1];
    return ka[0] < kb[0];
  });
  std::vector<int64_t> dof_of((size_t)n_nodes, -1);
  for (size_t r = 0; r < regular.size(); ++r) dof_of[(size_t)regular[r]] = (int64_t)r;
  h->n_dofs = (int64_t)regular.size();
  h->n_cells = nc;
  h->dof_pos.resize((size_t)h->n_dofs * 3);
  h->mask.assign((size_t)h->n_dofs, 0);
  const int mm[3] = {mx, my, mz};
  for (int64_t r = 0; r < h->n_dofs; ++r) {
    const double *x = &pos[(size_t)first[(size_t)regular[r]] * 3];
    for (int d = 0; d < 3; ++d) {
      h->dof_pos[(size_t)r * 3 + d] = h->lo[d] + x[d] * h->h[d];
      if (((desc->dirichlet_mask >> (2 * d)) & 1) && std::fabs(x[d]) < tol) h->mask[r] = 1;
      if (((desc->dirichlet_mask >> (2 * d + 1)) & 1) && std::fabs(x[d] - mm[d]) < tol)
        h->mask[r] = 1;
    }
  }
  // per cell: gathered DoFs and the hanging code (the neighbours of its parent one level down)
  h->cell_dofs.assign((size_t)nc * n3, -1);
  h->codes.assign((size_t)nc, 0);
  h->max_level = 0;
  auto lin = [n](int i, int j, int k) { return i + n * (j + n * k); };
  for (int64_t c = 0; c < nc; ++c) {
    const Cell &cl = cells[c];
    int64_t *idx = &h->cell_dofs[(size_t)c * n3];
    for (int l = 0; l < n3; ++l) idx[l] = dof_of[(size_t)node_of[c * n3 + l]];
    h->max_level = std::max(h->max_level, cl.level);
    if (cl.level == 0) continue;
    int s[3];
    int64_t par[3];
    for (int d = 0; d < 3; ++d) {
      s[d] = (int)(cl.g[d] & 1);
      par[d] = cl.g[d] >> 1;
    }
    const int L = cl.level - 1;
    int code = kFineBit | (cl.level << kLevelShift);
    int step[3], own[3], other[3];
    for (int d = 0; d < 3; ++d) {
      step[d] = s[d] ? 1 : -1;
      own[d] = s[d] ? n - 1 : 0;
      other[d] = n - 1 - own[d];
    }
    int64_t face_nb[3], edge_nb[3];
    bool face[3], edge[3];
    for (int d = 0; d < 3; ++d) {
      int64_t q[3] = {par[0], par[1], par[2]};
      q[d] += step[d];
      face_nb[d] = find_cell(L, q[0], q[1], q[2]);
      face[d] = face_nb[d] >= 0;
    }
    for (int d = 0; d < 3; ++d) {
      const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
      int64_t q[3] = {par[0], par[1], par[2]};
      q[d1] += step[d1];
      q[d2] += step[d2];
      edge_nb[d] = find_cell(L, q[0], q[1], q[2]);
      edge[d] = edge_nb[d] >= 0 && !face[d1] && !face[d2];
    }
    int hb = 0;
    for (int d = 0; d < 3; ++d) hb |= (face[d] ? 1 << (3 + d) : 0) | (edge[d] ? 1 << (6 + d) : 0);
    if (hb) code |= hb | s[0] | (s[1] << 1) | (s[2] << 2);
    h->codes[(size_t)c] = (uint16_t)code;
    // gather the neighbour's face / edge DoFs at the same local indices
    for (int d = 0; d < 3; ++d) {
      if (!face[d]) continue;
      const int64_t nb = face_nb[d];
      const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
      for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b) {
          int i[3], jn[3];
          i[d] = own[d];
          i[d1] = a;
          i[d2] = b;
          jn[d] = other[d];
          jn[d1] = a;
          jn[d2] = b;
          idx[lin(i[0], i[1], i[2])] = dof_of[(size_t)node_of[nb * n3 + lin(jn[0], jn[1], jn[2])]];
        }
    }
    for (int d = 0; d < 3; ++d) {
      if (!edge[d]) continue;
      const int d1 = (d + 1) % 3, d2 = (d + 2) % 3;
      const int64_t nb = edge_nb[d];
      for (int a = 0; a < n; ++a) {
        int i[3], jn[3];
        i[d] = a;
        i[d1] = own[d1];
        i[d2] = own[d2];
        jn[d] = a;
        jn[d1] = other[d1];
        jn[d2] = other[d2];
        idx[lin(i[0], i[1], i[2])] = dof_of[(size_t)node_of[nb * n3 + lin(jn[0], jn[1], jn[2])]];
      }
    }
  }
  for (int64_t v : h->cell_dofs)
    if (v < 0 || v >= h->n_dofs)
      return fail(MPDG_ERR_INVALID_ARGUMENT, "hanging node left ungathered (unsupported mesh)");
  return MPDG_OK;
}

}  // namespace

extern "C" int mpdg_amr_create(const mpdg_mesh_desc *desc, const uint8_t *refine, int device,
                               mpdg_amr **out)
{
  if (!desc || !refine || !out) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (desc->degree < 1 || desc->degree > kAmrMaxN - 1)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "hanging-node meshes: degree 1..4");
  if (desc->perturb != 0.0)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "hanging-node meshes: affine boxes only");
  for (int d = 0; d < 3; ++d)
    if (desc->cells[d] < 1 || !(desc->hi[d] > desc->lo[d]))
      return fail(MPDG_ERR_INVALID_ARGUMENT, "invalid box");
  // Bound the host description before building it: active cells x (p+1)^3 gathered entries
  // (32-bit device indices), and lattice coordinates below 2^20 (the cell map's key packs
  // each of them into 20 bits).
  {
    const int64_t n3 = (int64_t)(desc->degree + 1) * (desc->degree + 1) * (desc->degree + 1);
    const int64_t n_coarse = (int64_t)desc->cells[0] * desc->cells[1] * desc->cells[2];
    int max_level = 0;
    int64_t entries = 0;
    for (int64_t c = 0; c < n_coarse; ++c) {
      const int L = refine[c];
      if (L > kAmrMaxLevel)
        return fail(MPDG_ERR_INVALID_ARGUMENT, "refinement level above the maximum");
      max_level = std::max(max_level, L);
      entries += ((int64_t)1 << (3 * L)) * n3;
      if (entries >= ((int64_t)1 << 31))
        return fail(MPDG_ERR_INVALID_ARGUMENT,
                    "hanging-node mesh too large (cells x (p+1)^3 must stay below 2^31)");
    }
    for (int d = 0; d < 3; ++d)
      if (((int64_t)desc->cells[d] << max_level) >= ((int64_t)1 << 20))
        return fail(MPDG_ERR_INVALID_ARGUMENT,
                    "hanging-node mesh: cells per direction x 2^level must stay below 2^20");
  }
  mpdg_amr *h = new (std::nothrow) mpdg_amr();
  if (!h) return fail(MPDG_ERR_OUT_OF_MEMORY, "hanging-node mesh: host allocation failed");
  h->p = desc->degree;
  h->n = desc->degree + 1;
  h->device = device;
  for (int d = 0; d < 3; ++d) {
    h->m[d] = desc->cells[d];
    h->lo[d] = desc->lo[d];
    h->h[d] = (desc->hi[d] - desc->lo[d]) / desc->cells[d];
  }
  int rc;
  try {
    rc = build_host(h, desc, refine);
  } catch (const std::bad_alloc &) {
    rc = fail(MPDG_ERR_OUT_OF_MEMORY, "hanging-node mesh: host allocation failed");
  } catch (const std::exception &e) {
    rc = fail(MPDG_ERR_INVALID_ARGUMENT, std::string("hanging-node mesh: ") + e.what());
  }
  if (rc != MPDG_OK) {
    delete h;
    return rc;
  }
  if (device >= 0 && h->n_cells * (int64_t)h->n * h->n * h->n >= ((int64_t)1 << 31)) {
    delete h;
    return fail(MPDG_ERR_INVALID_ARGUMENT, "hanging-node mesh too large for 32-bit cell data");
  }
  if (device >= 0) {
    const int n3 = h->n * h->n * h->n;
    std::vector<int> idx32(h->cell_dofs.begin(), h->cell_dofs.end());
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaMalloc(&h->d_idx, sizeof(int) * idx32.size());
    if (e == cudaSuccess) e = cudaMalloc(&h->d_code, sizeof(uint16_t) * h->codes.size());
    if (e == cudaSuccess) e = cudaMalloc(&h->d_mask, h->mask.size());
    if (e == cudaSuccess)
      e = cudaMemcpy(h->d_idx, idx32.data(), sizeof(int) * idx32.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(h->d_code, h->codes.data(), sizeof(uint16_t) * h->codes.size(),
                     cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
      e = cudaMemcpy(h->d_mask, h->mask.data(), h->mask.size(), cudaMemcpyHostToDevice);
    (void)n3;
    if (e != cudaSuccess) {
      release(h);
      delete h;
      return fail(e == cudaErrorMemoryAllocation ? MPDG_ERR_OUT_OF_MEMORY : MPDG_ERR_CUDA,
                  std::string("hanging-node mesh: ") + cudaGetErrorString(e));
    }
  }
  *out = h;
  return MPDG_OK;
}

extern "C" int mpdg_amr_destroy(mpdg_amr *h)
{
  if (!h) return MPDG_OK;
  if (h->device >= 0) {
    cudaSetDevice(h->device);
    release(h);
  }
  delete h;
  return MPDG_OK;
}

extern "C" int64_t mpdg_amr_n_dofs(const mpdg_amr *h) { return h ? h->n_dofs : -1; }
extern "C" int64_t mpdg_amr_n_cells(const mpdg_amr *h) { return h ? h->n_cells : -1; }

extern "C" int mpdg_amr_support_points(const mpdg_amr *h, double *xyz)
{
  if (!h || !xyz) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  std::memcpy(xyz, h->dof_pos.data(), sizeof(double) * h->dof_pos.size());
  return MPDG_OK;
}

extern "C" int mpdg_amr_constraint_mask(const mpdg_amr *h, uint8_t *mask)
{
  if (!h || !mask) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  std::memcpy(mask, h->mask.data(), h->mask.size());
  return MPDG_OK;
}

extern "C" int mpdg_amr_cell_data(const mpdg_amr *h, int64_t *dofs, uint16_t *codes)
{
  if (!h) return fail(MPDG_ERR_INVALID_ARGUMENT, "null handle");
  if (dofs) std::memcpy(dofs, h->cell_dofs.data(), sizeof(int64_t) * h->cell_dofs.size());
  if (codes) std::memcpy(codes, h->codes.data(), sizeof(uint16_t) * h->codes.size());
  return MPDG_OK;
}

extern "C" int mpdg_amr_set_material(mpdg_amr *h, const mpdg_material *m, double dt)
{
  if (!h || !m) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  if (m->law != MPDG_LAW_CONSTANT && m->law != MPDG_LAW_LINEAR_K)
    return fail(MPDG_ERR_NOT_SUPPORTED, "hanging-node meshes: constant or LINEAR_K law");
  if (dt == 0.0) return fail(MPDG_ERR_ZERO_TIME_INCREMENT, "time increment is zero");
  h->mat = *m;
  h->dt = dt;
  h->mat_set = true;
  return MPDG_OK;
}

namespace {

int check_device_vectors(std::initializer_list<const void *> ptrs)
{
  for (const void *ptr : ptrs) {
    if (!ptr) continue;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess || at.type != cudaMemoryTypeDevice)
      return fail(MPDG_ERR_INVALID_ARGUMENT, "vectors must be device memory");
  }
  return MPDG_OK;
}

// kernel arguments of the handle's operator at the linearisation point T_lin (LINEAR_K)
AmrArgs make_args(const mpdg_amr *h, const double *T_lin)
{
  const bool tangent = h->mat.law == MPDG_LAW_LINEAR_K && h->mat.k1 != 0.0;
  AmrArgs a;
  std::memset(&a, 0, sizeof(a));
  a.idx = h->d_idx;
  a.code = h->d_code;
  a.mask = h->d_mask;
  a.Tl = T_lin;
  a.n_cells = h->n_cells;
  for (int d = 0; d < 3; ++d) a.h[d] = h->h[d];
  a.cval = h->mat.rho_l * h->mat.cp_l / h->dt;
  a.k0 = h->mat.k_l;
  a.k1 = h->mat.law == MPDG_LAW_LINEAR_K ? h->mat.k1 : 0.0;
  a.tangent = tangent;
  const int n = h->n;
  mpdg::Tables1D tb = mpdg::make_tables(n);
  for (int q = 0; q < n; ++q) {
    a.w[q] = tb.wg[q];
    for (int i = 0; i < n; ++i) {
      a.S[q * n + i] = mpdg::lagrange(tb.xl, n, i, tb.xg[q]);
      a.Sd[q * n + i] = mpdg::lagrange_d(tb.xl, n, i, tb.xg[q]);
    }
  }
  for (int s2 = 0; s2 < 2; ++s2)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i)
        a.I[s2][j * n + i] = mpdg::lagrange(tb.xl, n, i, 0.5 * (s2 + tb.xl[j]));
  return a;
}

enum { CELL_VMULT = 0, CELL_DIAG = 1, CELL_RHS = 2 };

// a persistent grid of as many CTAs (one cell each at a time) as the SMs hold at once
template <typename K> int resident_grid(K kernel, int threads, int64_t n_cells)
{
  static std::mutex mu;
  static std::map<const void *, int> per_sm_of;  // per kernel
  static int sms = 0;
  int per_sm = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    if (sms == 0) {
      int dev = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    auto it = per_sm_of.find(reinterpret_cast<const void *>(kernel));
    if (it == per_sm_of.end()) {
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess ||
          per_sm < 1)
        per_sm = 16;
      per_sm_of[reinterpret_cast<const void *>(kernel)] = per_sm;
    } else {
      per_sm = it->second;
    }
  }
  return (int)std::min<int64_t>(n_cells, (int64_t)per_sm * sms);
}

template <int n>
void launch_n(int kind, const AmrArgs &a)
{
  constexpr int n3 = n * n * n;
  if (kind == CELL_VMULT) {
    k_amr_vmult<n><<<resident_grid(k_amr_vmult<n>, n3, a.n_cells), n3>>>(a);
  } else if (kind == CELL_DIAG) {
    k_amr_diag<n><<<resident_grid(k_amr_diag<n>, n3, a.n_cells), n3>>>(a);
  } else {
    k_amr_rhs<n><<<resident_grid(k_amr_rhs<n>, n3, a.n_cells), n3>>>(a);
  }
}

int launch_cells(const mpdg_amr *h, int kind, const AmrArgs &a)
{
  switch (h->n) {
    case 2: launch_n<2>(kind, a); break;
    case 3: launch_n<3>(kind, a); break;
    case 4: launch_n<4>(kind, a); break;
    case 5: launch_n<5>(kind, a); break;
    default: return fail(MPDG_ERR_INVALID_ARGUMENT, "degree");
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MPDG_OK : fail(MPDG_ERR_CUDA, cudaGetErrorString(e));
}

int ready(const mpdg_amr *h)
{
  if (h->device < 0) return fail(MPDG_ERR_INVALID_ARGUMENT, "host-only hanging-node mesh");
  if (!h->mat_set) return fail(MPDG_ERR_INVALID_ARGUMENT, "call mpdg_amr_set_material first");
  const cudaError_t e = cudaSetDevice(h->device);
  return e == cudaSuccess ? MPDG_OK : fail(MPDG_ERR_CUDA, cudaGetErrorString(e));
}

int sync_status()
{
  const cudaError_t e = cudaDeviceSynchronize();
  return e == cudaSuccess ? MPDG_OK : fail(MPDG_ERR_CUDA, cudaGetErrorString(e));
}

int vgrid(int64_t n) { return (int)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8)); }

// the tangent fields of T_lin into h->tf (for the applications of one solve)
int tfields_impl(mpdg_amr *h, const double *T_lin)
{
  const int64_t nf = h->n_cells * 4 * (int64_t)h->n * h->n * h->n;
  if (!h->tf) {
    const cudaError_t e = cudaMalloc(&h->tf, sizeof(double) * (size_t)nf);
    if (e != cudaSuccess) {
      h->tf = nullptr;
      return fail(MPDG_ERR_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
  }
  AmrArgs a = make_args(h, T_lin);
  const int64_t nc = h->n_cells;
  switch (h->n) {
    case 2: k_amr_tfields<2><<<resident_grid(k_amr_tfields<2>, 8, nc), 8>>>(a, h->tf); break;
    case 3: k_amr_tfields<3><<<resident_grid(k_amr_tfields<3>, 27, nc), 27>>>(a, h->tf); break;
    case 4: k_amr_tfields<4><<<resident_grid(k_amr_tfields<4>, 64, nc), 64>>>(a, h->tf); break;
    case 5: k_amr_tfields<5><<<resident_grid(k_amr_tfields<5>, 125, nc), 125>>>(a, h->tf); break;
    default: return fail(MPDG_ERR_INVALID_ARGUMENT, "degree");
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MPDG_OK : fail(MPDG_ERR_CUDA, cudaGetErrorString(e));
}

int vmult_impl(mpdg_amr *h, double *dst, const double *src, const double *T_lin,
               const double *tf = nullptr)
{
  AmrArgs a = make_args(h, T_lin);
  a.src = src;
  a.dst = dst;
  a.tf = a.tangent ? tf : nullptr;
  if (!a.tangent) a.Tl = src;
  k_amr_zero<<<vgrid(h->n_dofs), 256>>>(h->n_dofs, dst);
  return launch_cells(h, CELL_VMULT, a);
}

int diag_impl(mpdg_amr *h, double *inv, const double *T_lin)
{
  AmrArgs a = make_args(h, T_lin);
  a.dst = inv;
  k_amr_zero<<<vgrid(h->n_dofs), 256>>>(h->n_dofs, inv);
  TRY_AMR(launch_cells(h, CELL_DIAG, a));
  k_amr_invert<<<vgrid(h->n_dofs), 256>>>(h->n_dofs, inv);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? MPDG_OK : fail(MPDG_ERR_CUDA, cudaGetErrorString(e));
}

int rhs_impl(mpdg_amr *h, double *dst, const double *T, const double *T_old, const double *q)
{
  AmrArgs a = make_args(h, T);
  a.Tl = T;
  a.src = T_old;
  a.q = q;
  a.dst = dst;
  return launch_cells(h, CELL_RHS, a);
}

int ensure_workspace(mpdg_amr *h)
{
  for (double *&v : h->w)
    if (!v) {
      const cudaError_t e = cudaMalloc(&v, sizeof(double) * (size_t)h->n_dofs);
      if (e != cudaSuccess) {
        v = nullptr;
        return fail(MPDG_ERR_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
      }
    }
  if (!h->d_sum) {
    const cudaError_t e = cudaMalloc(&h->d_sum, sizeof(double));
    if (e != cudaSuccess) {
      h->d_sum = nullptr;
      return fail(MPDG_ERR_OUT_OF_MEMORY, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
  }
  return MPDG_OK;
}

int dot(mpdg_amr *h, const double *a, const double *b, double *out)
{
  cudaMemset(h->d_sum, 0, sizeof(double));
  k_amr_dot<<<vgrid(h->n_dofs), 256>>>(h->n_dofs, a, b, h->d_sum);
  const cudaError_t e = cudaMemcpy(out, h->d_sum, sizeof(double), cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? MPDG_OK : fail(MPDG_ERR_CUDA, cudaGetErrorString(e));
}

// Jacobi-CG (deal.II SolverCG semantics, ReductionControl) on the refined mesh: x from 0
int cg_impl(mpdg_amr *h, double *x, const double *b, const double *inv, const double *T_lin,
            double rel_tol, double abs_tol, int max_it, int *iterations)
{
  TRY_AMR(ensure_workspace(h));
  const int64_t N = h->n_dofs;
  const int g = vgrid(N);
  double *r = h->w[0], *z = h->w[1], *p = h->w[2], *Ap = h->w[3];
  k_amr_zero<<<g, 256>>>(N, x);
  k_amr_axpby<<<g, 256>>>(N, 1.0, b, 0.0, r);
  k_amr_mul<<<g, 256>>>(N, inv, r, z);
  k_amr_axpby<<<g, 256>>>(N, 1.0, z, 0.0, p);
  double rr = 0.0, rz = 0.0;
  TRY_AMR(dot(h, r, r, &rr));
  TRY_AMR(dot(h, r, z, &rz));
  const double tol = std::max(abs_tol, rel_tol * std::sqrt(rr));
  *iterations = 0;
  if (std::sqrt(rr) <= tol) return MPDG_OK;
  // T_lin is fixed during the solve: its values and gradients at the q-points once
  const double *tf = nullptr;
  if (T_lin && h->mat.law == MPDG_LAW_LINEAR_K && h->mat.k1 != 0.0) {
    TRY_AMR(tfields_impl(h, T_lin));
    tf = h->tf;
  }
  for (int it = 1; it <= max_it; ++it) {
    TRY_AMR(vmult_impl(h, Ap, p, T_lin, tf));
    double pap = 0.0;
    TRY_AMR(dot(h, p, Ap, &pap));
    if (!(pap > 0.0)) return fail(MPDG_ERR_BREAKDOWN, "CG breakdown: p.Ap <= 0");
    const double alpha = rz / pap;
    k_amr_axpby<<<g, 256>>>(N, alpha, p, 1.0, x);
    k_amr_axpby<<<g, 256>>>(N, -alpha, Ap, 1.0, r);
    TRY_AMR(dot(h, r, r, &rr));
    if (!std::isfinite(rr)) return fail(MPDG_ERR_NAN, "CG residual is not finite");
    *iterations = it;
    if (std::sqrt(rr) <= tol) return MPDG_OK;
    k_amr_mul<<<g, 256>>>(N, inv, r, z);
    double rz_new = 0.0;
    TRY_AMR(dot(h, r, z, &rz_new));
    k_amr_axpby<<<g, 256>>>(N, 1.0, z, rz_new / rz, p);
    rz = rz_new;
  }
  return fail(MPDG_ERR_NOT_CONVERGED, "CG on the hanging-node mesh did not converge");
}

}  // namespace

extern "C" int mpdg_amr_vmult(mpdg_amr *h, double *dst, const double *src, const double *T_lin)
{
  if (!h || !dst || !src) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  TRY_AMR(ready(h));
  const bool tangent = h->mat.law == MPDG_LAW_LINEAR_K && h->mat.k1 != 0.0;
  if (tangent && !T_lin)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "LINEAR_K needs the linearisation point");
  TRY_AMR(check_device_vectors({dst, src, T_lin}));
  TRY_AMR(vmult_impl(h, dst, src, T_lin));
  return sync_status();
}

extern "C" int mpdg_amr_inverse_diagonal(mpdg_amr *h, double *inv_diag, const double *T_lin)
{
  if (!h || !inv_diag) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  TRY_AMR(ready(h));
  const bool tangent = h->mat.law == MPDG_LAW_LINEAR_K && h->mat.k1 != 0.0;
  if (tangent && !T_lin)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "LINEAR_K needs the linearisation point");
  TRY_AMR(check_device_vectors({inv_diag, T_lin}));
  TRY_AMR(diag_impl(h, inv_diag, T_lin));
  return sync_status();
}

extern "C" int mpdg_amr_create_rhs(mpdg_amr *h, double *dst, const double *T, const double *T_old,
                                   const double *heat_source)
{
  if (!h || !dst || !T || !T_old) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  TRY_AMR(ready(h));
  TRY_AMR(check_device_vectors({dst, T, T_old, heat_source}));
  TRY_AMR(rhs_impl(h, dst, T, T_old, heat_source));
  return sync_status();
}

extern "C" int mpdg_amr_linear_solve(mpdg_amr *h, double *x, const double *b, const double *T_lin,
                                     double rel_tolerance, double abs_tolerance,
                                     int max_iterations, int *iterations)
{
  if (!h || !x || !b) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  TRY_AMR(ready(h));
  const bool tangent = h->mat.law == MPDG_LAW_LINEAR_K && h->mat.k1 != 0.0;
  if (tangent && !T_lin)
    return fail(MPDG_ERR_INVALID_ARGUMENT, "LINEAR_K needs the linearisation point");
  TRY_AMR(check_device_vectors({x, b, T_lin}));
  TRY_AMR(ensure_workspace(h));
  int its = 0;
  double *inv = h->w[4];
  TRY_AMR(diag_impl(h, inv, T_lin));
  const int rc = cg_impl(h, x, b, inv, T_lin, rel_tolerance, abs_tolerance, max_iterations, &its);
  if (iterations) *iterations = its;
  if (rc != MPDG_OK) return rc;
  return sync_status();
}

extern "C" int mpdg_amr_time_step(mpdg_amr *h, double dt, double dt_old, double *T_cur,
                                  double *T_old, const double *heat_source,
                                  const mpdg_step_params *prm, mpdg_step_stats *stats)
{
  if (!h || !T_cur || !T_old || !prm) return fail(MPDG_ERR_INVALID_ARGUMENT, "null argument");
  TRY_AMR(ready(h));
  if (dt == 0.0) return fail(MPDG_ERR_ZERO_TIME_INCREMENT, "time increment is zero");
  TRY_AMR(check_device_vectors({T_cur, T_old, heat_source}));
  TRY_AMR(ensure_workspace(h));
  h->dt = dt;
  const int64_t N = h->n_dofs;
  const int g = vgrid(N);
  mpdg_step_stats s;
  std::memset(&s, 0, sizeof(s));
  // init_time_advance: linear predictor (predictor_linear.cpp:74-96) or a copy, history commit,
  // Dirichlet values (zero on these meshes); Jacobi at the predicted state
  const double r = (prm->predictor == MPDG_PREDICTOR_LINEAR && std::fabs(dt_old) >= 1e-12)
                     ? dt / dt_old : 0.0;
  k_amr_predict<<<g, 256>>>(N, r, T_cur, T_old, h->d_mask);
  const bool tangent = h->mat.law == MPDG_LAW_LINEAR_K && h->mat.k1 != 0.0;
  double *rhs = h->w[5], *delta = h->w[6], *inv = h->w[4];
  TRY_AMR(diag_impl(h, inv, tangent ? T_cur : nullptr));
  // Newton-Raphson (newton_raphson_solver.cpp:22-68): rhs = -R(T); J delta = rhs; converged
  // when |rhs| < tol_res and |delta| < tol_corr (the converged update is not applied)
  for (int it = 0; it < prm->newton_max_iterations; ++it) {
    k_amr_zero<<<g, 256>>>(N, rhs);
    TRY_AMR(rhs_impl(h, rhs, T_cur, T_old, heat_source));
    int its = 0;
    TRY_AMR(cg_impl(h, delta, rhs, inv, tangent ? T_cur : nullptr, prm->linear.rel_tolerance,
                    prm->linear.abs_tolerance, prm->linear.max_iterations, &its));
    s.linear_iterations += its;
    double rr = 0.0, dd = 0.0;
    TRY_AMR(dot(h, rhs, rhs, &rr));
    TRY_AMR(dot(h, delta, delta, &dd));
    if (std::sqrt(rr) < prm->newton_residual_tolerance &&
        std::sqrt(dd) < prm->newton_correction_tolerance) {
      s.converged = 1;
      s.newton_iterations = it + 1;
      break;
    }
    k_amr_axpby<<<g, 256>>>(N, 1.0, delta, 1.0, T_cur);
    s.newton_iterations = it + 1;
  }
  if (stats) *stats = s;
  TRY_AMR(sync_status());
  if (!s.converged) return fail(MPDG_ERR_NEWTON_NOT_CONVERGED, "Newton-Raphson did not converge");
  return MPDG_OK;
}
