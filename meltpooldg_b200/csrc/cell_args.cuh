// Argument structs shared by the cell kernels and the handle code.
#pragma once

#include <stdint.h>

#include "fe_tables.hpp"

namespace mpdg {

// ---------------------------------------------------------------------------
// argument structs
// ---------------------------------------------------------------------------
struct MeshDims {
  int m[3];   // cells per direction
  int nd[3];  // DoFs per direction
  int p;      // degree
  int dmask;  // Dirichlet faces (bit f: 0 x-,1 x+,2 y-,3 y+,4 z-,5 z+)
};

template <typename T>
struct MatParams {
  T rho_l, cp_l, k_l, rho_s, cp_s, k_s, rho_g, cp_g, k_g;
  T T_liq, T_sol, inv_mushy, k1;
  T idt;
  int sharp, vs, need_told;
  T latent;  // latent heat of fusion (> 0: apparent capacity of profile acap in the mushy zone)
  int acap;
};

template <typename T>
struct GeoParams {
  T detJ;                   // uniform box: det(J)
  T Gd[3];                  // uniform box: det(J) / h_d^2
  const T *__restrict__ q;  // deformed: [cell][7][n^3] = JxW, Gxx Gxy Gxz Gyy Gyz Gzz
};

// Scalars of a device-resident Krylov iteration (read by kernels, finalised
// by the last CTA of a reduction, polled by the host).
struct SolverState {
  double rz, rz_old, alpha, beta, pAp, rr, res, res0, tol, zAp;
  int it, max_it, done, status;  // done: 0 running, 1 converged, 2 stopped
  int first;                     // preconditioned CG: first direction (beta = 0)
  int record;                    // record alpha/beta history (Lanczos)
  double hist_alpha[64], hist_beta[64];
};

// ---------------------------------------------------------------------------
// the support points of the DoFs and a volumetric laser source evaluated there
// ---------------------------------------------------------------------------
struct Q1D {
  double xg[kMaxN], wg[kMaxN], xl[kMaxN];
};

struct PosArgs {
  MeshDims d;
  int geo;
  double lo[3], hc[3];
  Q1D q1;
  const double *vert;
};

struct LaserArgs {
  int profile, planar;  // planar: the y coordinate is ignored (2D profile in the x-z plane)
  double power, c[3], dir[3], radius, peak;
  double rho, beta, L, lambda, a, D;  // Gusarov
};

// a residual kernel's nodal heat source evaluated in place: the laser intensity at the
// support points (on = 1) instead of a nodal source vector
struct SourceEval {
  int on;
  LaserArgs laser;
  PosArgs pos;
};

enum FinMode { FIN_NONE = 0, FIN_STORE = 1, FIN_CG_ALPHA = 2 };

template <typename T>
struct CellArgs {
  int64_t n_cells;
  MeshDims d;
  GeoParams<T> g;
  MatParams<T> m;
  const T *__restrict__ src;
  T *dst;
  const T *__restrict__ Tl;
  const T *__restrict__ To;
  const T *__restrict__ qs;
  const float *__restrict__ kq;  // per-q conductivity [cell][n^3] (coefficient-field operator)
  // per-q coefficient fields, [cell][5][n^3]. LAW 4 (temperature-independent laws):
  // rho_cp JxW, k, JxW rho_cp J^-1 v (three components); LAW 5 (temperature-dependent
  // laws with a heaviside and/or a velocity): gas-liquid weight w, 0, JxW J^-1 v
  const T *__restrict__ cf;
  double *partials;    // per-CTA partial sums
  unsigned *counter;   // last-CTA election counter (reset by the last CTA)
  SolverState *st;     // early exit when st->done; alpha finalisation
  double *out;         // FIN_STORE destination
  const double *extra_dot;  // boundary-face part of src.dst, added at finalisation (nullable)
  int fin;
  SourceEval source;  // create_rhs: the laser source at the support points (source.on)
};

// ---------------------------------------------------------------------------
// launch shapes
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int cells_per_block(int n)
{
  return n == 2 ? 32 : n == 3 ? 14 : n == 4 ? 8 : n == 5 ? 5 : n == 6 ? 4 : 2;
}
__host__ __device__ constexpr int block_threads(int n) { return cells_per_block(n) * n * n; }

// Dirichlet-constrained DoF (I, J, K) of the lexicographic nodal grid
__device__ __forceinline__ bool constrained(const MeshDims &d, int I, int J, int K)
{
  return ((d.dmask & 1) && I == 0) || ((d.dmask & 2) && I == d.nd[0] - 1) ||
         ((d.dmask & 4) && J == 0) || ((d.dmask & 8) && J == d.nd[1] - 1) ||
         ((d.dmask & 16) && K == 0) || ((d.dmask & 32) && K == d.nd[2] - 1);
}

}  // namespace mpdg
