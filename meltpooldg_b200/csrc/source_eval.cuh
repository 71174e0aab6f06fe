// Positions of the DoF support points and the volumetric laser intensity, shared by the
// handle's source kernels and the residual kernels that evaluate the source in place.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/mpdg_heat.h"
#include "cell_args.cuh"
#include "fe_tables.hpp"

namespace mpdg {

__host__ __device__ __forceinline__ void trilinear(const double *__restrict__ vert, const MeshDims &d, int cx,
                                          int cy, int cz, const double xi[3], double x[3],
                                          double J[3][3])
{
  for (int a = 0; a < 3; ++a) {
    x[a] = 0.0;
    for (int b = 0; b < 3; ++b) J[a][b] = 0.0;
  }
  for (int v = 0; v < 8; ++v) {
    const int a = v & 1, b = (v >> 1) & 1, c = (v >> 2) & 1;
    const int64_t vid =
      (int64_t)(cx + a) + (int64_t)(d.m[0] + 1) * ((cy + b) + (int64_t)(d.m[1] + 1) * (cz + c));
    const double *X = vert + 3 * vid;
    const double na = a ? xi[0] : 1.0 - xi[0], da = a ? 1.0 : -1.0;
    const double nb = b ? xi[1] : 1.0 - xi[1], db = b ? 1.0 : -1.0;
    const double nc = c ? xi[2] : 1.0 - xi[2], dc = c ? 1.0 : -1.0;
    const double N = na * nb * nc;
    const double dN[3] = {da * nb * nc, na * db * nc, na * nb * dc};
    for (int e = 0; e < 3; ++e) {
      x[e] += X[e] * N;
      for (int f = 0; f < 3; ++f) J[e][f] += X[e] * dN[f];
    }
  }
}

__host__ __device__ __forceinline__ void dof_position(const PosArgs &a, int64_t idx, double x[3])
{
  const int64_t I = idx % a.d.nd[0];
  const int64_t J = (idx / a.d.nd[0]) % a.d.nd[1];
  const int64_t K = idx / ((int64_t)a.d.nd[0] * a.d.nd[1]);
  const int64_t pos[3] = {I, J, K};
  int cc[3];
  double xi[3];
  for (int e = 0; e < 3; ++e) {
    cc[e] = (int)(pos[e] / a.d.p);
    if (cc[e] >= a.d.m[e]) cc[e] = a.d.m[e] - 1;
    xi[e] = a.q1.xl[pos[e] - (int64_t)cc[e] * a.d.p];
  }
  if (a.geo == 0) {
    for (int e = 0; e < 3; ++e) x[e] = a.lo[e] + a.hc[e] * (cc[e] + xi[e]);
  } else {
    double J3[3][3];
    trilinear(a.vert, a.d, cc[0], cc[1], cc[2], xi, x, J3);
  }
}

// volumetric laser intensity at x (laser_intensity_profiles.hpp), parameters precomputed
// on the host (LaserArgs)
__device__ __forceinline__ double gusarov_dq_dxi(const LaserArgs &g, double xi)
{
  const double rho = g.rho, a = g.a, lambda = g.lambda;
  if (!(xi < lambda)) return 0.0;
  return (3 - 3 * rho) * (exp(-xi) + rho * exp(xi - 2 * lambda)) / (4 * rho - 3) +
         2 * a * a * rho / (g.D * (4 * rho - 3)) *
           (exp(-lambda) * (1 - rho * rho) * (exp(-2 * a * xi) * (a - 1) + exp(2 * a * xi) * (a + 1)) -
            (rho * exp(-2 * lambda) + 3) * (exp(2 * a * (xi - lambda)) * (1 - a - rho * (a + 1)) -
                                            exp(2 * a * (lambda - xi)) * (a + rho * (a - 1) + 1)));
}
__device__ __forceinline__ double laser_intensity(const LaserArgs &g, const double x[3])
{
  const double v0 = x[0] - g.c[0], v1 = g.planar ? 0.0 : x[1] - g.c[1], v2 = x[2] - g.c[2];
  if (g.profile == MPDG_LASER_UNIFORM) return g.power;
  if (g.profile == MPDG_LASER_GAUSS_VOLUMETRIC) {
    const double s2 = (v0 * v0 + v1 * v1 + v2 * v2) / (g.radius * g.radius);
    return g.peak * exp(-2.0 * s2);
  }
  if (g.profile == MPDG_LASER_GAUSS_PROJECTION) {
    const double w0 = v1 * g.dir[2] - v2 * g.dir[1], w1 = v2 * g.dir[0] - v0 * g.dir[2],
                 w2 = v0 * g.dir[1] - v1 * g.dir[0];
    const double s2 = (w0 * w0 + w1 * w1 + w2 * w2) / (g.radius * g.radius);
    return g.peak * exp(-2.0 * s2);
  }
  // Gusarov: z measured downwards from the beam centre; zero outside the layer
  const double dist = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
  const double z = -(x[2] - g.c[2]);
  if (z >= g.L || z < g.c[2]) return 0.0;
  double pd = 0.0;
  if (dist <= g.radius) {
    const double m = 1.0 - dist / g.radius, p = 1.0 + dist / g.radius;
    pd = 3.0 * g.power / (M_PI * g.radius * g.radius) * (m * m) * (p * p);
  }
  return -g.beta * pd * gusarov_dq_dxi(g, z * g.beta);
}
// the nodal heat source of DoF idx evaluated in place (SourceEval.on): the laser intensity at
// the DoF's support point, the value mpdg_heat_laser_source stores there
__device__ __forceinline__ double source_at(const SourceEval &s, int64_t idx)
{
  double x[3];
  dof_position(s.pos, idx, x);
  return laser_intensity(s.laser, x);
}

}  // namespace mpdg
