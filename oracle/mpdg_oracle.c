/*
 * CPU oracle for the matrix-free heat path (TEST INFRASTRUCTURE ONLY).
 * See mpdg_oracle.h for the reference files restated here. Never linked
 * into the product library.
 *
 * Two independent evaluation forms of every cell integral:
 *   form 0  sum factorisation: values at QGauss(n) by three 1D sweeps of the
 *           GLL->Gauss interpolation matrix, gradients by collocation
 *           derivatives at the Gauss points, even-odd 1D kernels, SIMD over a
 *           batch of ORC_VEC cells, OpenMP over batches of one colour
 *           (the deal.II FEEvaluation scheme, restated);
 *   form 1  direct quadrature with the full 3D basis tables (no sum
 *           factorisation, no collocation), one cell at a time.
 * Cells are coloured by the parity of their (i,j,k) index: cells of one
 * colour share no DoF, so scatter-adds within a colour never collide.
 */
#include "mpdg_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#define ORC_VEC 8
#define NMAX 7
#define NPT_MAX (NMAX * NMAX * NMAX)

/* ------------------------------------------------------------------ */
/* 1D polynomial tables                                                */
/* ------------------------------------------------------------------ */

/* Gauss-Legendre points/weights on [0,1] by Newton iteration on P_n. */
static void gauss_legendre(int n, double *x, double *w)
{
  for (int i = 0; i < n; ++i) {
    double t = cos(M_PI * (i + 0.75) / (n + 0.5));
    double dp = 0.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = t;
      for (int k = 2; k <= n; ++k) {
        double pk = ((2.0 * k - 1.0) * t * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = pk;
      }
      if (n == 1) { p1 = t; p0 = 1.0; }
      dp = n * (t * p1 - p0) / (t * t - 1.0);
      double dt = p1 / dp;
      t -= dt;
      if (fabs(dt) < 1e-16) break;
    }
    {
      double p0 = 1.0, p1 = t;
      for (int k = 2; k <= n; ++k) {
        double pk = ((2.0 * k - 1.0) * t * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = pk;
      }
      if (n == 1) { p1 = t; p0 = 1.0; }
      dp = n * (t * p1 - p0) / (t * t - 1.0);
    }
    /* ascending order on [0,1] */
    x[n - 1 - i] = 0.5 * (1.0 + t);
    w[n - 1 - i] = 1.0 / ((1.0 - t * t) * dp * dp);
  }
}

/* Gauss-Lobatto points on [0,1] (n >= 2): endpoints plus roots of P'_{n-1}. */
static void gauss_lobatto(int n, double *x)
{
  const int N = n - 1;
  double t[NMAX + 1], told[NMAX + 1];
  for (int i = 0; i <= N; ++i) t[i] = cos(M_PI * i / N);
  for (int it = 0; it < 200; ++it) {
    double maxd = 0.0;
    for (int i = 0; i <= N; ++i) {
      told[i] = t[i];
      double p0 = 1.0, p1 = t[i];
      for (int k = 2; k <= N; ++k) {
        double pk = ((2.0 * k - 1.0) * t[i] * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = pk;
      }
      if (N == 1) { p0 = 1.0; p1 = t[i]; }
      t[i] = told[i] - (t[i] * p1 - p0) / ((N + 1) * p1);
      double d = fabs(t[i] - told[i]);
      if (d > maxd) maxd = d;
    }
    if (maxd < 1e-16) break;
  }
  for (int i = 0; i <= N; ++i) x[N - i] = 0.5 * (1.0 + t[i]);
  x[0] = 0.0;
  x[N] = 1.0;
}

static double lagrange_value(const double *z, int n, int i, double x)
{
  double v = 1.0;
  for (int j = 0; j < n; ++j)
    if (j != i) v *= (x - z[j]) / (z[i] - z[j]);
  return v;
}

static double lagrange_deriv(const double *z, int n, int i, double x)
{
  double s = 0.0;
  for (int m = 0; m < n; ++m) {
    if (m == i) continue;
    double v = 1.0 / (z[i] - z[m]);
    for (int j = 0; j < n; ++j)
      if (j != i && j != m) v *= (x - z[j]) / (z[i] - z[j]);
    s += v;
  }
  return s;
}

/* 1D matrix with its even-odd split; rows = outputs, cols = inputs. */
typedef struct {
  double a[NMAX][NMAX];
  double ae[NMAX][NMAX], ao[NMAX][NMAX];
  int    sym; /* a[n-1-o][n-1-l] = sym * a[o][l] */
} mat1d;

static void mat_init(mat1d *m, int n, int sym)
{
  m->sym = sym;
  const int h = n / 2;
  for (int o = 0; o < n; ++o)
    for (int l = 0; l < h; ++l) {
      m->ae[o][l] = 0.5 * (m->a[o][l] + m->a[o][n - 1 - l]);
      m->ao[o][l] = 0.5 * (m->a[o][l] - m->a[o][n - 1 - l]);
    }
}

/* ------------------------------------------------------------------ */
/* handle                                                              */
/* ------------------------------------------------------------------ */

struct orc_heat {
  int      p, n, npt;
  int      m[3];
  int      nd[3];
  int64_t  n_dofs, n_cells;
  double   lo[3], hi[3];
  int      affine;
  double  *vert;  /* (m0+1)(m1+1)(m2+1) x 3 */
  double  *geo;   /* affine: n_cells x 7 ; else n_cells x npt x 7 */
  uint8_t *mask;  /* constrained DoFs */
  double  *dvalue; /* Dirichlet value per DoF (valid where mask) */
  int      dirichlet_mask;
  /* 1D data */
  double xg[NMAX], wg[NMAX], xl[NMAX];
  double S[NMAX][NMAX], Sd[NMAX][NMAX], D[NMAX][NMAX];
  mat1d  mS, mST, mD, mDT, mPT, mQT, mRT;
  double wq[NPT_MAX];
  /* colouring */
  int64_t *color_cells[8];
  int64_t  color_n[8];
  /* coefficients */
  orc_material mat;
  double       dt;
  int          tdep;      /* temperature-dependent law: tangent terms + T_lin */
  int          need_told; /* d(rho cp)/dT may be non-zero */
  const double *Hf, *vel; /* nodal heaviside and velocity ([3][n_dofs]) fields, or NULL */
  int          fields;    /* coefficients from the fields: gas-liquid law and/or convection */
  /* direct-form tables */
  double *phi, *dphi;
  /* boundary terms per face */
  int    btype[6];
  double bh[6], bTc[6], beps[6], bTr[6], bqn[6];
};

static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }
static int nthreads(void) { return g_threads > 0 ? g_threads : omp_get_max_threads(); }

static uint64_t splitmix64(uint64_t x)
{
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

/* uniform in [-1,1) from (seed, index): the mesh-perturbation convention */
static double hash_sym(uint64_t seed, uint64_t idx)
{
  uint64_t r = splitmix64(seed * 0xD1B54A32D192ED03ULL + idx);
  return 2.0 * ((double)(r >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
}

static inline int64_t vid(const orc_heat *h, int a, int b, int c)
{
  return (int64_t)a + (int64_t)(h->m[0] + 1) * ((int64_t)b + (int64_t)(h->m[1] + 1) * c);
}

static void cell_coords(const orc_heat *h, int64_t c, int *cx, int *cy, int *cz)
{
  *cx = (int)(c % h->m[0]);
  int64_t r = c / h->m[0];
  *cy = (int)(r % h->m[1]);
  *cz = (int)(r / h->m[1]);
}

/* trilinear map Jacobian and position at reference point xi of cell c */
static void cell_map(const orc_heat *h, int64_t c, const double xi[3], double x[3],
                     double J[3][3])
{
  int cx, cy, cz;
  cell_coords(h, c, &cx, &cy, &cz);
  for (int d = 0; d < 3; ++d) {
    x[d] = 0.0;
    for (int e = 0; e < 3; ++e) J[d][e] = 0.0;
  }
  for (int v = 0; v < 8; ++v) {
    const int a = v & 1, b = (v >> 1) & 1, cc = (v >> 2) & 1;
    const double *X = h->vert + 3 * vid(h, cx + a, cy + b, cz + cc);
    const double na = a ? xi[0] : 1.0 - xi[0], da = a ? 1.0 : -1.0;
    const double nb = b ? xi[1] : 1.0 - xi[1], db = b ? 1.0 : -1.0;
    const double nc = cc ? xi[2] : 1.0 - xi[2], dc = cc ? 1.0 : -1.0;
    const double N = na * nb * nc;
    const double dN[3] = {da * nb * nc, na * db * nc, na * nb * dc};
    for (int d = 0; d < 3; ++d) {
      x[d] += X[d] * N;
      for (int e = 0; e < 3; ++e) J[d][e] += X[d] * dN[e];
    }
  }
}

/* det(J) and G = det(J) J^-1 J^-T (6 comps: xx xy xz yy yz zz) */
static double geo_factors(const double J[3][3], double G[6])
{
  const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                     J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  double inv[3][3];
  inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
  inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
  inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
  inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
  inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
  inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
  inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
  inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
  inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
  /* (J^-1 J^-T)_{ab} = sum_d inv[a][d] inv[b][d] */
  const int ia[6] = {0, 0, 0, 1, 1, 2}, ib[6] = {0, 1, 2, 1, 2, 2};
  for (int k = 0; k < 6; ++k) {
    double s = 0.0;
    for (int d = 0; d < 3; ++d) s += inv[ia[k]][d] * inv[ib[k]][d];
    G[k] = det * s;
  }
  return det;
}

orc_heat *orc_create(const orc_mesh_desc *desc)
{
  if (desc->degree < 1 || desc->degree > 6) return NULL;
  orc_heat *h = (orc_heat *)calloc(1, sizeof(orc_heat));
  h->p = desc->degree;
  h->n = h->p + 1;
  h->npt = h->n * h->n * h->n;
  const int n = h->n;
  for (int d = 0; d < 3; ++d) {
    h->m[d] = desc->cells[d];
    h->nd[d] = h->p * h->m[d] + 1;
    h->lo[d] = desc->lo[d];
    h->hi[d] = desc->hi[d];
  }
  h->n_dofs = (int64_t)h->nd[0] * h->nd[1] * h->nd[2];
  h->n_cells = (int64_t)h->m[0] * h->m[1] * h->m[2];
  h->affine = desc->perturb == 0.0;

  /* 1D tables */
  gauss_legendre(n, h->xg, h->wg);
  gauss_lobatto(n, h->xl);
  for (int q = 0; q < n; ++q)
    for (int i = 0; i < n; ++i) {
      h->S[q][i] = lagrange_value(h->xl, n, i, h->xg[q]);
      h->D[q][i] = lagrange_deriv(h->xg, n, i, h->xg[q]);
    }
  /* Sd = D * S: gradient of the GLL basis at the Gauss points, computed the
   * way the collocation path computes it */
  for (int q = 0; q < n; ++q)
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int m = 0; m < n; ++m) s += h->D[q][m] * h->S[m][i];
      h->Sd[q][i] = s;
    }
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) {
      h->mS.a[a][b] = h->S[a][b];
      h->mST.a[a][b] = h->S[b][a];
      h->mD.a[a][b] = h->D[a][b];
      h->mDT.a[a][b] = h->D[b][a];
      h->mPT.a[a][b] = h->S[b][a] * h->S[b][a];
      h->mQT.a[a][b] = h->Sd[b][a] * h->Sd[b][a];
      h->mRT.a[a][b] = h->S[b][a] * h->Sd[b][a];
    }
  mat_init(&h->mS, n, 1);
  mat_init(&h->mST, n, 1);
  mat_init(&h->mD, n, -1);
  mat_init(&h->mDT, n, -1);
  mat_init(&h->mPT, n, 1);
  mat_init(&h->mQT, n, 1);
  mat_init(&h->mRT, n, -1);
  for (int k = 0; k < n; ++k)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) h->wq[i + n * (j + n * k)] = h->wg[i] * h->wg[j] * h->wg[k];

  /* vertices */
  const int64_t nv = (int64_t)(h->m[0] + 1) * (h->m[1] + 1) * (h->m[2] + 1);
  h->vert = (double *)malloc(sizeof(double) * 3 * nv);
  for (int c = 0; c <= h->m[2]; ++c)
    for (int b = 0; b <= h->m[1]; ++b)
      for (int a = 0; a <= h->m[0]; ++a) {
        const int idx[3] = {a, b, c};
        const int64_t v = vid(h, a, b, c);
        int interior = 1;
        for (int d = 0; d < 3; ++d)
          if (idx[d] == 0 || idx[d] == h->m[d]) interior = 0;
        for (int d = 0; d < 3; ++d) {
          const double hd = (h->hi[d] - h->lo[d]) / h->m[d];
          double x = h->lo[d] + hd * idx[d];
          if (interior && desc->perturb != 0.0)
            x += desc->perturb * hd * hash_sym(desc->seed, (uint64_t)(3 * v + d));
          h->vert[3 * v + d] = x;
        }
      }

  /* geometry */
  const int npt = h->npt;
  if (h->affine) {
    h->geo = (double *)malloc(sizeof(double) * 7 * h->n_cells);
#pragma omp parallel for num_threads(nthreads())
    for (int64_t c = 0; c < h->n_cells; ++c) {
      const double xi[3] = {0.5, 0.5, 0.5};
      double x[3], J[3][3], G[6];
      cell_map(h, c, xi, x, J);
      double det = geo_factors(J, G);
      h->geo[7 * c] = det;
      for (int k = 0; k < 6; ++k) h->geo[7 * c + 1 + k] = G[k];
    }
  } else {
    h->geo = (double *)malloc(sizeof(double) * 7 * h->n_cells * npt);
#pragma omp parallel for num_threads(nthreads())
    for (int64_t c = 0; c < h->n_cells; ++c)
      for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
          for (int i = 0; i < n; ++i) {
            const int q = i + n * (j + n * k);
            const double xi[3] = {h->xg[i], h->xg[j], h->xg[k]};
            double x[3], J[3][3], G[6];
            cell_map(h, c, xi, x, J);
            double det = geo_factors(J, G);
            double *g = h->geo + 7 * (c * npt + q);
            g[0] = det * h->wq[q];
            for (int t = 0; t < 6; ++t) g[1 + t] = G[t] * h->wq[q];
          }
  }

  /* constraints */
  h->mask = (uint8_t *)calloc((size_t)h->n_dofs, 1);
  h->dvalue = (double *)calloc((size_t)h->n_dofs, sizeof(double));
  h->dirichlet_mask = desc->dirichlet_mask;
  orc_set_dirichlet_values(h, desc->dirichlet_value);

  /* colouring */
  for (int col = 0; col < 8; ++col) h->color_n[col] = 0;
  for (int64_t c = 0; c < h->n_cells; ++c) {
    int cx, cy, cz;
    cell_coords(h, c, &cx, &cy, &cz);
    h->color_n[(cx & 1) | ((cy & 1) << 1) | ((cz & 1) << 2)]++;
  }
  for (int col = 0; col < 8; ++col) {
    h->color_cells[col] = (int64_t *)malloc(sizeof(int64_t) * (h->color_n[col] + 1));
    h->color_n[col] = 0;
  }
  for (int64_t c = 0; c < h->n_cells; ++c) {
    int cx, cy, cz;
    cell_coords(h, c, &cx, &cy, &cz);
    const int col = (cx & 1) | ((cy & 1) << 1) | ((cz & 1) << 2);
    h->color_cells[col][h->color_n[col]++] = c;
  }

  /* direct-form tables */
  h->phi = (double *)malloc(sizeof(double) * npt * npt);
  h->dphi = (double *)malloc(sizeof(double) * 3 * npt * npt);
  for (int q = 0; q < npt; ++q) {
    const int qx = q % n, qy = (q / n) % n, qz = q / (n * n);
    for (int i = 0; i < npt; ++i) {
      const int ix = i % n, iy = (i / n) % n, iz = i / (n * n);
      h->phi[q * npt + i] = h->S[qx][ix] * h->S[qy][iy] * h->S[qz][iz];
      h->dphi[(q * npt + i) * 3 + 0] = h->Sd[qx][ix] * h->S[qy][iy] * h->S[qz][iz];
      h->dphi[(q * npt + i) * 3 + 1] = h->S[qx][ix] * h->Sd[qy][iy] * h->S[qz][iz];
      h->dphi[(q * npt + i) * 3 + 2] = h->S[qx][ix] * h->S[qy][iy] * h->Sd[qz][iz];
    }
  }

  orc_material m0;
  memset(&m0, 0, sizeof(m0));
  m0.law = ORC_LAW_CONSTANT;
  m0.rho_l = m0.cp_l = m0.k_l = 1.0;
  orc_set_material(h, &m0, 1.0);
  return h;
}

void orc_destroy(orc_heat *h)
{
  if (!h) return;
  free(h->vert);
  free(h->geo);
  free(h->mask);
  free(h->dvalue);
  for (int c = 0; c < 8; ++c) free(h->color_cells[c]);
  free(h->phi);
  free(h->dphi);
  free(h);
}

int64_t orc_n_dofs(const orc_heat *h) { return h->n_dofs; }
int64_t orc_n_cells(const orc_heat *h) { return h->n_cells; }
void orc_dof_dims(const orc_heat *h, int dims[3])
{
  for (int d = 0; d < 3; ++d) dims[d] = h->nd[d];
}
void orc_constraint_mask(const orc_heat *h, uint8_t *mask)
{
  memcpy(mask, h->mask, (size_t)h->n_dofs);
}

void orc_support_points(const orc_heat *h, double *xyz)
{
#pragma omp parallel for num_threads(nthreads())
  for (int64_t K = 0; K < h->nd[2]; ++K)
    for (int64_t J = 0; J < h->nd[1]; ++J)
      for (int64_t I = 0; I < h->nd[0]; ++I) {
        const int64_t pos[3] = {I, J, K};
        int cc[3];
        double xi[3];
        for (int d = 0; d < 3; ++d) {
          cc[d] = (int)(pos[d] / h->p);
          if (cc[d] >= h->m[d]) cc[d] = h->m[d] - 1;
          xi[d] = h->xl[pos[d] - (int64_t)cc[d] * h->p];
        }
        const int64_t c = cc[0] + (int64_t)h->m[0] * (cc[1] + (int64_t)h->m[1] * cc[2]);
        double x[3], Jm[3][3];
        cell_map(h, c, xi, x, Jm);
        const int64_t idx = I + h->nd[0] * (J + (int64_t)h->nd[1] * K);
        for (int d = 0; d < 3; ++d) xyz[3 * idx + d] = x[d];
      }
}

/* Dirichlet values per face (the first flagged face in the order x-, x+, y-, y+, z-, z+ owns
 * an edge or corner DoF); called again for boundary data that change in time
 * (HeatData::enable_time_dependent_bc: init_time_advance rebuilds the constraints every step,
 * heat_diffuse_operation.cpp:219-226) */
void orc_set_dirichlet_values(orc_heat *h, const double values[6])
{
  for (int64_t K = 0; K < h->nd[2]; ++K)
    for (int64_t J = 0; J < h->nd[1]; ++J)
      for (int64_t I = 0; I < h->nd[0]; ++I) {
        const int64_t idx = I + h->nd[0] * (J + (int64_t)h->nd[1] * K);
        const int64_t pos[3] = {I, J, K};
        int owned = 0;
        for (int f = 0; f < 6; ++f) {
          if (!(h->dirichlet_mask & (1 << f))) continue;
          const int d = f / 2;
          const int64_t at = (f & 1) ? h->nd[d] - 1 : 0;
          if (pos[d] == at) {
            if (!owned) h->dvalue[idx] = values[f];
            owned = 1;
            h->mask[idx] = 1;
          }
        }
      }
}

void orc_distribute(const orc_heat *h, double *u)
{
#pragma omp parallel for num_threads(nthreads())
  for (int64_t i = 0; i < h->n_dofs; ++i)
    if (h->mask[i]) u[i] = h->dvalue[i];
}

int orc_set_material(orc_heat *h, const orc_material *m, double dt)
{
  if (h->vel && m->law == ORC_LAW_LINEAR_K) return -1;
  /* the reference throws for an apparent capacity with volume-specific rho*cp
   * (material.templates.hpp:321-328) */
  if (m->latent_heat > 0.0 && m->volume_specific) return -2;
  h->mat = *m;
  h->dt = dt;
  h->tdep = m->law == ORC_LAW_LINEAR_K || m->law == ORC_LAW_LIQUID_SOLID ||
            m->law == ORC_LAW_GAS_LIQUID_SOLID;
  h->fields = m->law == ORC_LAW_GAS_LIQUID || m->law == ORC_LAW_GAS_LIQUID_SOLID || h->vel != NULL;
  h->need_told = 0;
  if (m->law == ORC_LAW_LIQUID_SOLID || m->law == ORC_LAW_GAS_LIQUID_SOLID) {
    if (m->volume_specific)
      h->need_told = (m->rho_l * m->cp_l != m->rho_s * m->cp_s);
    else
      h->need_told = (m->rho_l != m->rho_s) || (m->cp_l != m->cp_s) || m->latent_heat > 0.0;
  }
  return 0;
}

int orc_set_fields(orc_heat *h, const double *heaviside, const double *velocity)
{
  if (velocity && h->mat.law == ORC_LAW_LINEAR_K) return -1;
  h->Hf = heaviside;
  h->vel = velocity;
  h->fields = h->mat.law == ORC_LAW_GAS_LIQUID || h->mat.law == ORC_LAW_GAS_LIQUID_SOLID ||
              velocity != NULL;
  return 0;
}

/* ------------------------------------------------------------------ */
/* material law (Material::compute_parameters, liquid_solid / gas,     */
/* plus the linear conductivity law k = k_l + k1 T)                    */
/* ------------------------------------------------------------------ */

/* J^-1 v at quadrature point q of cell c (reference-space transport direction: the
 * physical v.grad(u) equals (J^-1 v).grad_ref(u)) */
static void ref_direction(const orc_heat *h, int64_t c, int q, const double v[3], double b[3])
{
  const int n = h->n;
  const double xi[3] = {h->xg[q % n], h->xg[(q / n) % n], h->xg[q / (n * n)]};
  double x[3], J[3][3];
  cell_map(h, c, xi, x, J);
  const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                     J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
  double inv[3][3];
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) {
      /* cofactor of J[j][i] */
      const int r0 = (j + 1) % 3, r1 = (j + 2) % 3, c0 = (i + 1) % 3, c1 = (i + 2) % 3;
      inv[i][j] = (J[r0][c0] * J[r1][c1] - J[r0][c1] * J[r1][c0]) / det;
    }
  for (int i = 0; i < 3; ++i) b[i] = inv[i][0] * v[0] + inv[i][1] * v[1] + inv[i][2] * v[2];
}

/* liquid-solid interpolation of one property at temperature T (compute_solid_liquid_phases_
 * property and its temperature derivative, material.templates.hpp:540-600,745-780): solid
 * fraction sf from the mushy zone (or sharp at T_solidus), cubic smoothstep
 * interpolate_cubic(sf, l, s) = l + (s - l) (3 sf^2 - 2 sf^3), derivative
 * -(s - l) 6 sf (1 - sf) / (T_liquidus - T_solidus), both exact at sf = 0 and 1 */
static inline double solid_fraction(const orc_material *m, double T)
{
  if (m->sharp) return T < m->T_solidus ? 1.0 : 0.0;
  const double inv_mushy = 1.0 / (m->T_liquidus - m->T_solidus);
  const double sf = (m->T_liquidus - T) * inv_mushy;
  return sf < 0.0 ? 0.0 : (sf > 1.0 ? 1.0 : sf);
}

static inline void ls_interp(const orc_material *m, double T, double l, double s, double *val,
                             double *dval)
{
  const double inv_mushy = 1.0 / (m->T_liquidus - m->T_solidus);
  const double sf = solid_fraction(m, T);
  const double hs = -2.0 * sf * sf * sf + 3.0 * sf * sf; /* interpolate_cubic weight */
  const double dhs = -6.0 * sf * sf + 6.0 * sf;           /* its derivative */
  const int edge = (sf == 0.0 || sf == 1.0);
  *val = sf == 0.0 ? l : (sf == 1.0 ? s : l + (s - l) * hs);
  *dval = edge ? 0.0 : -1.0 * inv_mushy * ((s - l) * dhs);
}

/* ramp from (x1, y1) to (x2, y2) with zero slope at both ends: quadratic over the first and the
 * last `delta`, linear in between with the slope s = (y2 - y1) / (x2 - x1 - delta) that makes the
 * pieces meet with continuous slopes (qlq_zero_slope, source/heat/apparent_capacity.cpp:41-110);
 * *dy its derivative */
static inline double qlq_ramp(double x, double x1, double x2, double y1, double y2, double delta,
                              double *dy)
{
  const double s = (y2 - y1) / (x2 - x1 - delta);
  if (x < x1 + delta) {
    *dy = s / delta * (x - x1);
    return y1 + 0.5 * s / delta * (x - x1) * (x - x1);
  }
  if (x > x2 - delta) {
    *dy = -s / delta * (x - x2);
    return y2 - 0.5 * s / delta * (x - x2) * (x - x2);
  }
  *dy = s;
  return y1 + s * (x - x1 - 0.5 * delta);
}

/* apparent heat capacity of the latent heat of fusion L in the mushy zone, added to the liquid-
 * solid specific heat capacity when L > 0 (Heat::ApparentCapacity, apparent_capacity.cpp:
 * 157-300; compute_solid_liquid_phases_specific_heat_capacity and its derivative,
 * material.templates.hpp:562-616; material.hpp:655-656): zero unless 0 < sf < 1; with
 * dT = T_l - T_s each profile integrates to L over [T_s, T_l]:
 *   CONSTANT    L / dT
 *   QLQ         qlq_ramp from (T_s, 0) to (T_mid, 2 L / dT) and back to (T_l, 0), delta = dT / 6,
 *               at T = T_l - sf dT
 *   POLY4_BELL  (2 L / dT) f(xi), f(x) = 15/16 (x^2 - 1)^2, xi = 1 - 2 sf
 * *dA is the temperature derivative. */
static inline double apparent_capacity(const orc_material *m, double sf, double *dA)
{
  *dA = 0.0;
  if (!(m->latent_heat > 0.0) || sf <= 0.0 || sf >= 1.0) return 0.0;
  const double L = m->latent_heat, dT = m->T_liquidus - m->T_solidus;
  if (m->apparent_capacity == ORC_APPARENT_CONSTANT) return L / dT;
  if (m->apparent_capacity == ORC_APPARENT_POLY4_BELL) {
    const double r = 2.0 / dT, xi = 1.0 - 2.0 * sf, q = xi * xi - 1.0;
    *dA = L * r * r * 3.75 * xi * q;
    return L * r * 0.9375 * q * q;
  }
  const double T = m->T_liquidus - sf * dT, Tm = 0.5 * (m->T_solidus + m->T_liquidus);
  const double peak = 2.0 * L / dT, delta = dT / 6.0;
  return T <= Tm ? qlq_ramp(T, m->T_solidus, Tm, 0.0, peak, delta, dA)
                 : qlq_ramp(T, Tm, m->T_liquidus, peak, 0.0, delta, dA);
}

/* Material::compute_parameters of the heat operator's material types at temperature T and
 * level-set heaviside H (material.templates.hpp:104-137, 226-500), as rho*cp, k and their
 * temperature derivatives (HeatDiffuseMultiPhaseOperator::get_material_parameters_and_
 * derivatives, heat_diffuse_operator.cpp:1165-1215):
 *   CONSTANT          liquid values
 *   LINEAR_K          k = k_l + k1 T (no reference counterpart)
 *   LIQUID_SOLID      ls_interp of every property (:296-375)
 *   GAS_LIQUID        (1 - w) gas + w liquid, w = H or heaviside(H, 0.5) = H > 0.5
 *                     (LevelSet::Tools::interpolate, level_set_tools.hpp:40-43; :240-295,
 *                     :515-524, characteristic_functions.hpp:37-40); no T derivatives
 *   GAS_LIQUID_SOLID  (1 - w) gas + w ls_interp(T), derivatives w d ls_interp / dT (:376-500,
 *                     :620-740)
 * rho*cp is the product of the interpolated density and capacity, or with volume_specific the
 * interpolated rho*cp of the phases (:1138-1162). */
static inline void material_eval(const orc_material *m, double T, double H, double *rhocp,
                                 double *k, double *drhocp, double *dk)
{
  const int law = m->law;
  if (law == ORC_LAW_CONSTANT) {
    *rhocp = m->rho_l * m->cp_l;
    *k = m->k_l;
    *drhocp = 0.0;
    *dk = 0.0;
    return;
  }
  if (law == ORC_LAW_LINEAR_K) {
    *rhocp = m->rho_l * m->cp_l;
    *k = m->k_l + m->k1 * T;
    *drhocp = 0.0;
    *dk = m->k1;
    return;
  }
  /* phase values of the liquid(-solid) side and their T derivatives */
  double rho = 0.0, cp = 0.0, kk = 0.0, vs = 0.0, drho = 0.0, dcp = 0.0, dkk = 0.0, dvs = 0.0;
  if (law == ORC_LAW_GAS_LIQUID) {
    rho = m->rho_l, cp = m->cp_l, kk = m->k_l, vs = m->rho_l * m->cp_l;
    drho = dcp = dkk = dvs = 0.0;
  } else {
    ls_interp(m, T, m->k_l, m->k_s, &kk, &dkk);
    if (m->volume_specific) {
      ls_interp(m, T, m->rho_l * m->cp_l, m->rho_s * m->cp_s, &vs, &dvs);
    } else {
      ls_interp(m, T, m->rho_l, m->rho_s, &rho, &drho);
      ls_interp(m, T, m->cp_l, m->cp_s, &cp, &dcp);
      double dA;
      cp += apparent_capacity(m, solid_fraction(m, T), &dA);
      dcp += dA;
    }
  }
  if (law == ORC_LAW_LIQUID_SOLID) {
    *k = kk;
    *dk = dkk;
    if (m->volume_specific) {
      *rhocp = vs;
      *drhocp = dvs;
    } else {
      *rhocp = rho * cp;
      *drhocp = dcp * rho + drho * cp;
    }
    return;
  }
  /* gas mixing */
  const double w = m->sharp_gas_liquid ? (H > 0.5 ? 1.0 : 0.0) : H;
#define MIX(liq, gas) ((1.0 - w) * (gas) + w * (liq))
  *k = MIX(kk, m->k_g);
  *dk = w * dkk;
  if (m->volume_specific) {
    *rhocp = MIX(law == ORC_LAW_GAS_LIQUID ? m->rho_l * m->cp_l : vs, m->rho_g * m->cp_g);
    *drhocp = w * dvs;
  } else {
    const double r = MIX(rho, m->rho_g), c = MIX(cp, m->cp_g);
    *rhocp = r * c;
    *drhocp = (w * dcp) * r + (w * drho) * c;
  }
#undef MIX
}

void orc_material_eval(const orc_material *m, double T, double H, double out[4])
{
  material_eval(m, T, H, &out[0], &out[1], &out[2], &out[3]);
}

/* ------------------------------------------------------------------ */
/* form 0: sum factorisation over cell batches                         */
/* ------------------------------------------------------------------ */

typedef double lane_t[ORC_VEC];

/* one 1D sweep of matrix M along direction dir over all n^2 lines; even-odd */
static inline __attribute__((always_inline)) void sweep(const int n, const int dir,
                                                        const mat1d *M, const lane_t *in,
                                                        lane_t *out, const int add)
{
  const int st = dir == 0 ? 1 : (dir == 1 ? n : n * n);
  const int h = n / 2;
  for (int b = 0; b < n; ++b)
    for (int a = 0; a < n; ++a) {
      const int base = dir == 0 ? n * (a + n * b) : (dir == 1 ? a + n * n * b : a + n * b);
      lane_t e[NMAX / 2 + 1], od[NMAX / 2 + 1], mid;
      for (int l = 0; l < h; ++l)
        for (int v = 0; v < ORC_VEC; ++v) {
          e[l][v] = in[base + l * st][v] + in[base + (n - 1 - l) * st][v];
          od[l][v] = in[base + l * st][v] - in[base + (n - 1 - l) * st][v];
        }
      if (n & 1)
        for (int v = 0; v < ORC_VEC; ++v) mid[v] = in[base + h * st][v];
      for (int o = 0; o < h + (n & 1); ++o) {
        lane_t E, O;
        for (int v = 0; v < ORC_VEC; ++v) {
          E[v] = (n & 1) ? M->a[o][h] * mid[v] : 0.0;
          O[v] = 0.0;
        }
        for (int l = 0; l < h; ++l)
          for (int v = 0; v < ORC_VEC; ++v) {
            E[v] += M->ae[o][l] * e[l][v];
            O[v] += M->ao[o][l] * od[l][v];
          }
        if (o < h) {
          double *p0 = out[base + o * st], *p1 = out[base + (n - 1 - o) * st];
          for (int v = 0; v < ORC_VEC; ++v) {
            const double y0 = E[v] + O[v], y1 = M->sym * (E[v] - O[v]);
            p0[v] = add ? p0[v] + y0 : y0;
            p1[v] = add ? p1[v] + y1 : y1;
          }
        } else {
          double *p0 = out[base + o * st];
          for (int v = 0; v < ORC_VEC; ++v) {
            const double y0 = E[v] + O[v];
            p0[v] = add ? p0[v] + y0 : y0;
          }
        }
      }
    }
}

typedef struct {
  lane_t u[NPT_MAX], t1[NPT_MAX], t2[NPT_MAX];
  lane_t uq[NPT_MAX], gx[NPT_MAX], gy[NPT_MAX], gz[NPT_MAX];
  lane_t Tq[NPT_MAX], Tx[NPT_MAX], Ty[NPT_MAX], Tz[NPT_MAX], Toq[NPT_MAX], Sq[NPT_MAX];
  lane_t Hq[NPT_MAX], Vq[3][NPT_MAX];
  lane_t c[10][NPT_MAX];
} scratch_t;

static inline int64_t cell_base_dof(const orc_heat *h, int64_t c)
{
  int cx, cy, cz;
  cell_coords(h, c, &cx, &cy, &cz);
  return (int64_t)h->p * cx + (int64_t)h->nd[0] * ((int64_t)h->p * cy + (int64_t)h->nd[1] * h->p * cz);
}

static inline void gather(const orc_heat *h, const int64_t *cells, int nl, const double *src,
                          int masked, lane_t *u)
{
  const int n = h->n;
  for (int v = 0; v < ORC_VEC; ++v) {
    if (v >= nl) {
      for (int q = 0; q < h->npt; ++q) u[q][v] = 0.0;
      continue;
    }
    const int64_t base = cell_base_dof(h, cells[v]);
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          const int64_t g = base + i + (int64_t)h->nd[0] * (j + (int64_t)h->nd[1] * k);
          u[i + n * (j + n * k)][v] = (masked && h->mask[g]) ? 0.0 : src[g];
        }
  }
}

static inline void scatter_add(const orc_heat *h, const int64_t *cells, int nl, const lane_t *r,
                               double *dst)
{
  const int n = h->n;
  for (int v = 0; v < nl; ++v) {
    const int64_t base = cell_base_dof(h, cells[v]);
    for (int k = 0; k < n; ++k)
      for (int j = 0; j < n; ++j)
        for (int i = 0; i < n; ++i) {
          const int64_t g = base + i + (int64_t)h->nd[0] * (j + (int64_t)h->nd[1] * k);
          if (!h->mask[g]) dst[g] += r[i + n * (j + n * k)][v];
        }
  }
}

/* geometry of lane v at point q: JxW and G (with weights) */
static inline void geo_at(const orc_heat *h, const int64_t *cells, int nl, int v, int q,
                          double *jxw, double G[6])
{
  const int64_t c = cells[v < nl ? v : 0];
  if (h->affine) {
    const double *g = h->geo + 7 * c;
    const double w = h->wq[q];
    *jxw = g[0] * w;
    for (int t = 0; t < 6; ++t) G[t] = g[1 + t] * w;
  } else {
    const double *g = h->geo + 7 * (c * h->npt + q);
    *jxw = g[0];
    for (int t = 0; t < 6; ++t) G[t] = g[1 + t];
  }
}

/* values at q-points (3 sweeps) and collocation gradients (3 sweeps) */
static inline __attribute__((always_inline)) void eval_vg(const orc_heat *h, const int n,
                                                          lane_t *u, scratch_t *s, lane_t *vq,
                                                          lane_t *dx, lane_t *dy, lane_t *dz)
{
  sweep(n, 0, &h->mS, u, s->t1, 0);
  sweep(n, 1, &h->mS, s->t1, s->t2, 0);
  sweep(n, 2, &h->mS, s->t2, vq, 0);
  if (dx) {
    sweep(n, 0, &h->mD, vq, dx, 0);
    sweep(n, 1, &h->mD, vq, dy, 0);
    sweep(n, 2, &h->mD, vq, dz, 0);
  }
}

/* heaviside and velocity values at the q-points of a batch (fields mode) */
static inline __attribute__((always_inline)) void eval_fields(const orc_heat *h, const int n,
                                                              const int64_t *cells, int nl,
                                                              scratch_t *s)
{
  const int npt = n * n * n;
  if (h->Hf) {
    gather(h, cells, nl, h->Hf, 0, s->u);
    eval_vg(h, n, s->u, s, s->Hq, NULL, NULL, NULL);
  } else {
    for (int q = 0; q < npt; ++q)
      for (int v = 0; v < ORC_VEC; ++v) s->Hq[q][v] = 1.0;
  }
  for (int d = 0; d < 3; ++d) {
    if (h->vel) {
      gather(h, cells, nl, h->vel + (size_t)d * h->n_dofs, 0, s->u);
      eval_vg(h, n, s->u, s, s->Vq[d], NULL, NULL, NULL);
    } else {
      for (int q = 0; q < npt; ++q)
        for (int v = 0; v < ORC_VEC; ++v) s->Vq[d][q][v] = 0.0;
    }
  }
}

/* coefficients of lane v at point q: rho*cp, k, their T derivatives at temperature T and
 * the heaviside value there, and the reference-space transport vector b = J^-1 v (zero
 * without a velocity field) */
static inline void point_coefs(const orc_heat *h, const int64_t *cells, int nl, int v, int q,
                               const scratch_t *s, double T, double *rhocp, double *k,
                               double *drhocp, double *dk, double b[3])
{
  material_eval(&h->mat, T, h->fields ? s->Hq[q][v] : 1.0, rhocp, k, drhocp, dk);
  if (h->vel) {
    const double vv[3] = {s->Vq[0][q][v], s->Vq[1][q][v], s->Vq[2][q][v]};
    ref_direction(h, cells[v < nl ? v : 0], q, vv, b);
  } else {
    b[0] = b[1] = b[2] = 0.0;
  }
}

/* out = S^T (val + sum_d D_d^T f_d) ; val in vq, fluxes in fx, fy, fz */
static inline __attribute__((always_inline)) void integrate_vg(const orc_heat *h, const int n,
                                                               lane_t *vq, lane_t *fx,
                                                               lane_t *fy, lane_t *fz,
                                                               scratch_t *s, lane_t *out)
{
  sweep(n, 0, &h->mDT, fx, vq, 1);
  sweep(n, 1, &h->mDT, fy, vq, 1);
  sweep(n, 2, &h->mDT, fz, vq, 1);
  sweep(n, 2, &h->mST, vq, s->t1, 0);
  sweep(n, 1, &h->mST, s->t1, s->t2, 0);
  sweep(n, 0, &h->mST, s->t2, out, 0);
}

/* kind: 0 vmult, 1 rhs, 2 diagonal, 3 l2 norm accumulate, 4 vmult without the
 * dk/dT grad(T_lin) u term (Picard operator), 5 the diagonal of that operator */
static inline __attribute__((always_inline)) void batch_kernel(
  const orc_heat *h, const int n, const int kind, const int64_t *cells, int nl, double *dst,
  const double *src, const double *Tl, const double *To, const double *qs, scratch_t *s,
  double *acc)
{
  const int npt = n * n * n;
  const double idt = 1.0 / h->dt;
  if (h->fields && kind != 3) eval_fields(h, n, cells, nl, s);
  if (kind == 0 || kind == 4) {
    gather(h, cells, nl, src, 1, s->u);
    eval_vg(h, n, s->u, s, s->uq, s->gx, s->gy, s->gz);
    if (h->tdep) {
      gather(h, cells, nl, Tl, 0, s->u);
      eval_vg(h, n, s->u, s, s->Tq, s->Tx, s->Ty, s->Tz);
      if (h->need_told) {
        gather(h, cells, nl, To, 0, s->u);
        eval_vg(h, n, s->u, s, s->Toq, NULL, NULL, NULL);
      }
    }
    for (int q = 0; q < npt; ++q)
      for (int v = 0; v < ORC_VEC; ++v) {
        double jxw, G[6], rhocp, k, drhocp, dk, b[3];
        geo_at(h, cells, nl, v, q, &jxw, G);
        point_coefs(h, cells, nl, v, q, s, h->tdep ? s->Tq[q][v] : 0.0, &rhocp, &k, &drhocp, &dk, b);
        double cval = idt * rhocp;
        /* convection rho_cp v.grad(u), and with a temperature-dependent law
         * d(rho_cp)/dT (v.grad T_lin) u (heat_diffuse_operator.cpp:1038-1049) */
        double conv = rhocp * (b[0] * s->gx[q][v] + b[1] * s->gy[q][v] + b[2] * s->gz[q][v]);
        if (h->tdep)
          conv += drhocp * (b[0] * s->Tx[q][v] + b[1] * s->Ty[q][v] + b[2] * s->Tz[q][v]) *
                  s->uq[q][v];
        double g0 = k * s->gx[q][v], g1 = k * s->gy[q][v], g2 = k * s->gz[q][v];
        if (h->tdep) {
          if (h->need_told) cval += idt * drhocp * (s->Tq[q][v] - s->Toq[q][v]);
          const double uu = s->uq[q][v];
          if (kind == 4) dk = 0.0;
          g0 += dk * s->Tx[q][v] * uu;
          g1 += dk * s->Ty[q][v] * uu;
          g2 += dk * s->Tz[q][v] * uu;
        }
        s->uq[q][v] = (cval * s->uq[q][v] + conv) * jxw;
        s->gx[q][v] = G[0] * g0 + G[1] * g1 + G[2] * g2;
        s->gy[q][v] = G[1] * g0 + G[3] * g1 + G[4] * g2;
        s->gz[q][v] = G[2] * g0 + G[4] * g1 + G[5] * g2;
      }
    integrate_vg(h, n, s->uq, s->gx, s->gy, s->gz, s, s->u);
    scatter_add(h, cells, nl, s->u, dst);
  } else if (kind == 1) {
    gather(h, cells, nl, Tl, 0, s->u);
    eval_vg(h, n, s->u, s, s->Tq, s->Tx, s->Ty, s->Tz);
    gather(h, cells, nl, To, 0, s->u);
    eval_vg(h, n, s->u, s, s->Toq, NULL, NULL, NULL);
    gather(h, cells, nl, qs, 0, s->u);
    eval_vg(h, n, s->u, s, s->Sq, NULL, NULL, NULL);
    for (int q = 0; q < npt; ++q)
      for (int v = 0; v < ORC_VEC; ++v) {
        double jxw, G[6], rhocp, k, drhocp, dk, b[3];
        geo_at(h, cells, nl, v, q, &jxw, G);
        point_coefs(h, cells, nl, v, q, s, s->Tq[q][v], &rhocp, &k, &drhocp, &dk, b);
        /* rhs_cell_loop value term with the convection rho_cp grad(T).v (:493-500) */
        const double val = idt * rhocp * (s->Tq[q][v] - s->Toq[q][v]) - s->Sq[q][v] +
                           rhocp * (b[0] * s->Tx[q][v] + b[1] * s->Ty[q][v] + b[2] * s->Tz[q][v]);
        const double g0 = k * s->Tx[q][v], g1 = k * s->Ty[q][v], g2 = k * s->Tz[q][v];
        s->uq[q][v] = -val * jxw;
        s->gx[q][v] = -(G[0] * g0 + G[1] * g1 + G[2] * g2);
        s->gy[q][v] = -(G[1] * g0 + G[3] * g1 + G[4] * g2);
        s->gz[q][v] = -(G[2] * g0 + G[4] * g1 + G[5] * g2);
      }
    integrate_vg(h, n, s->uq, s->gx, s->gy, s->gz, s, s->u);
    scatter_add(h, cells, nl, s->u, dst);
  } else if (kind == 2 || kind == 5) {
    /* closed-form diagonal: sum_q c0 phi_i^2 + grad phi_i^T (kG) grad phi_i
     *                       + dk phi_i grad phi_i^T G grad T  (kind 5: without the last) */
    if (h->tdep) {
      gather(h, cells, nl, Tl, 0, s->u);
      eval_vg(h, n, s->u, s, s->Tq, s->Tx, s->Ty, s->Tz);
      if (h->need_told) {
        gather(h, cells, nl, To, 0, s->u);
        eval_vg(h, n, s->u, s, s->Toq, NULL, NULL, NULL);
      }
    }
    lane_t *C0 = s->c[0], *Gxx = s->c[1], *Gxy = s->c[2], *Gxz = s->c[3], *Gyy = s->c[4],
           *Gyz = s->c[5], *Gzz = s->c[6], *Bx = s->c[7], *By = s->c[8], *Bz = s->c[9];
    for (int q = 0; q < npt; ++q)
      for (int v = 0; v < ORC_VEC; ++v) {
        double jxw, G[6], rhocp, k, drhocp, dk, b[3];
        geo_at(h, cells, nl, v, q, &jxw, G);
        point_coefs(h, cells, nl, v, q, s, h->tdep ? s->Tq[q][v] : 0.0, &rhocp, &k, &drhocp, &dk, b);
        double cval = idt * rhocp;
        if (h->tdep && h->need_told) cval += idt * drhocp * (s->Tq[q][v] - s->Toq[q][v]);
        C0[q][v] = cval * jxw;
        if (h->tdep) /* d(rho_cp)/dT (v.grad T_lin) u: a mass-like term */
          C0[q][v] += drhocp * (b[0] * s->Tx[q][v] + b[1] * s->Ty[q][v] + b[2] * s->Tz[q][v]) * jxw;
        Gxx[q][v] = k * G[0];
        Gxy[q][v] = 2.0 * k * G[1];
        Gxz[q][v] = 2.0 * k * G[2];
        Gyy[q][v] = k * G[3];
        Gyz[q][v] = 2.0 * k * G[4];
        Gzz[q][v] = k * G[5];
        /* convection: phi_i (JxW rho_cp J^-1 v).grad_ref(phi_i) */
        Bx[q][v] = jxw * rhocp * b[0];
        By[q][v] = jxw * rhocp * b[1];
        Bz[q][v] = jxw * rhocp * b[2];
        if (h->tdep && kind == 2) {
          const double t0 = s->Tx[q][v], t1 = s->Ty[q][v], t2 = s->Tz[q][v];
          Bx[q][v] += dk * (G[0] * t0 + G[1] * t1 + G[2] * t2);
          By[q][v] += dk * (G[1] * t0 + G[3] * t1 + G[4] * t2);
          Bz[q][v] += dk * (G[2] * t0 + G[4] * t1 + G[5] * t2);
        }
      }
    /* (x,y) = (P,P): z P C0 + z Q Gzz + z R Bz */
    lane_t *A = s->t1, *B = s->t2, *X = s->uq, *Y = s->gx, *Z = s->gy, *W = s->gz;
    sweep(n, 2, &h->mPT, C0, A, 0);
    sweep(n, 2, &h->mQT, Gzz, A, 1);
    sweep(n, 2, &h->mRT, Bz, A, 1);
    sweep(n, 1, &h->mPT, A, X, 0); /* X: y-swept, x pending P */
    /* (P,Q): z P Gyy */
    sweep(n, 2, &h->mPT, Gyy, A, 0);
    sweep(n, 1, &h->mQT, A, X, 1);
    /* (P,R): z R Gyz + z P By */
    sweep(n, 2, &h->mRT, Gyz, A, 0);
    sweep(n, 2, &h->mPT, By, A, 1);
    sweep(n, 1, &h->mRT, A, X, 1);
    /* x P on X */
    sweep(n, 0, &h->mPT, X, W, 0);
    /* (Q,P): z P Gxx, y P, x Q */
    sweep(n, 2, &h->mPT, Gxx, A, 0);
    sweep(n, 1, &h->mPT, A, B, 0);
    sweep(n, 0, &h->mQT, B, W, 1);
    /* (R,R): z P Gxy, y R ; (R,P): z R Gxz + z P Bx, y P ; then x R */
    sweep(n, 2, &h->mPT, Gxy, A, 0);
    sweep(n, 1, &h->mRT, A, Y, 0);
    sweep(n, 2, &h->mRT, Gxz, A, 0);
    sweep(n, 2, &h->mPT, Bx, A, 1);
    sweep(n, 1, &h->mPT, A, Y, 1);
    sweep(n, 0, &h->mRT, Y, W, 1);
    (void)Z;
    scatter_add(h, cells, nl, W, dst);
  } else {
    gather(h, cells, nl, src, 0, s->u);
    eval_vg(h, n, s->u, s, s->uq, NULL, NULL, NULL);
    for (int v = 0; v < nl; ++v) {
      double sum = 0.0;
      for (int q = 0; q < npt; ++q) {
        double jxw, G[6];
        geo_at(h, cells, nl, v, q, &jxw, G);
        sum += s->uq[q][v] * s->uq[q][v] * jxw;
      }
      *acc += sum;
    }
  }
}

#define DEF_BATCH(N)                                                                          \
  static void batch_##N(const orc_heat *h, int kind, const int64_t *cells, int nl, double *dst, \
                        const double *src, const double *Tl, const double *To,               \
                        const double *qs, scratch_t *s, double *acc)                         \
  {                                                                                           \
    batch_kernel(h, N, kind, cells, nl, dst, src, Tl, To, qs, s, acc);                        \
  }
DEF_BATCH(2)
DEF_BATCH(3)
DEF_BATCH(4)
DEF_BATCH(5)
DEF_BATCH(6)
DEF_BATCH(7)

typedef void (*batch_fn)(const orc_heat *, int, const int64_t *, int, double *, const double *,
                         const double *, const double *, const double *, scratch_t *, double *);

static batch_fn pick_batch(int n)
{
  switch (n) {
  case 2: return batch_2;
  case 3: return batch_3;
  case 4: return batch_4;
  case 5: return batch_5;
  case 6: return batch_6;
  default: return batch_7;
  }
}

static double run_sf(const orc_heat *h, int kind, double *dst, const double *src, const double *Tl,
                     const double *To, const double *qs)
{
  batch_fn fn = pick_batch(h->n);
  double total = 0.0;
  const int nt = nthreads();
  scratch_t **scr = (scratch_t **)malloc(sizeof(scratch_t *) * nt);
  for (int t = 0; t < nt; ++t) scr[t] = (scratch_t *)aligned_alloc(64, sizeof(scratch_t));
  for (int col = 0; col < 8; ++col) {
    const int64_t nc = h->color_n[col];
    const int64_t nb = (nc + ORC_VEC - 1) / ORC_VEC;
    double acc = 0.0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 16) reduction(+ : acc)
    for (int64_t b = 0; b < nb; ++b) {
      const int64_t first = b * ORC_VEC;
      const int nl = (int)((nc - first) < ORC_VEC ? (nc - first) : ORC_VEC);
      double a = 0.0;
      fn(h, kind, h->color_cells[col] + first, nl, dst, src, Tl, To, qs,
         scr[omp_get_thread_num()], &a);
      acc += a;
    }
    total += acc;
  }
  for (int t = 0; t < nt; ++t) free(scr[t]);
  free(scr);
  return total;
}

/* ------------------------------------------------------------------ */
/* form 1: direct quadrature, one cell at a time                      */
/* ------------------------------------------------------------------ */

static void run_direct(const orc_heat *h, int kind, double *dst, const double *src,
                       const double *Tl, const double *To)
{
  const int n = h->n, npt = h->npt;
  const double idt = 1.0 / h->dt;
  for (int col = 0; col < 8; ++col) {
    const int64_t nc = h->color_n[col];
#pragma omp parallel for num_threads(nthreads()) schedule(dynamic, 4)
    for (int64_t ic = 0; ic < nc; ++ic) {
      const int64_t c = h->color_cells[col][ic];
      const int64_t base = cell_base_dof(h, c);
      double u[NPT_MAX], T[NPT_MAX], To_[NPT_MAX], out[NPT_MAX], Hn[NPT_MAX], Vn[3][NPT_MAX];
      int64_t gidx[NPT_MAX];
      for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
          for (int i = 0; i < n; ++i) {
            const int l = i + n * (j + n * k);
            gidx[l] = base + i + (int64_t)h->nd[0] * (j + (int64_t)h->nd[1] * k);
            u[l] = (kind == 0 && !h->mask[gidx[l]]) ? src[gidx[l]] : 0.0;
            T[l] = h->tdep ? Tl[gidx[l]] : 0.0;
            To_[l] = h->need_told ? To[gidx[l]] : 0.0;
            Hn[l] = h->Hf ? h->Hf[gidx[l]] : 1.0;
            for (int e = 0; e < 3; ++e) Vn[e][l] = h->vel ? h->vel[(size_t)e * h->n_dofs + gidx[l]] : 0.0;
            out[l] = 0.0;
          }
      const int64_t one[1] = {c};
      for (int q = 0; q < npt; ++q) {
        const double *ph = h->phi + (size_t)q * npt, *dph = h->dphi + (size_t)q * npt * 3;
        double uq = 0, gu[3] = {0, 0, 0}, Tq = 0, gT[3] = {0, 0, 0}, Toq = 0, Hq = 0,
               vq[3] = {0, 0, 0};
        for (int i = 0; i < npt; ++i) {
          uq += ph[i] * u[i];
          Tq += ph[i] * T[i];
          Toq += ph[i] * To_[i];
          Hq += ph[i] * Hn[i];
          for (int e = 0; e < 3; ++e) vq[e] += ph[i] * Vn[e][i];
          for (int d = 0; d < 3; ++d) {
            gu[d] += dph[3 * i + d] * u[i];
            gT[d] += dph[3 * i + d] * T[i];
          }
        }
        double jxw, G[6], rhocp, k, drhocp, dk, b[3] = {0.0, 0.0, 0.0};
        geo_at(h, one, 1, 0, q, &jxw, G);
        material_eval(&h->mat, Tq, h->fields ? Hq : 1.0, &rhocp, &k, &drhocp, &dk);
        if (h->vel) ref_direction(h, c, q, vq, b);
        const double bT = b[0] * gT[0] + b[1] * gT[1] + b[2] * gT[2];
        double cval = idt * rhocp;
        if (h->tdep && h->need_told) cval += idt * drhocp * (Tq - Toq);
        if (!h->tdep) dk = 0.0;
        const double Gm[3][3] = {{G[0], G[1], G[2]}, {G[1], G[3], G[4]}, {G[2], G[4], G[5]}};
        if (kind == 0) {
          double f[3], F[3];
          for (int d = 0; d < 3; ++d) f[d] = k * gu[d] + dk * gT[d] * uq;
          for (int d = 0; d < 3; ++d) F[d] = Gm[d][0] * f[0] + Gm[d][1] * f[1] + Gm[d][2] * f[2];
          const double val = (cval * uq + rhocp * (b[0] * gu[0] + b[1] * gu[1] + b[2] * gu[2]) +
                              (h->tdep ? drhocp * bT * uq : 0.0)) * jxw;
          for (int i = 0; i < npt; ++i)
            out[i] += ph[i] * val + dph[3 * i] * F[0] + dph[3 * i + 1] * F[1] + dph[3 * i + 2] * F[2];
        } else {
          double BT[3];
          for (int d = 0; d < 3; ++d)
            BT[d] = dk * (Gm[d][0] * gT[0] + Gm[d][1] * gT[1] + Gm[d][2] * gT[2]) +
                    jxw * rhocp * b[d];
          for (int i = 0; i < npt; ++i) {
            const double *g = dph + 3 * i;
            double s = (cval + (h->tdep ? drhocp * bT : 0.0)) * jxw * ph[i] * ph[i];
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) s += k * g[a] * Gm[a][b] * g[b];
            s += ph[i] * (g[0] * BT[0] + g[1] * BT[1] + g[2] * BT[2]);
            out[i] += s;
          }
        }
      }
      for (int i = 0; i < npt; ++i)
        if (!h->mask[gidx[i]]) dst[gidx[i]] += out[i];
    }
  }
}

/* ------------------------------------------------------------------ */
/* boundary faces: direct 2D quadrature on the flat box faces          */
/* ------------------------------------------------------------------ */

#define ORC_SIGMA 5.670374419e-8 /* physical_constants.hpp:6 */

int orc_set_boundary(orc_heat *h, int face, int type, double h_conv, double T_inf_conv,
                     double emissivity, double T_inf_rad, double q_n)
{
  if (face < 0 || face > 5) return -1;
  if ((type & 4) && (type & 3)) return -1; /* heat_diffuse_operator.cpp:708-712 */
  h->btype[face] = type;
  h->bh[face] = h_conv;
  h->bTc[face] = T_inf_conv;
  h->beps[face] = emissivity;
  h->bTr[face] = T_inf_rad;
  h->bqn[face] = q_n;
  return 0;
}

/* kind 0: dst += tangent u ; 1: dst += rhs(T) ; 2: dst += diagonal */
static void run_faces(const orc_heat *h, int kind, double *dst, const double *src,
                      const double *T)
{
  const int n = h->n, p = h->p;
  for (int f = 0; f < 6; ++f) {
    const int type = h->btype[f];
    if (!type) continue;
    const int d = f / 2, ea = d == 0 ? 1 : 0, eb = d == 2 ? 1 : 2;
    const double ha = (h->hi[ea] - h->lo[ea]) / h->m[ea], hb = (h->hi[eb] - h->lo[eb]) / h->m[eb];
    const int fixed = (f & 1) ? h->nd[d] - 1 : 0;
    for (int cb = 0; cb < h->m[eb]; ++cb)
      for (int ca = 0; ca < h->m[ea]; ++ca) {
        int64_t g[NMAX * NMAX];
        double u[NMAX * NMAX], Tv[NMAX * NMAX], out[NMAX * NMAX];
        for (int ib = 0; ib < n; ++ib)
          for (int ia = 0; ia < n; ++ia) {
            int64_t pos[3];
            pos[d] = fixed;
            pos[ea] = (int64_t)p * ca + ia;
            pos[eb] = (int64_t)p * cb + ib;
            const int l = ia + n * ib;
            g[l] = pos[0] + h->nd[0] * (pos[1] + (int64_t)h->nd[1] * pos[2]);
            u[l] = (kind == 0 && !h->mask[g[l]]) ? src[g[l]] : 0.0;
            Tv[l] = T ? T[g[l]] : 0.0;
            out[l] = 0.0;
          }
        for (int qb = 0; qb < n; ++qb)
          for (int qa = 0; qa < n; ++qa) {
            double uq = 0.0, Tq = 0.0;
            for (int ib = 0; ib < n; ++ib)
              for (int ia = 0; ia < n; ++ia) {
                const double ph = h->S[qa][ia] * h->S[qb][ib];
                uq += ph * u[ia + n * ib];
                Tq += ph * Tv[ia + n * ib];
              }
            const double jxw = ha * hb * h->wg[qa] * h->wg[qb];
            double val;
            if (kind == 1) {
              val = 0.0;
              if (type & 4) val -= h->bqn[f];
              if (type & 2)
                val -= h->beps[f] * ORC_SIGMA * (Tq * Tq * Tq * Tq - pow(h->bTr[f], 4));
              if (type & 1) val -= h->bh[f] * (Tq - h->bTc[f]);
            } else {
              val = 0.0;
              if (type & 1) val += h->bh[f];
              if (type & 2) val += 4.0 * h->beps[f] * ORC_SIGMA * Tq * Tq * Tq;
              if (kind == 0) val *= uq;
            }
            for (int ib = 0; ib < n; ++ib)
              for (int ia = 0; ia < n; ++ia) {
                const double ph = h->S[qa][ia] * h->S[qb][ib];
                out[ia + n * ib] += (kind == 2 ? ph * ph : ph) * val * jxw;
              }
          }
        for (int l = 0; l < n * n; ++l)
          if (!h->mask[g[l]]) dst[g[l]] += out[l];
      }
  }
}

/* ------------------------------------------------------------------ */
/* operator verbs                                                      */
/* ------------------------------------------------------------------ */

void orc_vmult(const orc_heat *h, double *dst, const double *src, const double *T_lin,
               const double *T_old, int form)
{
  memset(dst, 0, sizeof(double) * h->n_dofs);
  if (form == 0 || form == 2)
    run_sf(h, form == 0 ? 0 : 4, dst, src, T_lin, T_old, NULL);
  else
    run_direct(h, 0, dst, src, T_lin, T_old);
  run_faces(h, 0, dst, src, T_lin);
}

void orc_inverse_diagonal(const orc_heat *h, double *d, const double *T_lin, const double *T_old,
                          int form)
{
  memset(d, 0, sizeof(double) * h->n_dofs);
  if (form == 0 || form == 2)
    run_sf(h, form == 0 ? 2 : 5, d, NULL, T_lin, T_old, NULL);
  else
    run_direct(h, 2, d, NULL, T_lin, T_old);
  run_faces(h, 2, d, NULL, T_lin);
#pragma omp parallel for num_threads(nthreads())
  for (int64_t i = 0; i < h->n_dofs; ++i) d[i] = fabs(d[i]) > 1.0e-10 ? 1.0 / d[i] : 1.0;
}

void orc_create_rhs(const orc_heat *h, double *dst, const double *T, const double *T_old,
                    const double *heat_source)
{
  run_sf(h, 1, dst, NULL, T, T_old, heat_source);
  run_faces(h, 1, dst, NULL, T);
}

double orc_l2_norm(const orc_heat *h, const double *u)
{
  return sqrt(run_sf(h, 3, NULL, u, NULL, NULL, NULL));
}

void orc_gaussian_source(const orc_heat *h, double *q, double amp, const double c[3], double r)
{
  double *xyz = (double *)malloc(sizeof(double) * 3 * h->n_dofs);
  orc_support_points(h, xyz);
#pragma omp parallel for num_threads(nthreads())
  for (int64_t i = 0; i < h->n_dofs; ++i) {
    double d2 = 0.0;
    for (int d = 0; d < 3; ++d) d2 += (xyz[3 * i + d] - c[d]) * (xyz[3 * i + d] - c[d]);
    q[i] = amp * exp(-d2 / (r * r));
  }
  free(xyz);
}

/* Volumetric laser intensity profiles at the support points, following
 * include/meltpooldg/heat/laser_intensity_profiles.hpp: UniformIntensityProfile (:62-90),
 * GaussVolumetricIntensityProfile (:175-235), GaussProjectionIntensityProfile with
 * compute_distance_to_line (:36-60, :98-170) and GusarovIntensityProfile (:243-340), as
 * LaserHeatSourceVolumetric::compute_volumetric_heat_source evaluates them
 * (source/heat/laser_heat_source_volumetric.cpp:20-58). */
static double orc_gusarov_dq_dxi(double rho, double lambda, double a, double D, double xi)
{
  if (!(xi < lambda)) return 0.0;
  const double t1 = (3.0 - 3.0 * rho) * (exp(-xi) + rho * exp(xi - 2.0 * lambda)) / (4.0 * rho - 3.0);
  const double br = exp(-lambda) * (1.0 - rho * rho) *
                      (exp(-2.0 * a * xi) * (a - 1.0) + exp(2.0 * a * xi) * (a + 1.0)) -
                    (rho * exp(-2.0 * lambda) + 3.0) *
                      (exp(2.0 * a * (xi - lambda)) * (1.0 - a - rho * (a + 1.0)) -
                       exp(2.0 * a * (lambda - xi)) * (a + rho * (a - 1.0) + 1.0));
  return t1 + 2.0 * a * a * rho / (D * (4.0 * rho - 3.0)) * br;
}

void orc_laser_source(const orc_heat *h, double *q, int profile, double power, const double c[3],
                      const double dir[3], double radius, double rho, double beta, double L,
                      int planar)
{
  double *xyz = (double *)malloc(sizeof(double) * 3 * h->n_dofs);
  orc_support_points(h, xyz);
  const double pi = 3.14159265358979323846;
  const double sq = radius * sqrt(pi / 2.0);
  const double peak_vol = power / (sq * sq * sq);
  const double peak_proj = power / (radius * radius * (pi / 2.0));
  const double lambda = beta * L, a = sqrt(1.0 - rho);
  const double D = (1.0 - a) * (1.0 - a - rho * (1.0 + a)) * exp(-2.0 * a * lambda) -
                   (1.0 + a) * (1.0 + a - rho * (1.0 - a)) * exp(2.0 * a * lambda);
#pragma omp parallel for num_threads(nthreads())
  for (int64_t i = 0; i < h->n_dofs; ++i) {
    const double *x = xyz + 3 * i;
    const double v[3] = {x[0] - c[0], planar ? 0.0 : x[1] - c[1], x[2] - c[2]};
    double val = 0.0;
    if (profile == 0) {
      val = power;
    } else if (profile == 1) {
      const double s = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) / radius;
      val = peak_vol * exp(-2.0 * s * s);
    } else if (profile == 2) {
      const double w[3] = {v[1] * dir[2] - v[2] * dir[1], v[2] * dir[0] - v[0] * dir[2],
                           v[0] * dir[1] - v[1] * dir[0]};
      const double s = sqrt(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]) / radius;
      val = peak_proj * exp(-2.0 * s * s);
    } else {
      const double dist = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
      const double z = -(x[2] - c[2]);
      if (z >= L || z < c[2]) {
        val = 0.0;
      } else {
        const double pd = dist <= radius ? 3.0 * power / (pi * radius * radius) *
                                             pow(1.0 - dist / radius, 2) * pow(1.0 + dist / radius, 2)
                                         : 0.0;
        val = -beta * pd * orc_gusarov_dq_dxi(rho, lambda, a, D, z * beta);
      }
    }
    q[i] = val;
  }
  free(xyz);
}

/* ------------------------------------------------------------------ */
/* vector helpers and solvers                                          */
/* ------------------------------------------------------------------ */

static double dot(int64_t n, const double *a, const double *b)
{
  double s = 0.0;
#pragma omp parallel for num_threads(nthreads()) reduction(+ : s)
  for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}

static double *vec_new(int64_t n) { return (double *)calloc((size_t)n, sizeof(double)); }

void orc_chebyshev_apply(const orc_heat *h, const orc_solver_params *prm, double *x,
                         const double *r, const double *D, const double *T_lin,
                         const double *T_old)
{
  const int64_t N = h->n_dofs;
  const double a = prm->cheb_lambda_min, b = prm->cheb_lambda_max;
  const double theta = 0.5 * (b + a), delta = 0.5 * (b - a), sigma = theta / delta;
  double rho0 = 1.0 / sigma;
  double *d = vec_new(N), *Ax = vec_new(N);
#pragma omp parallel for num_threads(nthreads())
  for (int64_t i = 0; i < N; ++i) {
    d[i] = D[i] * r[i] / theta;
    x[i] = d[i];
  }
  for (int j = 1; j <= prm->cheb_degree; ++j) {
    orc_vmult(h, Ax, x, T_lin, T_old, 0);
    const double rho1 = 1.0 / (2.0 * sigma - rho0);
    const double c1 = rho1 * rho0, c2 = 2.0 * rho1 / delta;
#pragma omp parallel for num_threads(nthreads())
    for (int64_t i = 0; i < N; ++i) {
      d[i] = c1 * d[i] + c2 * D[i] * (r[i] - Ax[i]);
      x[i] += d[i];
    }
    rho0 = rho1;
  }
  free(d);
  free(Ax);
}

static void precond_apply(const orc_heat *h, const orc_solver_params *prm, double *z,
                          const double *r, const double *D, const double *T_lin,
                          const double *T_old)
{
  const int64_t N = h->n_dofs;
  if (prm->precond == 0) {
    memcpy(z, r, sizeof(double) * N);
  } else if (prm->precond == 1) {
#pragma omp parallel for num_threads(nthreads())
    for (int64_t i = 0; i < N; ++i) z[i] = D[i] * r[i];
  } else {
    orc_chebyshev_apply(h, prm, z, r, D, T_lin, T_old);
  }
}

int orc_cg(const orc_heat *h, const orc_solver_params *prm, double *x, const double *b,
           const double *D, const double *T_lin, const double *T_old, double *res_norm)
{
  const int64_t N = h->n_dofs;
  double *r = vec_new(N), *z = vec_new(N), *p = vec_new(N), *Ap = vec_new(N);
  orc_vmult(h, Ap, x, T_lin, T_old, 0);
#pragma omp parallel for num_threads(nthreads())
  for (int64_t i = 0; i < N; ++i) r[i] = b[i] - Ap[i];
  double res = sqrt(dot(N, r, r));
  const double tol = fmax(prm->abs_tolerance, prm->rel_tolerance * res);
  int it = 0, status = 0;
  double rz_old = 0.0;
  while (1) {
    if (res <= tol) break;
    if (it >= prm->max_iterations || isnan(res)) {
      status = -1;
      break;
    }
    precond_apply(h, prm, z, r, D, T_lin, T_old);
    const double rz = dot(N, r, z);
    const double beta = it == 0 ? 0.0 : rz / rz_old;
#pragma omp parallel for num_threads(nthreads())
    for (int64_t i = 0; i < N; ++i) p[i] = z[i] + beta * p[i];
    orc_vmult(h, Ap, p, T_lin, T_old, 0);
    const double alpha = rz / dot(N, p, Ap);
#pragma omp parallel for num_threads(nthreads())
    for (int64_t i = 0; i < N; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * Ap[i];
    }
    rz_old = rz;
    res = sqrt(dot(N, r, r));
    ++it;
  }
  if (res_norm) *res_norm = res;
  free(r);
  free(z);
  free(p);
  free(Ap);
  return status == 0 ? it : -1;
}

/* Restarted GMRES with right preconditioning (deal.II SolverGMRES with
 * right_preconditioning = true, as linear_solver.hpp:113-118 configures it).
 * The monitored quantity is the unpreconditioned residual norm, estimated by
 * the Givens-rotated least-squares residual; restart length = restart. */
int orc_gmres(const orc_heat *h, const orc_solver_params *prm, int restart, double *x,
              const double *b, const double *D, const double *T_lin, const double *T_old,
              double *res_norm)
{
  const int64_t N = h->n_dofs;
  const int m = restart;
  double *V = (double *)calloc((size_t)N * (m + 1), sizeof(double));
  double *Z = vec_new(N), *w = vec_new(N);
  double *H = (double *)calloc((size_t)(m + 1) * m, sizeof(double));
  double *cs = (double *)calloc(m, sizeof(double)), *sn = (double *)calloc(m, sizeof(double));
  double *g = (double *)calloc(m + 1, sizeof(double)), *y = (double *)calloc(m, sizeof(double));
  int it = 0, status = 0, first = 1;
  double tol = 0.0, res = 0.0;
  for (;;) {
    /* r = b - A x */
    orc_vmult(h, w, x, T_lin, T_old, 0);
    for (int64_t i = 0; i < N; ++i) V[i] = b[i] - w[i];
    const double beta = sqrt(dot(N, V, V));
    res = beta;
    if (first) {
      tol = fmax(prm->abs_tolerance, prm->rel_tolerance * beta);
      first = 0;
    }
    if (res <= tol) break;
    if (it >= prm->max_iterations || isnan(res)) {
      status = -1;
      break;
    }
    for (int64_t i = 0; i < N; ++i) V[i] /= beta;
    memset(g, 0, sizeof(double) * (m + 1));
    g[0] = beta;
    int j = 0, done = 0;
    for (; j < m; ++j) {
      double *vj = V + (size_t)j * N, *vn = V + (size_t)(j + 1) * N;
      precond_apply(h, prm, Z, vj, D, T_lin, T_old);
      orc_vmult(h, w, Z, T_lin, T_old, 0);
      /* modified Gram-Schmidt */
      for (int i = 0; i <= j; ++i) {
        const double *vi = V + (size_t)i * N;
        const double hij = dot(N, w, vi);
        H[i * m + j] = hij;
        for (int64_t t = 0; t < N; ++t) w[t] -= hij * vi[t];
      }
      const double hn = sqrt(dot(N, w, w));
      H[(j + 1) * m + j] = hn;
      for (int64_t t = 0; t < N; ++t) vn[t] = hn > 0.0 ? w[t] / hn : 0.0;
      for (int i = 0; i < j; ++i) {
        const double a = H[i * m + j], c = H[(i + 1) * m + j];
        H[i * m + j] = cs[i] * a + sn[i] * c;
        H[(i + 1) * m + j] = -sn[i] * a + cs[i] * c;
      }
      const double a = H[j * m + j], c = H[(j + 1) * m + j];
      const double r = sqrt(a * a + c * c);
      cs[j] = r > 0.0 ? a / r : 1.0;
      sn[j] = r > 0.0 ? c / r : 0.0;
      H[j * m + j] = r;
      H[(j + 1) * m + j] = 0.0;
      g[j + 1] = -sn[j] * g[j];
      g[j] = cs[j] * g[j];
      ++it;
      res = fabs(g[j + 1]);
      if (res <= tol || it >= prm->max_iterations || hn == 0.0) {
        ++j;
        done = 1;
        break;
      }
    }
    /* solve the triangular system and update x += M^-1 V y */
    for (int i = j - 1; i >= 0; --i) {
      double s = g[i];
      for (int k = i + 1; k < j; ++k) s -= H[i * m + k] * y[k];
      y[i] = s / H[i * m + i];
    }
    memset(w, 0, sizeof(double) * N);
    for (int i = 0; i < j; ++i) {
      const double *vi = V + (size_t)i * N;
      for (int64_t t = 0; t < N; ++t) w[t] += y[i] * vi[t];
    }
    precond_apply(h, prm, Z, w, D, T_lin, T_old);
    for (int64_t t = 0; t < N; ++t) x[t] += Z[t];
    if (done && res <= tol) break;
    if (it >= prm->max_iterations) {
      status = -1;
      break;
    }
  }
  if (res_norm) *res_norm = res;
  free(V);
  free(Z);
  free(w);
  free(H);
  free(cs);
  free(sn);
  free(g);
  free(y);
  return status == 0 ? it : -1;
}

/* number of eigenvalues of the symmetric tridiagonal (d, e) below x (Sturm) */
static int sturm_count(int m, const double *d, const double *e, double x)
{
  int cnt = 0;
  double q = d[0] - x;
  if (q < 0) ++cnt;
  for (int i = 1; i < m; ++i) {
    if (q == 0.0) q = 1e-300;
    q = d[i] - x - e[i - 1] * e[i - 1] / q;
    if (q < 0) ++cnt;
  }
  return cnt;
}

static double tridiag_eig(int m, const double *d, const double *e, int which)
{
  double lo = 1e300, hi = -1e300;
  for (int i = 0; i < m; ++i) {
    const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < m - 1 ? fabs(e[i]) : 0.0);
    if (d[i] - r < lo) lo = d[i] - r;
    if (d[i] + r > hi) hi = d[i] + r;
  }
  for (int it = 0; it < 200; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (sturm_count(m, d, e, mid) > which)
      hi = mid;
    else
      lo = mid;
  }
  return 0.5 * (lo + hi);
}

void orc_estimate_eigenvalues(const orc_heat *h, const double *D, const double *T_lin,
                              const double *T_old, int n_it, double *lmin, double *lmax)
{
  const int64_t N = h->n_dofs;
  double *r = vec_new(N), *z = vec_new(N), *p = vec_new(N), *Ap = vec_new(N);
  /* deterministic pseudo-random right-hand side, zero at constrained DoFs */
  for (int64_t i = 0; i < N; ++i) r[i] = h->mask[i] ? 0.0 : hash_sym(12345, (uint64_t)i);
  double *alpha = (double *)calloc(n_it + 1, sizeof(double));
  double *beta = (double *)calloc(n_it + 1, sizeof(double));
  double rz_old = 0.0;
  int m = 0;
  for (int it = 0; it < n_it; ++it) {
    for (int64_t i = 0; i < N; ++i) z[i] = D[i] * r[i];
    const double rz = dot(N, r, z);
    const double b = it == 0 ? 0.0 : rz / rz_old;
    for (int64_t i = 0; i < N; ++i) p[i] = z[i] + b * p[i];
    orc_vmult(h, Ap, p, T_lin, T_old, 0);
    const double pAp = dot(N, p, Ap);
    if (!(pAp > 0.0)) break;
    alpha[it] = rz / pAp;
    beta[it] = b;
    for (int64_t i = 0; i < N; ++i) r[i] -= alpha[it] * Ap[i];
    rz_old = rz;
    m = it + 1;
  }
  double *dd = (double *)calloc(m + 1, sizeof(double)), *ee = (double *)calloc(m + 1, sizeof(double));
  for (int j = 0; j < m; ++j) {
    dd[j] = 1.0 / alpha[j] + (j > 0 ? beta[j] / alpha[j - 1] : 0.0);
    if (j + 1 < m) ee[j] = sqrt(beta[j + 1]) / alpha[j];
  }
  *lmin = m > 0 ? tridiag_eig(m, dd, ee, 0) : 1.0;
  *lmax = m > 0 ? tridiag_eig(m, dd, ee, m - 1) : 1.0;
  free(dd);
  free(ee);
  free(alpha);
  free(beta);
  free(r);
  free(z);
  free(p);
  free(Ap);
}

void orc_linear_predictor(const orc_heat *h, const double *T_cur, const double *T_oldv,
                          double *pred, double dt, double dt_old)
{
  const int64_t N = h->n_dofs;
  if (fabs(dt_old) < 1e-12) {
    memcpy(pred, T_cur, sizeof(double) * N);
    return;
  }
  const double f = dt / dt_old;
#pragma omp parallel for num_threads(nthreads())
  for (int64_t i = 0; i < N; ++i) pred[i] = (f + 1.0) * T_cur[i] - f * T_oldv[i];
}

int orc_time_step_newton(orc_heat *h, double *T_cur, double *T_old, const double *heat_source,
                         double dt, double dt_old, int predictor, int solver_type,
                         const orc_solver_params *lin, const orc_newton_params *nl,
                         orc_step_stats *stats)
{
  const int gmres_restart = 28;
  const int64_t N = h->n_dofs;
  h->dt = dt;
  double *pred = vec_new(N), *rhs = vec_new(N), *du = vec_new(N), *D = vec_new(N);
  /* init_time_advance: predictor, commit history, apply constraints */
  if (predictor == 1)
    orc_linear_predictor(h, T_cur, T_old, pred, dt, dt_old);
  else
    memcpy(pred, T_cur, sizeof(double) * N);
  memcpy(T_old, T_cur, sizeof(double) * N);
  memcpy(T_cur, pred, sizeof(double) * N);
  orc_distribute(h, T_cur);
  /* preconditioner update at the predicted state */
  orc_inverse_diagonal(h, D, T_cur, T_old, 0);
  stats->newton_iterations = 0;
  stats->linear_iterations = 0;
  stats->converged = 0;
  for (int i = 0; i < nl->max_iterations; ++i) {
    memset(rhs, 0, sizeof(double) * N);
    memset(du, 0, sizeof(double) * N);
    orc_create_rhs(h, rhs, T_cur, T_old, heat_source);
    int its = solver_type == 1 ? orc_gmres(h, lin, gmres_restart, du, rhs, D, T_cur, T_old, NULL)
                               : orc_cg(h, lin, du, rhs, D, T_cur, T_old, NULL);
    if (its < 0) break;
    stats->linear_iterations += its;
    const double rn = sqrt(dot(N, rhs, rhs)), un = sqrt(dot(N, du, du));
    if (rn < nl->residual_tolerance && un < nl->correction_tolerance) {
      stats->converged = 1;
      break;
    }
#pragma omp parallel for num_threads(nthreads())
    for (int64_t j = 0; j < N; ++j) T_cur[j] += du[j];
    orc_distribute(h, T_cur);
    stats->newton_iterations = i + 1;
  }
  free(pred);
  free(rhs);
  free(du);
  free(D);
  return stats->converged ? 0 : -1;
}
