// 1D finite-element tables for FE_Q(p) on Gauss-Lobatto support points with
// QGauss(p+1) quadrature (source/utilities/fe_util.cpp:40-55,
// source/core/finite_element_data.cpp:62-65 in MeltPoolDG), plus the even-odd
// split of every 1D matrix the cell kernels contract with.
//
// Matrix kinds (rows = outputs, columns = inputs), n = p + 1:
//   S   interpolation GLL nodes -> Gauss points      S[q][i] = phi_i(x_q)
//   ST  its transpose (integration)
//   D   collocation derivative at the Gauss points   D[q][m] = l_m'(x_q)
//   DT  its transpose
//   PT  (S o S)^T, QT = (Sd o Sd)^T, RT = (S o Sd)^T, with Sd = D S: the
//       element-wise products that give the closed-form diagonal
// All of them are centro-(anti)symmetric: A[n-1-o][n-1-l] = sym * A[o][l].
#pragma once

#include <cmath>
#include <vector>

#ifdef __CUDACC__
#define MPDG_HD __host__ __device__
#else
#define MPDG_HD
#endif

namespace mpdg {

constexpr int kMaxN = 7;
enum MatKind { kS = 0, kST = 1, kD = 2, kDT = 3, kPT = 4, kQT = 5, kRT = 6, kNumKinds = 7 };

MPDG_HD constexpr int kind_sym(int kind) { return (kind == kD || kind == kDT || kind == kRT) ? -1 : 1; }

// Per (n, kind) block: ae[n][h], ao[n][h], mid[n] with h = n/2.
MPDG_HD constexpr int tab_block(int n) { return 2 * n * (n / 2) + n; }
MPDG_HD constexpr int tab_offset_n(int n)
{
  int off = 0;
  for (int m = 2; m < n; ++m) off += kNumKinds * tab_block(m);
  return off;
}
MPDG_HD constexpr int tab_off(int n, int kind) { return tab_offset_n(n) + kind * tab_block(n); }
constexpr int kTabSize = tab_offset_n(kMaxN + 1);
// 1D quadrature weights and GLL points, per n
MPDG_HD constexpr int w_off(int n)
{
  int off = 0;
  for (int m = 2; m < n; ++m) off += m;
  return off;
}
constexpr int kWSize = w_off(kMaxN + 1);

struct Tables1D {
  int n = 0;
  double xg[kMaxN], wg[kMaxN], xl[kMaxN];
  double A[kNumKinds][kMaxN][kMaxN];
};

inline void legendre(int N, double t, double &pN, double &pNm1)
{
  double p0 = 1.0, p1 = t;
  if (N == 0) {
    pN = 1.0;
    pNm1 = 0.0;
    return;
  }
  for (int k = 2; k <= N; ++k) {
    const double pk = ((2.0 * k - 1.0) * t * p1 - (k - 1.0) * p0) / k;
    p0 = p1;
    p1 = pk;
  }
  pN = p1;
  pNm1 = p0;
}

// Gauss-Legendre nodes/weights on [0,1], ascending.
inline void gauss_points(int n, double *x, double *w)
{
  for (int i = 0; i < n; ++i) {
    double t = std::cos(M_PI * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      double pn, pm;
      legendre(n, t, pn, pm);
      const double dp = n * (t * pn - pm) / (t * t - 1.0);
      const double step = pn / dp;
      t -= step;
      if (std::fabs(step) < 1e-16) break;
    }
    double pn, pm;
    legendre(n, t, pn, pm);
    const double dp = n * (t * pn - pm) / (t * t - 1.0);
    x[n - 1 - i] = 0.5 * (1.0 + t);
    w[n - 1 - i] = 1.0 / ((1.0 - t * t) * dp * dp);
  }
}

// Gauss-Lobatto nodes on [0,1]: 0, 1 and the roots of P'_{n-1}, ascending.
inline void lobatto_points(int n, double *x)
{
  const int N = n - 1;
  double t[kMaxN];
  for (int i = 0; i <= N; ++i) t[i] = std::cos(M_PI * i / N);
  for (int it = 0; it < 200; ++it) {
    double change = 0.0;
    for (int i = 0; i <= N; ++i) {
      double pn, pm;
      legendre(N, t[i], pn, pm);
      const double tn = t[i] - (t[i] * pn - pm) / ((N + 1) * pn);
      change = std::fmax(change, std::fabs(tn - t[i]));
      t[i] = tn;
    }
    if (change < 1e-16) break;
  }
  for (int i = 0; i <= N; ++i) x[N - i] = 0.5 * (1.0 + t[i]);
  x[0] = 0.0;
  x[N] = 1.0;
}

inline double lagrange(const double *z, int n, int i, double x)
{
  double v = 1.0;
  for (int j = 0; j < n; ++j)
    if (j != i) v *= (x - z[j]) / (z[i] - z[j]);
  return v;
}

inline double lagrange_d(const double *z, int n, int i, double x)
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

inline Tables1D make_tables(int n)
{
  Tables1D t;
  t.n = n;
  gauss_points(n, t.xg, t.wg);
  lobatto_points(n, t.xl);
  double S[kMaxN][kMaxN], D[kMaxN][kMaxN], Sd[kMaxN][kMaxN];
  for (int q = 0; q < n; ++q)
    for (int i = 0; i < n; ++i) {
      S[q][i] = lagrange(t.xl, n, i, t.xg[q]);
      D[q][i] = lagrange_d(t.xg, n, i, t.xg[q]);
    }
  for (int q = 0; q < n; ++q)
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      for (int m = 0; m < n; ++m) s += D[q][m] * S[m][i];
      Sd[q][i] = s;
    }
  for (int a = 0; a < n; ++a)
    for (int b = 0; b < n; ++b) {
      t.A[kS][a][b] = S[a][b];
      t.A[kST][a][b] = S[b][a];
      t.A[kD][a][b] = D[a][b];
      t.A[kDT][a][b] = D[b][a];
      t.A[kPT][a][b] = S[b][a] * S[b][a];
      t.A[kQT][a][b] = Sd[b][a] * Sd[b][a];
      t.A[kRT][a][b] = S[b][a] * Sd[b][a];
    }
  return t;
}

// Flattened even-odd tables for all n = 2..kMaxN (what the kernels read).
inline void fill_even_odd(std::vector<double> &tab, std::vector<double> &w,
                          std::vector<double> &xl)
{
  tab.assign(kTabSize, 0.0);
  w.assign(kWSize, 0.0);
  xl.assign(kWSize, 0.0);
  for (int n = 2; n <= kMaxN; ++n) {
    const Tables1D t = make_tables(n);
    const int h = n / 2;
    for (int kind = 0; kind < kNumKinds; ++kind) {
      double *blk = tab.data() + tab_off(n, kind);
      for (int o = 0; o < n; ++o) {
        for (int l = 0; l < h; ++l) {
          blk[o * h + l] = 0.5 * (t.A[kind][o][l] + t.A[kind][o][n - 1 - l]);
          blk[n * h + o * h + l] = 0.5 * (t.A[kind][o][l] - t.A[kind][o][n - 1 - l]);
        }
        blk[2 * n * h + o] = (n & 1) ? t.A[kind][o][h] : 0.0;
      }
    }
    for (int i = 0; i < n; ++i) {
      w[w_off(n) + i] = t.wg[i];
      xl[w_off(n) + i] = t.xl[i];
    }
  }
}

}  // namespace mpdg
