// Grid metrics and Jacobian on the host: 6th-order derivatives of the
// coordinates (value_half_node_1d + flux_dxyz_1d), the cross-product metrics,
// the optional Visbal conservative (GCL) form, and the volume floor, as
// compute_grid_metrics / check_grid_metrics do (src/mesh/MetricComputer.cpp:21-500).
// Compiled without floating-point contraction so the results are bit-identical
// to the reference's.
#include <algorithm>
#include <cstddef>
#include <vector>

#include "orion_gpu.h"

namespace {

constexpr int NG = 3;

// Half-node values of a line of n points (q[v + nvar*i]) at n+1 half points.
void half_node(int nvar, int n, const double* q, double* h) {
  auto Q = [&](int v, int i) { return q[v + nvar * i]; };
  for (int i = 2; i < n - 1; ++i)
    for (int m = 0; m < nvar; ++m) h[m + nvar * i] = (9.0 * (Q(m, i - 1) + Q(m, i)) + -1.0 * (Q(m, i + 1) + Q(m, i - 2))) / 16.0;
  for (int m = 0; m < nvar; ++m) {
    h[m + nvar * 1] = (5.0 * Q(m, 0) + 15.0 * Q(m, 1) + -5.0 * Q(m, 2) + 1.0 * Q(m, 3)) / 16.0;
    h[m + nvar * (n - 1)] = (5.0 * Q(m, n - 1) + 15.0 * Q(m, n - 2) + -5.0 * Q(m, n - 3) + 1.0 * Q(m, n - 4)) / 16.0;
    h[m + nvar * 0] = (35.0 * Q(m, 0) - 35.0 * Q(m, 1) + 21.0 * Q(m, 2) - 5.0 * Q(m, 3)) / 16.0;
    h[m + nvar * n] = (35.0 * Q(m, n - 1) - 35.0 * Q(m, n - 2) + 21.0 * Q(m, n - 3) - 5.0 * Q(m, n - 4)) / 16.0;
  }
}

// Node derivatives from half-node values (6th order inside, 4th/3rd at the ends).
void half_diff(int nvar, int n, const double* f, double* df) {
  auto F = [&](int v, int i) { return f[v + nvar * i]; };
  for (int i = 2; i <= n - 3; ++i)
    for (int m = 0; m < nvar; ++m) {
      const double t1 = F(m, i + 1) - F(m, i);
      const double t2 = F(m, i + 2) - F(m, i - 1);
      const double t3 = F(m, i + 3) - F(m, i - 2);
      df[m + nvar * i] = (2250.0 * t1 - 125.0 * t2 + 9.0 * t3) / 1920.0;
    }
  for (int m = 0; m < nvar; ++m) {
    df[m + nvar * 0] = (-23.0 * F(m, 0) + 21.0 * F(m, 1) + 3.0 * F(m, 2) - F(m, 3)) / 24.0;
    df[m + nvar * 1] = (F(m, 0) - 27.0 * F(m, 1) + 27.0 * F(m, 2) - F(m, 3)) / 24.0;
    df[m + nvar * (n - 2)] = -(F(m, n) - 27.0 * F(m, n - 1) + 27.0 * F(m, n - 2) - F(m, n - 3)) / 24.0;
    df[m + nvar * (n - 1)] = -(-23.0 * F(m, n) + 21.0 * F(m, n - 1) + 3.0 * F(m, n - 2) - F(m, n - 3)) / 24.0;
  }
}

}  // namespace

extern "C" int orion_grid_metrics_host(int ni, int nj, int nk, const double* x, const double* y, const double* z,
                                       int gcl, double* metrics, double* vol) {
  if (ni <= 2 * NG || nj <= 2 * NG || nk <= 2 * NG || !x || !y || !z || !metrics || !vol) return ORION_E_INVALID;
  const int px = ni + 2 * NG, py = nj + 2 * NG, pz = nk + 2 * NG;
  const size_t np = (size_t)px * py * pz;
  std::fill(metrics, metrics + 9 * np, 0.0);
  std::fill(vol, vol + np, 0.0);
  const size_t n = (size_t)ni * nj * nk;
  auto G = [&](int i, int j, int k) { return (size_t)i + (size_t)ni * ((size_t)j + (size_t)nj * k); };
  auto P = [&](int i, int j, int k) { return (size_t)(i + NG) + (size_t)px * ((size_t)(j + NG) + (size_t)py * (k + NG)); };
  std::vector<double> dxyz(18 * n, 0.0);
  auto D = [&](int c, int i, int j, int k) -> double& { return dxyz[c + 18 * G(i, j, k)]; };
  const int nmax = std::max({ni, nj, nk});
  std::vector<double> lin(6 * nmax), half(6 * (nmax + 1)), out(6 * nmax);

  // generic line pass: gather nvar values along direction d, differentiate, scatter
  auto pass = [&](int d, int nvar, auto gather, auto scatter) {
    const int nl = d == 0 ? ni : (d == 1 ? nj : nk);
    const int na = d == 0 ? nj : ni;
    const int nb = d == 2 ? nj : nk;
    for (int b = 0; b < nb; ++b)
      for (int a = 0; a < na; ++a) {
        for (int t = 0; t < nl; ++t) {
          int i, j, k;
          if (d == 0) { i = t; j = a; k = b; }
          else if (d == 1) { i = a; j = t; k = b; }
          else { i = a; j = b; k = t; }
          gather(i, j, k, &lin[(size_t)nvar * t]);
        }
        half_node(nvar, nl, lin.data(), half.data());
        half_diff(nvar, nl, half.data(), out.data());
        for (int t = 0; t < nl; ++t) {
          int i, j, k;
          if (d == 0) { i = t; j = a; k = b; }
          else if (d == 1) { i = a; j = t; k = b; }
          else { i = a; j = b; k = t; }
          scatter(i, j, k, &out[(size_t)nvar * t]);
        }
      }
  };

  // pass 1: coordinate derivatives (x_xi -> 0, y_xi -> 3, z_xi -> 6; eta +1; zeta +2)
  for (int d = 0; d < 3; ++d)
    pass(d, 3,
         [&](int i, int j, int k, double* v) {
           const size_t g = G(i, j, k);
           v[0] = x[g];
           v[1] = y[g];
           v[2] = z[g];
         },
         [&](int i, int j, int k, const double* v) {
           D(0 + d, i, j, k) = v[0];
           D(3 + d, i, j, k) = v[1];
           D(6 + d, i, j, k) = v[2];
         });

  auto M = [&](int c, int i, int j, int k) -> double& { return metrics[c * np + P(i, j, k)]; };
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i) {
        const double x_xi = D(0, i, j, k), x_et = D(1, i, j, k), x_zt = D(2, i, j, k);
        const double y_xi = D(3, i, j, k), y_et = D(4, i, j, k), y_zt = D(5, i, j, k);
        const double z_xi = D(6, i, j, k), z_et = D(7, i, j, k), z_zt = D(8, i, j, k);
        const double kcx = y_et * z_zt - z_et * y_zt;
        const double kcy = z_et * x_zt - x_et * z_zt;
        const double kcz = x_et * y_zt - y_et * x_zt;
        const double etx = y_zt * z_xi - z_zt * y_xi;
        const double ety = z_zt * x_xi - x_zt * z_xi;
        const double etz = x_zt * y_xi - y_zt * x_xi;
        const double ctx = y_xi * z_et - z_xi * y_et;
        const double cty = z_xi * x_et - x_xi * z_et;
        const double ctz = x_xi * y_et - y_xi * x_et;
        M(0, i, j, k) = kcx; M(1, i, j, k) = kcy; M(2, i, j, k) = kcz;
        M(3, i, j, k) = etx; M(4, i, j, k) = ety; M(5, i, j, k) = etz;
        M(6, i, j, k) = ctx; M(7, i, j, k) = cty; M(8, i, j, k) = ctz;
        vol[P(i, j, k)] = x_xi * kcx + x_et * etx + x_zt * ctx;
      }

  if (gcl == 1) {
    // Visbal conservative form
    std::vector<double> xkc(3 * n);
    for (int k = 0; k < nk; ++k)
      for (int j = 0; j < nj; ++j)
        for (int i = 0; i < ni; ++i) {
          const size_t g = G(i, j, k);
          const double xm = x[g], ym = y[g], zm = z[g];
          xkc[3 * g + 0] = D(0, i, j, k);
          xkc[3 * g + 1] = D(1, i, j, k);
          xkc[3 * g + 2] = D(2, i, j, k);
          M(0, i, j, k) = D(0, i, j, k) * ym;
          M(1, i, j, k) = D(1, i, j, k) * ym;
          M(2, i, j, k) = D(2, i, j, k) * ym;
          M(3, i, j, k) = D(3, i, j, k) * zm;
          M(4, i, j, k) = D(4, i, j, k) * zm;
          M(5, i, j, k) = D(5, i, j, k) * zm;
          M(6, i, j, k) = D(6, i, j, k) * xm;
          M(7, i, j, k) = D(7, i, j, k) * xm;
          M(8, i, j, k) = D(8, i, j, k) * xm;
        }
    const int src[3][6] = {{7, 8, 1, 2, 4, 5}, {6, 8, 0, 2, 3, 5}, {6, 7, 0, 1, 3, 4}};
    for (int d = 0; d < 3; ++d)
      pass(d, 6,
           [&](int i, int j, int k, double* v) {
             for (int m = 0; m < 6; ++m) v[m] = M(src[d][m], i, j, k);
           },
           [&](int i, int j, int k, const double* v) {
             for (int m = 0; m < 6; ++m) D(m + 6 * d, i, j, k) = v[m];
           });
    for (int k = 0; k < nk; ++k)
      for (int j = 0; j < nj; ++j)
        for (int i = 0; i < ni; ++i) {
          const double kcx = D(17, i, j, k) - D(11, i, j, k);
          const double kcy = D(13, i, j, k) - D(7, i, j, k);
          const double kcz = D(15, i, j, k) - D(9, i, j, k);
          const double etx = D(5, i, j, k) - D(16, i, j, k);
          const double ety = D(1, i, j, k) - D(12, i, j, k);
          const double etz = D(3, i, j, k) - D(14, i, j, k);
          const double ctx = D(10, i, j, k) - D(4, i, j, k);
          const double cty = D(6, i, j, k) - D(0, i, j, k);
          const double ctz = D(8, i, j, k) - D(2, i, j, k);
          M(0, i, j, k) = kcx; M(1, i, j, k) = kcy; M(2, i, j, k) = kcz;
          M(3, i, j, k) = etx; M(4, i, j, k) = ety; M(5, i, j, k) = etz;
          M(6, i, j, k) = ctx; M(7, i, j, k) = cty; M(8, i, j, k) = ctz;
          const size_t g = G(i, j, k);
          vol[P(i, j, k)] = xkc[3 * g + 0] * kcx + xkc[3 * g + 1] * etx + xkc[3 * g + 2] * ctx;
        }
  }
  // check_grid_metrics: floor non-positive Jacobians (MetricComputer.cpp:435-471)
  for (int k = 0; k < nk; ++k)
    for (int j = 0; j < nj; ++j)
      for (int i = 0; i < ni; ++i)
        if (vol[P(i, j, k)] < 1.0e-15) vol[P(i, j, k)] = 1.0e-15;
  return 0;
}
