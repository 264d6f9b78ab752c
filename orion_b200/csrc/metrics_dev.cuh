// Grid metrics and Jacobian on the device (compute_grid_metrics and
// check_grid_metrics, src/mesh/MetricComputer.cpp:21-500): the same formulas
// and operation order as the host restatement (metrics_host.cpp), evaluated
// per point from a stencil of coordinates instead of line passes, so the FP64
// results are bit-identical (this header is compiled only in the strict FP64
// translation unit, --fmad=false).
#pragma once
#include <cuda_runtime.h>

namespace orion {
namespace gm {

constexpr int NGM = 3;

// Value of a line of n points at position t, component stride cs.
struct LineRef {
  const double* q;  // point 0 of the line
  long long st;     // stride between consecutive points
  __device__ __forceinline__ double operator()(int t) const { return q[(long long)t * st]; }
};

// Half-node value h[i], 0 <= i <= n (value_half_node_1d: 4th order inside,
// one-sided at both ends).
template <class Q>
__device__ __forceinline__ double half_val(const Q& Qv, int n, int i) {
  if (i >= 2 && i <= n - 2) return (9.0 * (Qv(i - 1) + Qv(i)) + -1.0 * (Qv(i + 1) + Qv(i - 2))) / 16.0;
  if (i == 1) return (5.0 * Qv(0) + 15.0 * Qv(1) + -5.0 * Qv(2) + 1.0 * Qv(3)) / 16.0;
  if (i == n - 1) return (5.0 * Qv(n - 1) + 15.0 * Qv(n - 2) + -5.0 * Qv(n - 3) + 1.0 * Qv(n - 4)) / 16.0;
  if (i == 0) return (35.0 * Qv(0) - 35.0 * Qv(1) + 21.0 * Qv(2) - 5.0 * Qv(3)) / 16.0;
  return (35.0 * Qv(n - 1) - 35.0 * Qv(n - 2) + 21.0 * Qv(n - 3) - 5.0 * Qv(n - 4)) / 16.0;  // i == n
}

// Node derivative at t from half-node values (flux_dxyz_1d: 6th order inside,
// 4th/3rd order at the ends).
template <class Q>
__device__ __forceinline__ double node_diff(const Q& Qv, int n, int t) {
  auto F = [&](int i) { return half_val(Qv, n, i); };
  if (t >= 2 && t <= n - 3) {
    const double t1 = F(t + 1) - F(t);
    const double t2 = F(t + 2) - F(t - 1);
    const double t3 = F(t + 3) - F(t - 2);
    return (2250.0 * t1 - 125.0 * t2 + 9.0 * t3) / 1920.0;
  }
  if (t == 0) return (-23.0 * F(0) + 21.0 * F(1) + 3.0 * F(2) - F(3)) / 24.0;
  if (t == 1) return (F(0) - 27.0 * F(1) + 27.0 * F(2) - F(3)) / 24.0;
  if (t == n - 2) return -(F(n) - 27.0 * F(n - 1) + 27.0 * F(n - 2) - F(n - 3)) / 24.0;
  return -(-23.0 * F(n) + 21.0 * F(n - 1) + 3.0 * F(n - 2) - F(n - 3)) / 24.0;  // t == n - 1
}

struct GridDims {
  int ni, nj, nk;
  long long n;  // ni * nj * nk
  __device__ __forceinline__ long long g(int i, int j, int k) const {
    return i + (long long)ni * (j + (long long)nj * k);
  }
  __device__ __forceinline__ int len(int d) const { return d == 0 ? ni : (d == 1 ? nj : nk); }
  __device__ __forceinline__ long long stride(int d) const {
    return d == 0 ? 1 : (d == 1 ? (long long)ni : (long long)ni * nj);
  }
  __device__ __forceinline__ int pos(int d, int i, int j, int k) const { return d == 0 ? i : (d == 1 ? j : k); }
};

// Pass 1: the 9 coordinate derivatives of every point, D[c * n + g]:
// x_xi, x_eta, x_zeta, y_xi, ..., z_zeta (component 3 * coord + direction).
__global__ void k_coord_derivs(GridDims G, const double* __restrict__ xyz, double* __restrict__ D) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= G.n) return;
  const int i = (int)(p % G.ni), r = (int)(p / G.ni);
  const int j = r % G.nj, k = r / G.nj;
  for (int d = 0; d < 3; ++d) {
    const int t = G.pos(d, i, j, k);
    const long long st = G.stride(d);
    const long long base = p - (long long)t * st;
    for (int c = 0; c < 3; ++c) {
      const LineRef L{xyz + (long long)c * G.n + base, st};
      D[(long long)(3 * c + d) * G.n + p] = node_diff(L, G.len(d), t);
    }
  }
}

// Product field of the conservative form at point q: D[comp] * coordinate
// (y for components 0-2, z for 3-5, x for 6-8), as metrics_host.cpp forms it.
struct ProductRef {
  const double* D;    // derivative component, point 0 of the line
  const double* crd;  // coordinate, point 0 of the line
  long long st;
  __device__ __forceinline__ double operator()(int t) const {
    const long long o = (long long)t * st;
    return D[o] * crd[o];
  }
};

// Pass 2: metrics (padded, component stride np) and vol, cross-product form or
// (gcl == 1) the Visbal conservative form; then the Jacobian floor.
__global__ void k_metrics_final(GridDims G, int px, int py, long long np, int gcl, const double* __restrict__ xyz,
                                const double* __restrict__ D, double* __restrict__ met, double* __restrict__ vol) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= G.n) return;
  const int i = (int)(p % G.ni), r = (int)(p / G.ni);
  const int j = r % G.nj, k = r / G.nj;
  const long long P = (i + NGM) + (long long)px * ((j + NGM) + (long long)py * (k + NGM));
  auto d = [&](int c) { return D[(long long)c * G.n + p]; };
  const double x_xi = d(0), x_et = d(1), x_zt = d(2);
  double m[9], v;
  if (gcl != 1) {
    const double y_xi = d(3), y_et = d(4), y_zt = d(5);
    const double z_xi = d(6), z_et = d(7), z_zt = d(8);
    m[0] = y_et * z_zt - z_et * y_zt;
    m[1] = z_et * x_zt - x_et * z_zt;
    m[2] = x_et * y_zt - y_et * x_zt;
    m[3] = y_zt * z_xi - z_zt * y_xi;
    m[4] = z_zt * x_xi - x_zt * z_xi;
    m[5] = x_zt * y_xi - y_zt * x_xi;
    m[6] = y_xi * z_et - z_xi * y_et;
    m[7] = z_xi * x_et - x_xi * z_et;
    m[8] = x_xi * y_et - y_xi * x_et;
    v = x_xi * m[0] + x_et * m[3] + x_zt * m[6];
  } else {
    // E[m + 6 dir]: derivative along dir of product field src[dir][m]
    const int src[3][6] = {{7, 8, 1, 2, 4, 5}, {6, 8, 0, 2, 3, 5}, {6, 7, 0, 1, 3, 4}};
    double E[18];
    for (int dir = 0; dir < 3; ++dir) {
      const int t = G.pos(dir, i, j, k);
      const long long st = G.stride(dir);
      const long long base = p - (long long)t * st;
      for (int mm = 0; mm < 6; ++mm) {
        const int comp = src[dir][mm];
        const int coord = comp < 3 ? 1 : (comp < 6 ? 2 : 0);
        const ProductRef L{D + (long long)comp * G.n + base, xyz + (long long)coord * G.n + base, st};
        E[mm + 6 * dir] = node_diff(L, G.len(dir), t);
      }
    }
    m[0] = E[17] - E[11];
    m[1] = E[13] - E[7];
    m[2] = E[15] - E[9];
    m[3] = E[5] - E[16];
    m[4] = E[1] - E[12];
    m[5] = E[3] - E[14];
    m[6] = E[10] - E[4];
    m[7] = E[6] - E[0];
    m[8] = E[8] - E[2];
    v = x_xi * m[0] + x_et * m[3] + x_zt * m[6];
  }
  for (int c = 0; c < 9; ++c) met[(long long)c * np + P] = m[c];
  if (v < 1.0e-15) v = 1.0e-15;  // check_grid_metrics (MetricComputer.cpp:435-471)
  vol[P] = v;
}

}  // namespace gm
}  // namespace orion
