// Point- and face-level numerics of ORION's per-step path, as device functions.
//
// Every function reproduces the reference's arithmetic operation by operation
// (same operands, same association, no contraction: the FP64 translation unit is
// compiled with --fmad=false), so the plain FP64 path is bit-identical to the
// reference wherever the reference uses only + - * / sqrt.  Templated on the
// compute type T so the mixed-precision path runs the same formulas in FP32.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace orion {

template <typename T> __device__ __forceinline__ T tabs(T x) { return x < T(0) ? -x : x; }
template <> __device__ __forceinline__ double tabs<double>(double x) { return fabs(x); }
template <> __device__ __forceinline__ float tabs<float>(float x) { return fabsf(x); }
template <typename T> __device__ __forceinline__ T tsqrt(T x);
template <> __device__ __forceinline__ double tsqrt<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float tsqrt<float>(float x) { return sqrtf(x); }
template <typename T> __device__ __forceinline__ T tmax(T a, T b) { return (a < b) ? b : a; }  // std::max

// ---------------------------------------------------------------------------
// Roe flux with Harten entropy fix: flux_Roe + calc_physical_flux
// (src/solver/InviscidFluxComputer.cpp:14-131).  q = (rho,u,v,w,p).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void physical_flux(const T q[5], T gamma, T nx, T ny, T nz, T nt, T f[5]) {
  const T rho = q[0], u = q[1], v = q[2], w = q[3], p = q[4];
  const T V = u * nx + v * ny + w * nz + nt;
  const T E = p / (gamma - T(1)) + T(0.5) * rho * (u * u + v * v + w * w);
  const T H = (E + p) / rho;
  f[0] = rho * V;
  f[1] = rho * u * V + p * nx;
  f[2] = rho * v * V + p * ny;
  f[3] = rho * w * V + p * nz;
  f[4] = rho * H * V + p * nt;
}

template <typename T>
__device__ __forceinline__ void roe_flux(const T ql[5], const T qr[5], T nx, T ny, T nz, T nt, T efix, T gamma,
                                         T f[5]) {
  T fl[5], fr[5];
  physical_flux(ql, gamma, nx, ny, nz, nt, fl);
  physical_flux(qr, gamma, nx, ny, nz, nt, fr);
  const T drho = qr[0] - ql[0], du = qr[1] - ql[1], dv = qr[2] - ql[2], dw = qr[3] - ql[3], dp = qr[4] - ql[4];
  const T gamma1 = gamma - T(1);
  const T gamma2 = gamma / gamma1;
  const T hl = gamma2 * ql[4] / ql[0] + T(0.5) * (ql[1] * ql[1] + ql[2] * ql[2] + ql[3] * ql[3]);
  const T hr = gamma2 * qr[4] / qr[0] + T(0.5) * (qr[1] * qr[1] + qr[2] * qr[2] + qr[3] * qr[3]);
  const T sqrt_rL = tsqrt(ql[0]);
  const T sqrt_rR = tsqrt(qr[0]);
  const T inv_den = T(1) / (sqrt_rL + sqrt_rR);
  const T rho_roe = sqrt_rL * sqrt_rR;
  const T u_roe = (sqrt_rL * ql[1] + sqrt_rR * qr[1]) * inv_den;
  const T v_roe = (sqrt_rL * ql[2] + sqrt_rR * qr[2]) * inv_den;
  const T w_roe = (sqrt_rL * ql[3] + sqrt_rR * qr[3]) * inv_den;
  const T h_roe = (sqrt_rL * hl + sqrt_rR * hr) * inv_den;
  const T v2 = u_roe * u_roe + v_roe * v_roe + w_roe * w_roe;
  T c2 = (h_roe - T(0.5) * v2) * gamma1;
  if (c2 <= T(0)) c2 = T(1.0e-6);
  const T c = tsqrt(c2);
  const T U_contra = u_roe * nx + v_roe * ny + w_roe * nz + nt;
  T grad_mag = tsqrt(nx * nx + ny * ny + nz * nz);
  grad_mag = tmax(grad_mag, T(1.0e-30));
  const T inv_mag = T(1) / grad_mag;
  const T nx_n = nx * inv_mag, ny_n = ny * inv_mag, nz_n = nz * inv_mag;
  const T c_mag = c * grad_mag;
  T l1 = tabs(U_contra - c_mag);
  T l4 = tabs(U_contra);
  T l5 = tabs(U_contra + c_mag);
  const T delta = efix * c_mag;
  const T delta2 = delta * delta;
  if (l1 < delta) l1 = tsqrt(l1 * l1 + delta2);
  if (l4 < delta) l4 = tsqrt(l4 * l4 + delta2);
  if (l5 < delta) l5 = tsqrt(l5 * l5 + delta2);
  const T rodcta = rho_roe * (du * nx_n + dv * ny_n + dw * nz_n);
  const T dp_c2 = dp / c2;
  const T rodctac = rodcta / c;
  const T a1 = l4 * (drho - dp_c2);
  const T a2 = l5 * (dp_c2 + rodctac) * T(0.5);
  const T a3 = l1 * (dp_c2 - rodctac) * T(0.5);
  const T a4 = a1 + a2 + a3;
  const T a5 = c * (a2 - a3);
  const T a6 = l4 * (rho_roe * du - nx_n * rodcta);
  const T a7 = l4 * (rho_roe * dv - ny_n * rodcta);
  const T a8 = l4 * (rho_roe * dw - nz_n * rodcta);
  const T df0 = a4;
  const T df1 = u_roe * a4 + nx_n * a5 + a6;
  const T df2 = v_roe * a4 + ny_n * a5 + a7;
  const T df3 = w_roe * a4 + nz_n * a5 + a8;
  const T df4 = h_roe * a4 + U_contra * inv_mag * a5 + u_roe * a6 + v_roe * a7 + w_roe * a8 - c2 * a1 / gamma1;
  f[0] = T(0.5) * (fl[0] + fr[0] - df0);
  f[1] = T(0.5) * (fl[1] + fr[1] - df1);
  f[2] = T(0.5) * (fl[2] + fr[2] - df2);
  f[3] = T(0.5) * (fl[3] + fr[3] - df3);
  f[4] = T(0.5) * (fl[4] + fr[4] - df4);
}

// ---------------------------------------------------------------------------
// WCNS-E-5 left/right states at one face for one variable
// (src/solver/InviscidFluxComputer.cpp:259-315).  s[0..5] are the six line
// points q_line[i..i+5] around face i.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T wcns_w(T g, T s, T C) {
  const T EPS = T(1.0e-6);
  const T IS = g * g + s * s;
  return C / ((EPS + IS) * (EPS + IS));
}

template <typename T>
__device__ __forceinline__ T wcns_left(T q_m2, T q_m1, T q_0, T q_p1, T q_p2) {
  const T CL1 = T(1.0 / 16.0), CL2 = T(10.0 / 16.0), CL3 = T(5.0 / 16.0);
  const T s1 = q_m2 - T(2) * q_m1 + q_0;
  const T s2 = q_m1 - T(2) * q_0 + q_p1;
  const T s3 = q_0 - T(2) * q_p1 + q_p2;
  const T g1 = T(0.5) * (q_m2 - T(4) * q_m1 + T(3) * q_0);
  const T g2 = T(0.5) * (q_p1 - q_m1);
  const T g3 = T(0.5) * (T(-3) * q_0 + T(4) * q_p1 - q_p2);
  const T wl1 = wcns_w(g1, s1, CL1);
  const T wl2 = wcns_w(g2, s2, CL2);
  const T wl3 = wcns_w(g3, s3, CL3);
  const T sum = wl1 + wl2 + wl3;
  return q_0 + T(0.125) * ((wl1 / sum) * (s1 + T(4) * g1) + (wl2 / sum) * (s2 + T(4) * g2) +
                           (wl3 / sum) * (s3 + T(4) * g3));
}

template <typename T>
__device__ __forceinline__ T wcns_right(T q_m1, T q_0, T q_p1, T q_p2, T q_p3) {
  // sr1 = s2, sr2 = s3 of the left stencil; the right state is centred on q_p1.
  const T CL1 = T(1.0 / 16.0), CL2 = T(10.0 / 16.0), CL3 = T(5.0 / 16.0);
  const T sr1 = q_m1 - T(2) * q_0 + q_p1;
  const T sr2 = q_0 - T(2) * q_p1 + q_p2;
  const T sr3 = q_p1 - T(2) * q_p2 + q_p3;
  const T gr1 = T(0.5) * (q_m1 - T(4) * q_0 + T(3) * q_p1);
  const T gr2 = T(0.5) * (q_p2 - q_0);
  const T gr3 = T(0.5) * (T(-3) * q_p1 + T(4) * q_p2 - q_p3);
  const T wr1 = wcns_w(gr1, sr1, CL3);
  const T wr2 = wcns_w(gr2, sr2, CL2);
  const T wr3 = wcns_w(gr3, sr3, CL1);
  const T sum = wr1 + wr2 + wr3;
  return q_p1 + T(0.125) * ((wr1 / sum) * (sr1 - T(4) * gr1) + (wr2 / sum) * (sr2 - T(4) * gr2) +
                            (wr3 / sum) * (sr3 - T(4) * gr3));
}

// 6th-order / boundary flux differences (FLUX_DXYZ,
// src/solver/InviscidFluxComputer.cpp:197-233 and src/solver/FluxComputer.cpp:257-296,
// identical formulas).  f points at face values with stride `st`; point t in [0,ni).
// F(k) is face k's flux (faces 0..ni).
template <typename T, typename F>
__device__ __forceinline__ T flux_diff_at(F f, int t, int ni) {
  if (t >= 2 && t < ni - 2) {
    const T term1 = T(2250) * (f(t + 1) - f(t));
    const T term2 = T(-125) * (f(t + 2) - f(t - 1));
    const T term3 = T(9) * (f(t + 3) - f(t - 2));
    return (term1 + term2 + term3) / T(1920);
  }
  if (t == 0) return (T(-23) * f(0) + T(21) * f(1) + T(3) * f(2) - f(3)) / T(24);
  if (t == 1) return (f(0) - T(27) * f(1) + T(27) * f(2) - f(3)) / T(24);
  if (t == ni - 1) return -(T(-23) * f(ni) + T(21) * f(ni - 1) + T(3) * f(ni - 2) - f(ni - 3)) / T(24);
  // t == ni - 2
  return -(f(ni) - T(27) * f(ni - 1) + T(27) * f(ni - 2) - f(ni - 3)) / T(24);
}

template <typename T>
__device__ __forceinline__ T flux_diff(const T* f, int st, int t, int ni) {
  return flux_diff_at<T>([&](int k) -> T { return f[k * st]; }, t, ni);
}

// ---------------------------------------------------------------------------
// Spectral radii and flux splitting of the implicit sweeps
// (src/solver/StateUpdater.cpp:175-265).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T spectral_radius(T rho, T u, T v, T w, T p, T gamma, T kx, T ky, T kz) {
  if (rho < T(1e-30)) rho = T(1e-30);
  if (p < T(1e-30)) p = T(1e-30);
  const T c2 = gamma * p / rho;
  const T c = tsqrt(c2);
  const T U = u * kx + v * ky + w * kz + T(0);
  const T grad_mag = tsqrt(kx * kx + ky * ky + kz * kz);
  return tabs(U) + c * grad_mag;
}

template <typename T>
__device__ __forceinline__ T visc_spectral_radius(T rho, T mu, T vol, T reynolds, T kx, T ky, T kz) {
  if (rho < T(1e-30)) rho = T(1e-30);
  const T grad2 = kx * kx + ky * ky + kz * kz;
  const T rm_vol = rho * vol;
  const T coef = T(2) * mu / (tabs(reynolds) * rm_vol + T(1.0e-30));
  return coef * grad2;
}

// compute_flux_splitting with nt = 0; sign is +1 or -1.
template <typename T>
__device__ __forceinline__ void flux_split(const T prim[5], const T dq[5], T nx, T ny, T nz, T r, T sign,
                                           T gamma, T out[5]) {
  T rm = prim[0];
  const T um = prim[1], vm = prim[2], wm = prim[3];
  T pm = prim[4];
  const T drm = dq[0], dum = dq[1], dvm = dq[2], dwm = dq[3], dEm = dq[4];
  const T nt = T(0);
  const T v2 = um * um + vm * vm + wm * wm;
  if (rm < T(1e-30)) rm = T(1e-30);
  if (pm < T(1e-30)) pm = T(1e-30);
  const T c2 = gamma * pm / rm;
  const T cm = tsqrt(c2);
  const T H = (gamma / (gamma - T(1))) * (pm / rm) + T(0.5) * v2;
  const T ct = nx * um + ny * vm + nz * wm + nt;
  T grad_mag = tsqrt(nx * nx + ny * ny + nz * nz);
  if (grad_mag < T(1.0e-30)) grad_mag = T(1.0e-30);
  T l1 = ct;
  T l4 = ct + cm * grad_mag;
  T l5 = ct - cm * grad_mag;
  l1 = T(0.5) * (l1 + sign * r);
  l4 = T(0.5) * (l4 + sign * r);
  l5 = T(0.5) * (l5 + sign * r);
  const T x1 = (T(2) * l1 - l4 - l5) / (T(2) * c2);
  const T x2 = (l4 - l5) / (T(2) * cm);
  const T inv_mag = T(1) / grad_mag;
  const T nx_n = nx * inv_mag, ny_n = ny * inv_mag, nz_n = nz * inv_mag;
  const T ct_n = (ct - nt) * inv_mag;
  const T gm1 = gamma - T(1);
  const T af = T(0.5) * gm1 * v2;
  const T dc = ct_n * drm - (nx_n * dum + ny_n * dvm + nz_n * dwm);
  const T dh = af * drm - gm1 * (um * dum + vm * dvm + wm * dwm - dEm);
  const T c2dc = c2 * dc;
  out[0] = l1 * drm - dh * x1 - dc * x2;
  out[1] = l1 * dum + (nx_n * c2dc - um * dh) * x1 + (nx_n * dh - um * dc) * x2;
  out[2] = l1 * dvm + (ny_n * c2dc - vm * dh) * x1 + (ny_n * dh - vm * dc) * x2;
  out[3] = l1 * dwm + (nz_n * c2dc - wm * dh) * x1 + (nz_n * dh - wm * dc) * x2;
  out[4] = l1 * dEm + (ct_n * c2dc - H * dh) * x1 + (ct_n * dh - H * dc) * x2;
}

}  // namespace orion
