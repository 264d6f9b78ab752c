// Kernels of the per-step path.  Each kernel cites the reference routine whose
// arithmetic it reproduces.  Templates: S = storage type of the lowered fields
// (double for the plain form, float for the mixed form), T = compute type of
// the flux / viscous / sweep arithmetic.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_types.cuh"
#include "numerics.cuh"

namespace orion {

// Arrays the flux kernels read: FP32 shadows on the mixed path (exactly the
// values its FP32 arithmetic converts the FP64 arrays to), the FP64 arrays on
// the plain path.
template <typename S> struct FluxSrc;
template <> struct FluxSrc<double> {
  static __device__ __forceinline__ const double* prim(const BlockDev<double>& B) { return B.prim; }
  static __device__ __forceinline__ const double* metrics(const BlockDev<double>& B) { return B.metrics; }
  static __device__ __forceinline__ const double* vol(const BlockDev<double>& B) { return B.vol; }
};
template <> struct FluxSrc<float> {
  static __device__ __forceinline__ const float* prim(const BlockDev<float>& B) { return B.prim_f; }
  static __device__ __forceinline__ const float* metrics(const BlockDev<float>& B) { return B.met_f; }
  static __device__ __forceinline__ const float* vol(const BlockDev<float>& B) { return B.vol_f; }
};


template <typename S>
__device__ __forceinline__ long long lin(const BlockDev<S>& B, int i, int j, int k) {
  return (long long)i + (long long)B.nx * ((long long)j + (long long)B.ny * (long long)k);
}

template <typename S>
__device__ __forceinline__ int dim_along(const BlockDev<S>& B, int d) {
  return d == 0 ? B.ni : (d == 1 ? B.nj : B.nk);
}

template <typename S>
__device__ __forceinline__ long long stride_along(const BlockDev<S>& B, int d) {
  return d == 0 ? 1LL : (d == 1 ? (long long)B.nx : (long long)B.nx * B.ny);
}

// Memory index of along-line coordinate 0 of line `l` in direction d.  Lines
// enumerate the transverse interior coordinates, the lower one fastest.
template <typename S>
__device__ __forceinline__ long long line_origin(const BlockDev<S>& B, int d, int l) {
  if (d == 0) {
    const int jj = l % B.nj, kk = l / B.nj;
    return lin(B, 0, NG + jj, NG + kk);
  } else if (d == 1) {
    const int ii = l % B.ni, kk = l / B.ni;
    return lin(B, NG + ii, 0, NG + kk);
  }
  const int ii = l % B.ni, jj = l / B.ni;
  return lin(B, NG + ii, NG + jj, 0);
}

// ===========================================================================
// Halo copy of prim[0..4] into interface ghosts (HaloExchanger::exchange_bc,
// src/solver/HaloExchanger.cpp:70-179).  The host flattened the pack/unpack
// order into (src, dst) element offsets, last writer kept.
// ===========================================================================
static __global__ void k_halo_copy(double* __restrict__ arena, const long long* __restrict__ src,
                            const long long* __restrict__ dst, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) arena[dst[t]] = arena[src[t]];
}

// The same copy for a group of cases: blockIdx.y is the member, which copies
// through its own list into its own arena (nothing is concatenated).
static __global__ void k_halo_copy_group(const GroupMember* __restrict__ members) {
  const GroupMember& M = members[blockIdx.y];
  double* const arena = M.arena;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < M.n_halo; t += gridDim.x * blockDim.x)
    arena[M.halo_dst[t]] = arena[M.halo_src[t]];
}

// ===========================================================================
// Physical BCs (src/bc/PhysicalBC.cpp:12-613).  One launch per phase; phase p
// holds the p-th physical region of every block (regions of one block are
// sequential in file order; columns of one region are independent).
// ===========================================================================
template <typename S>
__device__ __forceinline__ void bc_normal(const BlockDev<S>& B, long long idx, int s_nd, double& nx, double& ny,
                                          double& nz) {
  // get_normal (PhysicalBC.cpp:12-44)
  const int off = (s_nd - 1) * 3;
  const double mx = B.metrics[(off + 0) * B.npad + idx];
  const double my = B.metrics[(off + 1) * B.npad + idx];
  const double mz = B.metrics[(off + 2) * B.npad + idx];
  double len = sqrt(mx * mx + my * my + mz * mz);
  if (len < 1.0e-30) len = 1.0e-30;
  nx = mx / len;
  ny = my / len;
  nz = mz / len;
}

template <typename S>
__device__ __forceinline__ void dif_average(const BlockDev<S>& B, long long idx0, long long step_out) {
  // apply_dif_average (PhysicalBC.cpp:71-92): face point = mean of ghost 1 and inner 1.
  const long long ig = idx0 + step_out, ii = idx0 - step_out;
  for (int m = 0; m < 6; ++m) {
    const double vg = B.prim[m * B.npad + ig];
    const double vi = B.prim[m * B.npad + ii];
    B.prim[m * B.npad + idx0] = 0.5 * (vg + vi);
  }
}

template <typename S>
__global__ void k_bc_phase(const BlockDev<S>* __restrict__ blocks, const RegionDev* __restrict__ regions,
                           const int* __restrict__ phase_regions) {
  const RegionDev R = regions[phase_regions[blockIdx.y]];
  const int pt = blockIdx.x * blockDim.x + threadIdx.x;
  if (pt >= R.npts) return;
  const BlockDev<S> B = blocks[R.block];
  const ParamsDev& P = B.prm;
  const int wi = R.hi[0] - R.lo[0] + 1, wj = R.hi[1] - R.lo[1] + 1;
  const int i = R.lo[0] + pt % wi;
  const int j = R.lo[1] + (pt / wi) % wj;
  const int k = R.lo[2] + pt / (wi * wj);
  const long long idx0 = lin(B, i, j, k);
  const long long sd = (R.dir == 0) ? 1LL : (R.dir == 1 ? (long long)B.nx : (long long)B.nx * B.ny);
  const long long out = (R.lr == 1) ? sd : -sd;  // step from the face towards the ghosts
  const long long np = B.npad;
  double* prim = B.prim;
  auto PR = [&](int m, long long id) -> double& { return prim[m * np + id]; };

  switch (R.type) {
    case 2: {
      if (P.nvis == 1) {
        // apply_viscid_wall (PhysicalBC.cpp:254-363)
        const double gama = P.gamma, mach = P.moo;
        const double moocp = mach * mach * gama;
        const bool isothermal = (P.twall > 1.0e-6);
        const double twall_dim = (isothermal && fabs(P.tref) > 1e-16) ? P.twall / P.tref : P.twall;
        const long long i1 = idx0 - out, i2 = idx0 - 2 * out;
        const double p1 = PR(4, i1), p2 = PR(4, i2);
        double p_wall = (4.0 * p1 - p2) / 3.0;
        if (p_wall < 1.0e-6) p_wall = p1;
        double t_wall;
        if (isothermal) {
          t_wall = twall_dim;
        } else {
          const double t1 = PR(5, i1), t2 = PR(5, i2);
          t_wall = (4.0 * t1 - t2) / 3.0;
          if (t_wall < 1e-6) t_wall = t1;
        }
        const double rho_wall = moocp * p_wall / t_wall;
        for (int l = 0; l < NG; ++l) {
          const int dist = l + 1;
          const long long ig = idx0 + dist * out, ii = idx0 - dist * out;
          const double u_i = PR(1, ii), v_i = PR(2, ii), w_i = PR(3, ii);
          PR(1, ig) = -u_i;
          PR(2, ig) = -v_i;
          PR(3, ig) = -w_i;
          PR(4, ig) = PR(4, ii);
          if (isothermal) {
            const double t_inner = PR(5, ii);
            PR(5, ig) = 2.0 * t_wall - t_inner;
          } else {
            PR(5, ig) = PR(5, ii);
          }
          const double pg = PR(4, ig);
          double tg = PR(5, ig);
          if (tg < 1e-6) tg = 1.0;
          const double rho_calc = moocp * pg / tg;
          PR(0, ig) = (dist == 3) ? -rho_calc : rho_calc;
        }
        PR(0, idx0) = rho_wall;
        PR(1, idx0) = 0.0;
        PR(2, idx0) = 0.0;
        PR(3, idx0) = 0.0;
        PR(4, idx0) = p_wall;
        PR(5, idx0) = t_wall;
      } else {
        // apply_inviscid_wall (PhysicalBC.cpp:191-248)
        double nx, ny, nz;
        bc_normal(B, idx0, R.s_nd, nx, ny, nz);
        for (int l = 0; l < NG; ++l) {
          const int dist = l + 1;
          const long long ig = idx0 + dist * out, ii = idx0 - dist * out;
          const double rho_i = PR(0, ii), u_i = PR(1, ii), v_i = PR(2, ii), w_i = PR(3, ii), p_i = PR(4, ii);
          const double t_i = PR(5, ii);
          const double v_dot_n = u_i * nx + v_i * ny + w_i * nz;
          PR(0, ig) = (dist == 3) ? -rho_i : rho_i;
          PR(1, ig) = u_i - 2.0 * v_dot_n * nx;
          PR(2, ig) = v_i - 2.0 * v_dot_n * ny;
          PR(3, ig) = w_i - 2.0 * v_dot_n * nz;
          PR(4, ig) = p_i;
          PR(5, ig) = t_i;
        }
        if (P.method == 1) dif_average(B, idx0, out);
      }
      break;
    }
    case 3: {
      // apply_symmetry_bc (PhysicalBC.cpp:97-183)
      if (R.is2d) {
        for (int l = 0; l < NG; ++l) {
          const int dist = l + 1;
          const long long ig = idx0 + dist * out, ii = idx0 - dist * out;
          PR(0, ig) = PR(0, ii);
          PR(1, ig) = PR(1, ii);
          PR(2, ig) = PR(2, ii);
          PR(4, ig) = PR(4, ii);
          PR(5, ig) = PR(5, ii);
          PR(3, ig) = -PR(3, ii);
        }
      } else {
        const int im = (R.lo[0] + R.hi[0]) / 2, jm = (R.lo[1] + R.hi[1]) / 2, km = (R.lo[2] + R.hi[2]) / 2;
        double nx, ny, nz;
        bc_normal(B, lin(B, im, jm, km), R.s_nd, nx, ny, nz);
        for (int l = 0; l < NG; ++l) {
          const int dist = l + 1;
          const long long ig = idx0 + dist * out, ii = idx0 - dist * out;
          const double rho = PR(0, ii), u = PR(1, ii), v = PR(2, ii), w = PR(3, ii), p = PR(4, ii);
          const double v_dot_n = u * nx + v * ny + w * nz;
          PR(0, ig) = rho;
          PR(1, ig) = u - 2.0 * v_dot_n * nx;
          PR(2, ig) = v - 2.0 * v_dot_n * ny;
          PR(3, ig) = w - 2.0 * v_dot_n * nz;
          PR(4, ig) = p;
          PR(5, ig) = PR(5, ii);
        }
      }
      if (P.method == 1) dif_average(B, idx0, out);
      break;
    }
    case 4: {
      // apply_farfield_bc (PhysicalBC.cpp:369-472)
      const double gama = P.gamma, gm1 = gama - 1.0;
      const double rho_inf = P.roo, u_inf = P.uoo, v_inf = P.voo, w_inf = P.woo, p_inf = P.poo;
      const double c_inf = sqrt(gama * p_inf / rho_inf);
      double nx, ny, nz;
      bc_normal(B, idx0, R.s_nd, nx, ny, nz);
      if (R.lr == -1) {
        nx = -nx;
        ny = -ny;
        nz = -nz;
      }
      const long long ii = idx0 - out;
      const double rho_in = PR(0, ii), u_in = PR(1, ii), v_in = PR(2, ii), w_in = PR(3, ii), p_in = PR(4, ii);
      const double c_in = sqrt(gama * p_in / rho_in);
      const double s_in = p_in / pow(rho_in, gama);
      const double s_inf = p_inf / pow(rho_inf, gama);
      const double vn_in = u_in * nx + v_in * ny + w_in * nz;
      const double vn_inf = u_inf * nx + v_inf * ny + w_inf * nz;
      const double vel_mag = sqrt(u_in * u_in + v_in * v_in + w_in * w_in);
      const double mach = vel_mag / c_in;
      double rho_b, u_b, v_b, w_b, p_b;
      if (mach < 1.0) {
        const double R_plus = vn_in + 2.0 * c_in / gm1;
        const double R_minus = vn_inf - 2.0 * c_inf / gm1;
        const double vn_b = 0.5 * (R_plus + R_minus);
        const double c_b = 0.25 * gm1 * (R_plus - R_minus);
        double s_b, u_ref, v_ref, w_ref, vn_ref;
        if (vn_b > 0.0) {
          s_b = s_in; u_ref = u_in; v_ref = v_in; w_ref = w_in; vn_ref = vn_in;
        } else {
          s_b = s_inf; u_ref = u_inf; v_ref = v_inf; w_ref = w_inf; vn_ref = vn_inf;
        }
        rho_b = pow(c_b * c_b / (gama * s_b), 1.0 / gm1);
        p_b = s_b * pow(rho_b, gama);
        u_b = u_ref + (vn_b - vn_ref) * nx;
        v_b = v_ref + (vn_b - vn_ref) * ny;
        w_b = w_ref + (vn_b - vn_ref) * nz;
      } else {
        if (vn_in > 0.0) {
          rho_b = rho_in; u_b = u_in; v_b = v_in; w_b = w_in; p_b = p_in;
        } else {
          rho_b = rho_inf; u_b = u_inf; v_b = v_inf; w_b = w_inf; p_b = p_inf;
        }
      }
      const double t_b = (mach * mach * gama) * p_b / rho_b;
      for (int l = 0; l < NG; ++l) {
        const int dist = l + 1;
        const long long ig = idx0 + dist * out;
        PR(0, ig) = (dist == 3) ? -rho_b : rho_b;
        PR(1, ig) = u_b;
        PR(2, ig) = v_b;
        PR(3, ig) = w_b;
        PR(4, ig) = p_b;
        PR(5, ig) = t_b;
      }
      break;
    }
    case 5: {
      // apply_freestream_bc (PhysicalBC.cpp:477-521)
      for (int l = 0; l < NG; ++l) {
        const long long ig = idx0 + (l + 1) * out;
        PR(0, ig) = P.roo;
        PR(1, ig) = P.uoo;
        PR(2, ig) = P.voo;
        PR(3, ig) = P.woo;
        PR(4, ig) = P.poo;
        PR(5, ig) = P.too;
      }
      break;
    }
    case 6: {
      // apply_extrapolation_bc (PhysicalBC.cpp:526-571)
      const long long is = idx0 - out;
      double v[6];
      for (int m = 0; m < 6; ++m) v[m] = PR(m, is);
      for (int l = 0; l < NG; ++l) {
        const long long ig = idx0 + (l + 1) * out;
        for (int m = 0; m < 6; ++m) PR(m, ig) = v[m];
      }
      break;
    }
    default:
      break;
  }
}

// ===========================================================================
// Derived state + dq := 0 (+ local time step when DO_DT)
// update_flow_states (src/solver/StateUpdater.cpp:15-168) and
// calculate_spectrum / calculate_local_dt_cell (src/solver/TimeIntegrator.cpp:20-125),
// one pass over the padded points.  The spectral radii are consumed in place
// (they are read nowhere else).  phydtime = min(1000, min dt*vol) via atomicMin
// on the bit pattern of a positive double.
// ===========================================================================
template <typename S, bool DO_Q>
__device__ __forceinline__ void state_point(const BlockDev<S>& B, const ParamsDev& P, long long idx, int i, int j,
                                            int k, S& c_out, S& mu_out) {
  // arithmetic in the storage precision S of c, mu, dt (FP64 on the plain path)
  const long long np = B.npad;
  const bool inI = (i >= NG && i < NG + B.ni), inJ = (j >= NG && j < NG + B.nj), inK = (k >= NG && k < NG + B.nk);
  const int nin = (int)inI + (int)inJ + (int)inK;
  double* prim = B.prim;
  const S gamma = (S)P.gamma, moo = (S)P.moo, visc = (S)P.visc;
  S T = (S)prim[5 * np + idx];
  S cval = B.c[idx];
  if (nin >= 2) {
    // interior (nin == 3) or ghost face slab (nin == 2), update_thermodynamics_block
    S rho = (S)__ldg(prim + idx);
    const S p = (S)__ldg(prim + 4 * np + idx);
    if (nin == 2) rho = tabs(rho);
    const S a2 = gamma * p / rho;
    cval = tsqrt(tabs(a2));
    B.c[idx] = cval;
    if (P.nvis == 1) {
      T = (moo * moo) * a2;
      prim[5 * np + idx] = (double)T;
    }
    if (DO_Q) {
      // update_conservative_block (StateUpdater.cpp:94-149), FP64
      const double r0 = __ldg(prim + idx), u = __ldg(prim + np + idx), v = __ldg(prim + 2 * np + idx),
                   w = __ldg(prim + 3 * np + idx), pd = __ldg(prim + 4 * np + idx);
      const bool use_abs = (nin == 2);
      const double rc = (use_abs || r0 < 0.0) ? fabs(r0) : r0;
      const double gm1_inv = 1.0 / (P.gamma - 1.0);
      B.q[idx] = rc;
      B.q[np + idx] = rc * u;
      B.q[2 * np + idx] = rc * v;
      B.q[3 * np + idx] = rc * w;
      const double ke = 0.5 * rc * (u * u + v * v + w * w);
      B.q[4 * np + idx] = pd * gm1_inv + ke;
    }
  }
  S muv = B.mu[idx];
  if (P.nvis == 1) {
    // update_viscosity_block (StateUpdater.cpp:75-92): whole padded array
    S tm = T;
    if (tm < S(1e-6)) tm = S(1e-6);
    muv = tm * tsqrt(tm) * (S(1) + visc) / (tm + visc);
    B.mu[idx] = muv;
  }
  for (int m = 0; m < 5; ++m) B.dq[m * np + idx] = (S)0;
  if (sizeof(S) == 4) {  // the flux kernels' FP32 copy of prim, after the BCs and T
    for (int m = 0; m < 5; ++m) B.prim_f[m * np + idx] = (float)prim[m * np + idx];
    B.prim_f[5 * np + idx] = (float)prim[5 * np + idx];
  }
  c_out = cval;
  mu_out = muv;
}

template <typename S>
__device__ __forceinline__ S timestep_point(const BlockDev<S>& B, const ParamsDev& P, long long idx, S c, S mu) {
  // calculate_spectrum + calculate_local_dt_cell (TimeIntegrator.cpp:20-125)
  const long long np = B.npad;
  const S u = (S)__ldg(B.prim + np + idx), v = (S)__ldg(B.prim + 2 * np + idx), w = (S)__ldg(B.prim + 3 * np + idx);
  const S rho = (S)__ldg(B.prim + idx);
  const S vol = (S)__ldg(FluxSrc<S>::vol(B) + idx);
  const S reynolds = (S)P.reynolds, csrv = (S)P.csrv;
  S sum_spec = S(0);
  const auto* met = FluxSrc<S>::metrics(B);
  for (int d = 0; d < 3; ++d) {
    const S mx = (S)__ldg(met + (3 * d + 0) * np + idx);
    const S my = (S)__ldg(met + (3 * d + 1) * np + idx);
    const S mz = (S)__ldg(met + (3 * d + 2) * np + idx);
    const S U_contra = tabs(u * mx + v * my + w * mz);
    const S grad_len = tsqrt(mx * mx + my * my + mz * mz);
    const S spec = U_contra + c * grad_len;
    S specv = S(0);
    if (P.nvis == 1) {
      const S grad_sq = mx * mx + my * my + mz * mz;
      const S denom = reynolds * rho * vol + S(1.0e-30);
      specv = (S(2) * mu / denom) * grad_sq * csrv;
    }
    sum_spec += spec + specv;
  }
  const S dt_phys = (S)P.cfl / (sum_spec + S(1.0e-30));
  return dt_phys / vol;
}

// CTA-wide minimum written to part[blockIdx.x] (no same-address atomics: a
// few thousand of those serialize for milliseconds).
__device__ __forceinline__ void block_min_to(double v, double* part) {
  for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, off));
  __shared__ double s_min[32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) s_min[w] = v;
  __syncthreads();
  if (w == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    v = (l < nw) ? s_min[l] : 1000.0;
    for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, off));
    if (l == 0) part[blockIdx.x] = v;
  }
}

// phydtime = min(1000, min over the partials) (TimeIntegrator.cpp:151-176), stored as bits.
__device__ __forceinline__ void dtmin_final_body(const double* __restrict__ part, int n,
                                                 unsigned long long* __restrict__ dtmin_bits);

static __global__ void __launch_bounds__(1024) k_dtmin_final(const double* __restrict__ part, int n,
                                                             unsigned long long* __restrict__ dtmin_bits) {
  dtmin_final_body(part, n, dtmin_bits);
}

__device__ __forceinline__ void dtmin_final_body(const double* __restrict__ part, int n,
                                                 unsigned long long* __restrict__ dtmin_bits) {
  double v = 1000.0;
  for (int t = threadIdx.x; t < n; t += 1024) v = fmin(v, part[t]);
  for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, off));
  __shared__ double s_min[32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) s_min[w] = v;
  __syncthreads();
  if (w == 0) {
    v = s_min[l];
    for (int off = 16; off > 0; off >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, off));
    if (l == 0) *dtmin_bits = (unsigned long long)__double_as_longlong(v);
  }
}

// CTAs per SM (256 threads each) the state and sweep-preparation kernels are
// compiled for (register cap 65536 / (256 n)), per precision.  Measured on C3
// against the compiler's own choice (80-109 registers): FP32 six, FP64 four
// (a few spilled registers each) took the mixed step from 16.7 to 15.9 ms and
// the plain step from 32.7 to 31.7 ms.
#ifndef ORION_PTWISE_MINB_F32
#define ORION_PTWISE_MINB_F32 6
#endif
#ifndef ORION_PTWISE_MINB_F64
#define ORION_PTWISE_MINB_F64 4
#endif
template <typename T> struct PointwiseMinBlocks;
template <> struct PointwiseMinBlocks<float> { static constexpr int n = ORION_PTWISE_MINB_F32; };
template <> struct PointwiseMinBlocks<double> { static constexpr int n = ORION_PTWISE_MINB_F64; };

template <typename S, bool DO_Q, bool DO_DT>
__global__ void __launch_bounds__(256, PointwiseMinBlocks<S>::n) k_state(const BlockDev<S>* __restrict__ blocks, const Chunk* __restrict__ chunks,
                        double* __restrict__ dt_part) {
  const Chunk ch = chunks[blockIdx.x];
  const BlockDev<S> B = blocks[ch.block];
  const ParamsDev& P = B.prm;
  double local_min = 1000.0;
#pragma unroll 4
  for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
    const long long idx = ch.start + t;
    const int i32 = (int)idx;  // padded index < 2^31
    const int i = i32 % B.nx;
    const int r = i32 / B.nx;
    const int j = r % B.ny;
    const int k = r / B.ny;
    S c, mu;
    state_point<S, DO_Q>(B, P, idx, i, j, k, c, mu);
    if (DO_DT) {
      const bool interior = (i >= NG && i < NG + B.ni && j >= NG && j < NG + B.nj && k >= NG && k < NG + B.nk);
      if (interior) {
        const S dtv = timestep_point(B, P, idx, c, mu);
        B.dt[idx] = dtv;
        const double dt_phys = (double)dtv * B.vol[idx];
        if (dt_phys < local_min) local_min = dt_phys;
      }
    }
  }
  if (DO_DT) block_min_to(local_min, dt_part);
}

// time step alone (per-stage entry point): interior points of interior chunks
template <typename S>
__global__ void k_timestep(const BlockDev<S>* __restrict__ blocks, const Chunk* __restrict__ chunks,
                        double* __restrict__ dt_part) {
  const Chunk ch = chunks[blockIdx.x];
  const BlockDev<S> B = blocks[ch.block];
  const ParamsDev& P = B.prm;
  double local_min = 1000.0;
  for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
    const long long n = ch.start + t;  // interior index
    const int n32 = (int)n, r32 = n32 / B.ni;
    const int ii = n32 - r32 * B.ni, jj = r32 % B.nj, kk = r32 / B.nj;
    const long long idx = lin(B, NG + ii, NG + jj, NG + kk);
    const S dtv = timestep_point(B, P, idx, B.c[idx], B.mu[idx]);
    B.dt[idx] = dtv;
    const double dt_phys = (double)dtv * B.vol[idx];
    if (dt_phys < local_min) local_min = dt_phys;
  }
  block_min_to(local_min, dt_part);
}


// ===========================================================================
// Node derivatives of (u,v,w,T) along xi, eta, zeta at interior points
// (compute_derivatives_cell + compute_node_deriv_line,
// src/solver/FluxComputer.cpp:13-67, 301-376).
// ===========================================================================
template <typename T, typename A>
__device__ __forceinline__ T node_deriv(const A* __restrict__ q, long long o, long long st, int t, int L,
                                        bool fl, bool fr) {
  // q + o is memory coordinate 0 of the line, st the along-line stride, t the interior index.
  auto Q = [&](int p) -> T { return (T)q[o + (long long)p * st]; };
  if (fl && t == 0) {
    const T q1 = Q(3), q2 = Q(4), q3 = Q(5), q4 = Q(6);
    return (T(-11) * q1 + T(18) * q2 - T(9) * q3 + T(2) * q4) / T(6);
  }
  if (fl && t == 1) {
    const T q1 = Q(3), q2 = Q(4), q3 = Q(5), q4 = Q(6), q5 = Q(7);
    return (T(-3) * q1 + T(-10) * q2 + T(18) * q3 + T(-6) * q4 + T(1) * q5) / T(12);
  }
  if (fr && t == L - 1) {
    const T qn = Q(L + 2), qn_1 = Q(L + 1), qn_2 = Q(L), qn_3 = Q(L - 1);
    return -(T(-11) * qn + T(18) * qn_1 - T(9) * qn_2 + T(2) * qn_3) / T(6);
  }
  if (fr && t == L - 2) {
    const T qn = Q(L + 2), qn_1 = Q(L + 1), qn_2 = Q(L), qn_3 = Q(L - 1), qn_4 = Q(L - 2);
    return -(T(-3) * qn + T(-10) * qn_1 + T(18) * qn_2 + T(-6) * qn_3 + T(1) * qn_4) / T(12);
  }
  const int p = t + NG;
  return (T(8) * (Q(p + 1) - Q(p - 1)) + T(-1) * (Q(p + 2) - Q(p - 2))) / T(12);
}

template <typename S, typename T>
__global__ void k_node_derivs(const BlockDev<S>* __restrict__ blocks, const Chunk* __restrict__ chunks) {
  const Chunk ch = chunks[blockIdx.x];
  const BlockDev<S> B = blocks[ch.block];
  const long long np = B.npad;
  for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
    const long long n = ch.start + t;
    const int n32 = (int)n, r32 = n32 / B.ni;
    const int ii = n32 - r32 * B.ni, jj = r32 % B.nj, kk = r32 / B.nj;
    const long long idx = lin(B, NG + ii, NG + jj, NG + kk);
    const int tt[3] = {ii, jj, kk};
    for (int d = 0; d < 3; ++d) {
      const long long st = stride_along(B, d);
      const long long o = idx - (long long)(tt[d] + NG) * st;  // along-line coordinate 0
      const int L = dim_along(B, d);
      const bool fl = B.prim[o] < 0.0;
      const bool fr = B.prim[o + (long long)(L + 5) * st] < 0.0;
      const int comp[4] = {1, 2, 3, 5};
      for (int m = 0; m < 4; ++m) {
        const T v = node_deriv<T>(FluxSrc<S>::prim(B) + comp[m] * np, o, st, tt[d], L, fl, fr);
        B.duvwt[(m + 4 * d) * np + idx] = (S)v;
      }
    }
  }
}

// ===========================================================================
// Viscous RHS along one direction D (compute_viscous_flux_block,
// src/solver/FluxComputer.cpp:466-722, with interp_line_to_half :129-178,
// compute_half_deriv_line :72-124, transform_derivs_to_phys :183-205,
// compute_viscous_flux_1d :210-252, compute_flux_diff_1d :257-296).
// One CTA per tile of whole lines: face fluxes to shared memory, then the
// 6th-order difference and dq -= dfv / Re.
// ===========================================================================
template <typename T, typename A>
__device__ __forceinline__ T interp_half(const A* __restrict__ a, long long o, long long st, int f, int L,
                                         bool fl, bool fr) {
  // interp_line_to_half at face f of a line of L points; a + o is memory coordinate 0.
  auto Q = [&](int p) -> T { return (T)a[o + (long long)p * st]; };
  if (fl && f == 0) return (T(35) * Q(3) + T(-35) * Q(4) + T(21) * Q(5) + T(-5) * Q(6)) / T(16);
  if (fl && f == 1) return (T(5) * Q(3) + T(15) * Q(4) + T(-5) * Q(5) + T(1) * Q(6)) / T(16);
  if (fr && f == L) return (T(35) * Q(L + 2) + T(-35) * Q(L + 1) + T(21) * Q(L) + T(-5) * Q(L - 1)) / T(16);
  if (fr && f == L - 1) return (T(5) * Q(L + 2) + T(15) * Q(L + 1) + T(-5) * Q(L) + T(1) * Q(L - 1)) / T(16);
  return (T(9) * (Q(f + 2) + Q(f + 3)) + T(-1) * (Q(f + 4) + Q(f + 1))) / T(16);
}

template <typename T, typename S>
__device__ __forceinline__ T interp_half_s(const S* __restrict__ a, long long o, long long st, int f) {
  auto Q = [&](int p) -> T { return (T)a[o + (long long)p * st]; };
  return (T(9) * (Q(f + 2) + Q(f + 3)) + T(-1) * (Q(f + 4) + Q(f + 1))) / T(16);
}

template <typename T, typename A>
__device__ __forceinline__ T half_deriv(const A* __restrict__ a, long long o, long long st, int f, int L, bool fl,
                                        bool fr) {
  auto Q = [&](int p) -> T { return (T)a[o + (long long)p * st]; };
  if (fl && f == 0) return (T(-71) * Q(3) + T(141) * Q(4) + T(-93) * Q(5) + T(23) * Q(6)) / T(24);
  if (fl && f == 1) return (T(-22) * Q(3) + T(17) * Q(4) + T(9) * Q(5) + T(-5) * Q(6) + T(1) * Q(7)) / T(24);
  if (fr && f == L) return -(T(-71) * Q(L + 2) + T(141) * Q(L + 1) + T(-93) * Q(L) + T(23) * Q(L - 1)) / T(24);
  if (fr && f == L - 1)
    return -(T(-22) * Q(L + 2) + T(17) * Q(L + 1) + T(9) * Q(L) + T(-5) * Q(L - 1) + T(1) * Q(L - 2)) / T(24);
  return (T(27) * (Q(f + 3) - Q(f + 2)) + T(-1) * (Q(f + 4) - Q(f + 1))) / T(24);
}

// cross derivative interpolated to face f with the source index clamped to the interior
template <typename T, typename S>
__device__ __forceinline__ T cross_half(const S* __restrict__ a, long long o, long long st, int f, int L) {
  auto Q = [&](int p) -> T {
    const int pc = p < NG ? NG : (p > L + NG - 1 ? L + NG - 1 : p);
    return (T)a[o + (long long)pc * st];
  };
  return (T(9) * (Q(f + 2) + Q(f + 3)) + T(-1) * (Q(f + 4) + Q(f + 1))) / T(16);
}

template <int D, typename S, typename T>
__device__ __forceinline__ void viscous_face(const BlockDev<S>& B, const ParamsDev& P, long long o, int f, int L,
                                             bool fl, bool fr, T cp_prl, T fv[4]) {
  const long long np = B.npad;
  const long long st = stride_along(B, D);
  const auto* prim = FluxSrc<S>::prim(B);
  T uvwt[4];
  const int comp[4] = {1, 2, 3, 5};
  for (int m = 0; m < 4; ++m) uvwt[m] = interp_half<T>(prim + comp[m] * np, o, st, f, L, fl, fr);
  const T vs = interp_half_s<T, S>(B.mu, o, st, f);
  const T kcp = vs * cp_prl;
  const T volh = interp_half_s<T, S>(FluxSrc<S>::vol(B), o, st, f);
  T kxyz[9];
  const auto* met = FluxSrc<S>::metrics(B);
  for (int m = 0; m < 9; ++m) kxyz[m] = interp_half_s<T, S>(met + m * np, o, st, f);
  T d[12];
  // derivative along the line (half point), cross derivatives interpolated
  for (int m = 0; m < 4; ++m) d[m + 4 * D] = half_deriv<T>(prim + comp[m] * np, o, st, f, L, fl, fr);
#pragma unroll
  for (int dd = 0; dd < 3; ++dd) {
    if (dd == D) continue;
    for (int m = 0; m < 4; ++m) d[m + 4 * dd] = cross_half<T, S>(B.duvwt + (m + 4 * dd) * np, o, st, f, L);
  }
  // transform_derivs_to_phys
  const T vol_inv = T(1) / volh;
  T g[12];
  for (int m = 0; m < 3; ++m) {
    const T k1 = kxyz[m], k2 = kxyz[m + 3], k3 = kxyz[m + 6];
    for (int v = 0; v < 4; ++v) g[v * 3 + m] = (k1 * d[v] + k2 * d[v + 4] + k3 * d[v + 8]) * vol_inv;
  }
  // compute_viscous_flux_1d
  const T CC = T(2.0 / 3.0);
  const T vscc = vs * CC;
  const T dudx = g[0], dudy = g[1], dudz = g[2];
  const T dvdx = g[3], dvdy = g[4], dvdz = g[5];
  const T dwdx = g[6], dwdy = g[7], dwdz = g[8];
  const T txx = vscc * (T(2) * dudx - dvdy - dwdz);
  const T tyy = vscc * (T(2) * dvdy - dwdz - dudx);
  const T tzz = vscc * (T(2) * dwdz - dudx - dvdy);
  const T txy = vs * (dudy + dvdx);
  const T txz = vs * (dudz + dwdx);
  const T tyz = vs * (dvdz + dwdy);
  const T nx = kxyz[3 * D + 0], ny = kxyz[3 * D + 1], nz = kxyz[3 * D + 2];
  fv[0] = txx * nx + txy * ny + txz * nz;
  fv[1] = txy * nx + tyy * ny + tyz * nz;
  fv[2] = txz * nx + tyz * ny + tzz * nz;
  const T work = uvwt[0] * fv[0] + uvwt[1] * fv[1] + uvwt[2] * fv[2];
  const T heat = kcp * (g[9] * nx + g[10] * ny + g[11] * nz);
  fv[3] = work + heat;
}

template <int D>
__device__ __forceinline__ void tile_item(int it, int nlanes, int nfaces, int& lane, int& pos) {
  if (D == 0) {
    lane = it / nfaces;
    pos = it - lane * nfaces;
  } else {
    pos = it / nlanes;
    lane = it - pos * nlanes;
  }
}

// CTAs per SM the line kernels are compiled for (register cap 65536/(256*n)),
// per compute precision, measured on C3: FP32 five (viscous; 3.91 ms against
// 4.03 at six and 4.09 at four) and five (inviscid; four and six were slower),
// FP64 three (viscous) and three (inviscid, with its boundary rounds in their
// own kernel; two CTAs when they were inline).
#ifndef ORION_VISC_MINB_F32
#define ORION_VISC_MINB_F32 5
#endif
#ifndef ORION_INV_MINB_F32
#define ORION_INV_MINB_F32 5
#endif
#ifndef ORION_VISC_MINB_F64
#define ORION_VISC_MINB_F64 3
#endif
#ifndef ORION_INV_MINB_F64
#define ORION_INV_MINB_F64 3
#endif
template <typename T> struct LineMinBlocks;
template <> struct LineMinBlocks<float> { static constexpr int visc = ORION_VISC_MINB_F32, inv = ORION_INV_MINB_F32; };
template <> struct LineMinBlocks<double> { static constexpr int visc = ORION_VISC_MINB_F64, inv = ORION_INV_MINB_F64; };

template <int D, typename S, typename T>
__global__ void __launch_bounds__(256, LineMinBlocks<T>::visc) k_viscous(const BlockDev<S>* __restrict__ blocks, const LineTile* __restrict__ tiles) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* fsh = reinterpret_cast<T*>(smem_raw);
  const LineTile tl = tiles[blockIdx.x];
  const BlockDev<S> B = blocks[tl.block];
  const ParamsDev& P = B.prm;
  const int L = dim_along(B, D);
  const int nf = L + 1;
  const long long st = stride_along(B, D);
  const T cp = T(1) / ((T(P.gamma) - T(1)) * T(P.moo) * T(P.moo));
  const T cp_prl = cp / T(P.prl);
  const T re_inv = (fabs(P.reynolds) > 1.0e-30) ? T(1) / T(P.reynolds) : T(0);
  const int nitems = tl.count * nf;
  for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
    int lane, f;
    tile_item<D>(it, tl.count, nf, lane, f);
    const long long o = line_origin(B, D, tl.first + lane);
    const bool fl = B.prim[o] < 0.0;
    const bool fr = B.prim[o + (long long)(L + 5) * st] < 0.0;
    T fv[4];
    viscous_face<D, S, T>(B, P, o, f, L, fl, fr, cp_prl, fv);
    T* dst = fsh + ((size_t)lane * nf + f) * 4;
    dst[0] = fv[0];
    dst[1] = fv[1];
    dst[2] = fv[2];
    dst[3] = fv[3];
  }
  __syncthreads();
  const int npts = tl.count * L;
  for (int it = threadIdx.x; it < npts; it += blockDim.x) {
    int lane, t;
    tile_item<D>(it, tl.count, L, lane, t);
    const long long o = line_origin(B, D, tl.first + lane);
    const long long idx = o + (long long)(t + NG) * st;
    const T* fb = fsh + (size_t)lane * nf * 4;
    for (int m = 0; m < 4; ++m) {
      const T dfv = flux_diff<T>(fb + m, 4, t, L);
      S* q = B.dq + (m + 1) * B.npad + idx;
      *q = (S)((T)*q - re_inv * dfv);
    }
  }
}

// ===========================================================================
// Inviscid RHS along one direction D (compute_block_inviscid + compute_flux_line,
// src/solver/InviscidFluxComputer.cpp:136-192, 238-522, 543-647).
// Face fluxes from WCNS-E-5 states (fixed stencils where the ghost-3 density
// flag is set) and the Roe flux, then the flux difference; the boundary
// re-calculation rounds (:377-521) are evaluated per output point by the
// threads of points 0..2 and L-3..L-1 of flagged line ends.
// ===========================================================================
template <typename S, typename T>
struct InvLine {
  const S* prim;  // FluxSrc<S>::prim
  long long o, st, np;
  int L;
  __device__ __forceinline__ T q(int p, int m) const { return (T)prim[m * np + o + (long long)p * st]; }
};

template <typename S, typename T>
__device__ __forceinline__ T metric_half(const BlockDev<S>& B, int mc, long long o, long long st, int f, int L) {
  // interp_metrics_half (InviscidFluxComputer.cpp:136-192), ni > 2
  const S* a = FluxSrc<S>::metrics(B) + mc * B.npad;
  auto Q = [&](int p) -> T { return (T)a[o + (long long)p * st]; };
  if (f == 0) return (T(35) * Q(3) + T(-35) * Q(4) + T(21) * Q(5) + T(-5) * Q(6)) / T(16);
  if (f == 1) return (T(5) * Q(3) + T(15) * Q(4) + T(-5) * Q(5) + T(1) * Q(6)) / T(16);
  if (f == L) return (T(35) * Q(L + 2) + T(-35) * Q(L + 1) + T(21) * Q(L) + T(-5) * Q(L - 1)) / T(16);
  if (f == L - 1) return (T(5) * Q(L + 2) + T(15) * Q(L + 1) + T(-5) * Q(L) + T(1) * Q(L - 1)) / T(16);
  return (T(9) * (Q(f + 2) + Q(f + 3)) + T(-1) * (Q(f + 4) + Q(f + 1))) / T(16);
}

// Initial left/right states at face f (main WCNS loop + fixed boundary stencils).
template <typename S, typename T>
__device__ __forceinline__ void initial_states(const InvLine<S, T>& ln, int f, bool fl, bool fr, T ql[5], T qr[5]) {
  const int L = ln.L;
  const int ist = fl ? 2 : 0, ied = fr ? L - 2 : L;
  for (int m = 0; m < 5; ++m) {
    T l = T(0), r = T(0);
    if (f >= ist && f <= ied) {
      const T a0 = ln.q(f, m), a1 = ln.q(f + 1, m), a2 = ln.q(f + 2, m), a3 = ln.q(f + 3, m), a4 = ln.q(f + 4, m),
              a5 = ln.q(f + 5, m);
      l = wcns_left<T>(a0, a1, a2, a3, a4);
      r = wcns_right<T>(a1, a2, a3, a4, a5);
    }
    if (ist > 1 && f <= 2) {
      const T q1 = ln.q(3, m), q2 = ln.q(4, m), q3 = ln.q(5, m), q4 = ln.q(6, m);
      if (f == 0) {
        l = (T(35.) * q1 - T(35.) * q2 + T(21.) * q3 - T(5.) * q4) / T(16.);
        r = l;
      } else if (f == 1) {
        l = (T(5.) * q1 + T(15.) * q2 - T(5.) * q3 + q4) / T(16.);
        r = l;
      } else {
        l = (-q1 + T(9.) * q2 + T(9.) * q3 - q4) / T(16.);
      }
    }
    if (ied < L && f >= L - 2) {
      const T qn = ln.q(L + 2, m), qn1 = ln.q(L + 1, m), qn2 = ln.q(L, m), qn3 = ln.q(L - 1, m);
      if (f == L) {
        r = (T(35.) * qn - T(35.) * qn1 + T(21.) * qn2 - T(5.) * qn3) / T(16.);
        l = r;
      } else if (f == L - 1) {
        r = (T(5.) * qn + T(15.) * qn1 - T(5.) * qn2 + qn3) / T(16.);
        l = r;
      } else {
        r = (-qn + T(9.) * qn1 + T(9.) * qn2 - qn3) / T(16.);
      }
    }
    ql[m] = l;
    qr[m] = r;
  }
}

template <int D, typename S, typename T>
__device__ __forceinline__ void face_metric(const BlockDev<S>& B, long long o, long long st, int f, int L, T& kx,
                                            T& ky, T& kz) {
  kx = metric_half<S, T>(B, 3 * D + 0, o, st, f, L);
  ky = metric_half<S, T>(B, 3 * D + 1, o, st, f, L);
  kz = metric_half<S, T>(B, 3 * D + 2, o, st, f, L);
}

// Positivity fallback + Roe flux at face f (calc_flux_loop, InviscidFluxComputer.cpp:342-364).
template <typename S, typename T>
__device__ __forceinline__ void fallback_roe(const InvLine<S, T>& ln, int f, T ql[5], T qr[5], T kx, T ky, T kz,
                                             T gamma, T out[5]) {
  const int L = ln.L;
  if (ql[0] <= T(1e-6) || ql[4] <= T(1e-6)) {
    const int p = (f - 1 > 0 ? f - 1 : 0) + 2;
    for (int m = 0; m < 5; ++m) ql[m] = ln.q(p, m);
  }
  if (qr[0] <= T(1e-6) || qr[4] <= T(1e-6)) {
    const int p = (L - 1 < f ? L - 1 : f) + 3;
    for (int m = 0; m < 5; ++m) qr[m] = ln.q(p, m);
  }
  roe_flux<T>(ql, qr, kx, ky, kz, T(0), T(0.1), gamma, out);
}

// Left-end re-calculation rounds (InviscidFluxComputer.cpp:377-448): the value
// of fc[t] for t = 0, 1, 2 when the ghost-3 density flag is set.
// Boundary re-calculation rounds of a flagged line end
// (InviscidFluxComputer.cpp:377-521).  Each output point needs one round of
// 4-5 Roe fluxes; every flux is folded into the output as soon as it is
// computed, in the order and with the coefficients of the reference's formula,
// so no per-face array is kept.
template <int D, typename S, typename T>
struct Cascade {
  const BlockDev<S>& B;
  const InvLine<S, T>& ln;
  T gamma;
  T acc[5];
  __device__ __forceinline__ void flux(int f, const T l[5], const T r[5], T coef, bool first) {
    T ql[5], qr[5], out[5];
    for (int m = 0; m < 5; ++m) { ql[m] = l[m]; qr[m] = r[m]; }
    T kx, ky, kz;
    face_metric<D, S, T>(B, ln.o, ln.st, f, ln.L, kx, ky, kz);
    fallback_roe<S, T>(ln, f, ql, qr, kx, ky, kz, gamma, out);
    // acc = coef*F (first term) or acc + coef*F; a coefficient of +1 or -1 is an
    // exact add or subtract of F as in the reference's expression
    for (int m = 0; m < 5; ++m) {
      if (first) acc[m] = coef * out[m];
      else if (coef == T(1)) acc[m] = acc[m] + out[m];
      else if (coef == T(-1)) acc[m] = acc[m] - out[m];
      else acc[m] = acc[m] + coef * out[m];
    }
  }
};

template <int D, typename S, typename T>
__device__ void cascade_left(const BlockDev<S>& B, const InvLine<S, T>& ln, int t, T gamma, T fc[5]) {
  Cascade<D, S, T> cs{B, ln, gamma, {}};
  T Q3[5], Q4[5], Q5[5], Q6[5];
  for (int m = 0; m < 5; ++m) { Q3[m] = ln.q(3, m); Q4[m] = ln.q(4, m); Q5[m] = ln.q(5, m); Q6[m] = ln.q(6, m); }
  T s[5], s2[5];
  if (t == 0) {
    // fc[0] = (-23 F0 + 21 F1 + 3 F2 - F3) / 24 over round-1 states
    for (int m = 0; m < 5; ++m) s[m] = (T(3.) * Q3[m] - T(1.) * Q4[m]) / T(2.0);
    cs.flux(0, s, s, T(-23.), true);
    for (int m = 0; m < 5; ++m) s[m] = (T(19.) * Q3[m] + T(25.) * Q4[m] - T(2.) * Q5[m]) / T(42.0);
    cs.flux(1, s, s, T(21.), false);
    for (int m = 0; m < 5; ++m) s[m] = (T(4.) * Q3[m] + T(3.) * Q4[m] + T(9.) * Q5[m] + T(2.) * Q6[m]) / T(18.0);
    cs.flux(2, s, s, T(3.), false);
    for (int m = 0; m < 5; ++m) s[m] = (T(-2.) * Q3[m] + T(3.) * Q4[m] + T(3.) * Q5[m] + T(2.) * Q6[m]) / T(6.0);
    cs.flux(3, s, s, T(-1), false);
  } else if (t == 1) {
    // fc[1] = (-22 F1 + 17 F2 + 9 F3 - 5 F4 + F5) / 24 over round-2 states
    for (int m = 0; m < 5; ++m) s[m] = (T(3.) * Q3[m] + T(6.) * Q4[m] - Q5[m]) / T(8.0);
    cs.flux(1, s, s, T(-22.), true);
    for (int m = 0; m < 5; ++m) {
      s[m] = (T(-30.) * Q3[m] + T(145.) * Q4[m] + T(29.) * Q5[m] - T(8.) * Q6[m]) / T(136.0);
      s2[m] = (T(2.) * Q3[m] + T(49.) * Q4[m] + T(125.) * Q5[m] - T(40.) * Q6[m]) / T(136.0);
    }
    cs.flux(2, s, s2, T(17.), false);
    for (int m = 0; m < 5; ++m) s[m] = (-Q4[m] + T(6.) * Q5[m] + T(3.) * Q6[m]) / T(8.0);
    cs.flux(3, s, s, T(9.), false);
    for (int m = 0; m < 5; ++m) s[m] = (Q4[m] + T(2.) * Q5[m] + T(5.) * Q6[m]) / T(8.0);
    cs.flux(4, s, s, T(-5.), false);
    for (int m = 0; m < 5; ++m) s[m] = (Q4[m] + Q5[m] + T(6.) * Q6[m]) / T(8.0);
    cs.flux(5, s, s, T(1), false);
  } else {
    // fc[2] = (F1 - 27 F2 + 27 F3 - F4) / 24 over round-3 states; face 1 keeps the
    // round-2 left state and the restored fixed right state, faces 2..4 the
    // restored WCNS right states
    for (int m = 0; m < 5; ++m) {
      s[m] = (T(3.) * Q3[m] + T(6.) * Q4[m] - Q5[m]) / T(8.0);
      s2[m] = (T(5.) * Q3[m] + T(15.) * Q4[m] - T(5.) * Q5[m] + Q6[m]) / T(16.);
    }
    cs.flux(1, s, s2, T(1), true);
    const T coef[3] = {T(-27.), T(27.), T(-1)};
    for (int f = 2; f <= 4; ++f) {
      for (int m = 0; m < 5; ++m) {
        if (f == 2) s[m] = (T(-29.) * Q3[m] + T(170.) * Q4[m] + T(63.) * Q5[m] + T(12.) * Q6[m]) / T(216.0);
        else if (f == 3) s[m] = (-Q4[m] + T(6.) * Q5[m] + T(3.) * Q6[m]) / T(8.0);
        else s[m] = (Q4[m] + T(2.) * Q5[m] + T(5.) * Q6[m]) / T(8.0);
        s2[m] = wcns_right<T>(ln.q(f + 1, m), ln.q(f + 2, m), ln.q(f + 3, m), ln.q(f + 4, m), ln.q(f + 5, m));
      }
      cs.flux(f, s, s2, coef[f - 2], false);
    }
  }
  for (int m = 0; m < 5; ++m) fc[m] = cs.acc[m] / T(24.0);
}

template <int D, typename S, typename T>
__device__ void cascade_right(const BlockDev<S>& B, const InvLine<S, T>& ln, int t, T gamma, T fc[5]) {
  const int N = ln.L;
  Cascade<D, S, T> cs{B, ln, gamma, {}};
  T Qn[5], Qn1[5], Qn2[5], Qn3[5];
  for (int m = 0; m < 5; ++m) {
    Qn[m] = ln.q(N + 2, m); Qn1[m] = ln.q(N + 1, m); Qn2[m] = ln.q(N, m); Qn3[m] = ln.q(N - 1, m);
  }
  T s[5], s2[5];
  if (t == N - 1) {
    // fc[N-1] = -(-23 F[N] + 21 F[N-1] + 3 F[N-2] - F[N-3]) / 24
    for (int m = 0; m < 5; ++m) s[m] = (T(3.) * Qn[m] - T(1.) * Qn1[m]) / T(2.0);
    cs.flux(N, s, s, T(-23.), true);
    for (int m = 0; m < 5; ++m) s[m] = (T(19.) * Qn[m] + T(25.) * Qn1[m] - T(2.) * Qn2[m]) / T(42.0);
    cs.flux(N - 1, s, s, T(21.), false);
    for (int m = 0; m < 5; ++m) s[m] = (T(4.) * Qn[m] + T(3.) * Qn1[m] + T(9.) * Qn2[m] + T(2.) * Qn3[m]) / T(18.0);
    cs.flux(N - 2, s, s, T(3.), false);
    for (int m = 0; m < 5; ++m) s[m] = (T(-2.) * Qn[m] + T(3.) * Qn1[m] + T(3.) * Qn2[m] + T(2.) * Qn3[m]) / T(6.0);
    cs.flux(N - 3, s, s, T(-1), false);
  } else if (t == N - 2) {
    // fc[N-2] = -(-22 F[N-1] + 17 F[N-2] + 9 F[N-3] - 5 F[N-4] + F[N-5]) / 24
    for (int m = 0; m < 5; ++m) s[m] = (T(3.) * Qn[m] + T(6.) * Qn1[m] - Qn2[m]) / T(8.0);
    cs.flux(N - 1, s, s, T(-22.), true);
    for (int m = 0; m < 5; ++m) {
      s2[m] = (T(-30.) * Qn[m] + T(145.) * Qn1[m] + T(29.) * Qn2[m] - T(8.) * Qn3[m]) / T(136.0);  // right
      s[m] = (T(2.) * Qn[m] + T(49.) * Qn1[m] + T(125.) * Qn2[m] - T(40.) * Qn3[m]) / T(136.0);    // left
    }
    cs.flux(N - 2, s, s2, T(17.), false);
    for (int m = 0; m < 5; ++m) s[m] = (-Qn1[m] + T(6.) * Qn2[m] + T(3.) * Qn3[m]) / T(8.0);
    cs.flux(N - 3, s, s, T(9.), false);
    for (int m = 0; m < 5; ++m) s[m] = (Qn1[m] + T(2.) * Qn2[m] + T(5.) * Qn3[m]) / T(8.0);
    cs.flux(N - 4, s, s, T(-5.), false);
    for (int m = 0; m < 5; ++m) s[m] = (Qn1[m] + Qn2[m] + T(6.) * Qn3[m]) / T(8.0);
    cs.flux(N - 5, s, s, T(1), false);
  } else {
    // fc[N-3] = -(F[N-1] - 27 F[N-2] + 27 F[N-3] - F[N-4]) / 24
    for (int m = 0; m < 5; ++m) {
      s2[m] = (T(3.) * Qn[m] + T(6.) * Qn1[m] - Qn2[m]) / T(8.0);
      s[m] = (T(5.) * Qn[m] + T(15.) * Qn1[m] - T(5.) * Qn2[m] + Qn3[m]) / T(16.);
    }
    cs.flux(N - 1, s, s2, T(1), true);
    const T coef[3] = {T(-27.), T(27.), T(-1)};
    for (int f = N - 2; f >= N - 4; --f) {
      for (int m = 0; m < 5; ++m) {
        if (f == N - 2) s2[m] = (T(-29.) * Qn[m] + T(170.) * Qn1[m] + T(63.) * Qn2[m] + T(12.) * Qn3[m]) / T(216.0);
        else if (f == N - 3) s2[m] = (-Qn1[m] + T(6.) * Qn2[m] + T(3.) * Qn3[m]) / T(8.0);
        else s2[m] = (Qn1[m] + T(2.) * Qn2[m] + T(5.) * Qn3[m]) / T(8.0);
        s[m] = wcns_left<T>(ln.q(f, m), ln.q(f + 1, m), ln.q(f + 2, m), ln.q(f + 3, m), ln.q(f + 4, m));
      }
      cs.flux(f, s, s2, coef[N - 2 - f], false);
    }
  }
  for (int m = 0; m < 5; ++m) fc[m] = -cs.acc[m] / T(24.0);
}

// Boundary re-calculation of flagged line ends (InviscidFluxComputer.cpp:377-521)
// for one tile: the six outputs of each line's two ends by consecutive threads.
// k_inviscid's regular loop skips these points, so each point's dq gets
// direction D's terms once and in direction order.
template <int D, typename S, typename T>
__device__ __forceinline__ void inv_boundary_rounds(const BlockDev<S>& B, const LineTile& tl, int L, long long st,
                                                    T gamma) {
  const int nbnd = tl.count * 6;
  for (int it = threadIdx.x; it < nbnd; it += blockDim.x) {
    const int lane = it / 6, slot = it - lane * 6;
    const long long o = line_origin(B, D, tl.first + lane);
    const bool left = slot < 3;
    const bool flag = left ? (B.prim[o] < 1.0e-20) : (B.prim[o + (long long)(L + 5) * st] < 1.0e-20);
    if (!flag) continue;
    const int t = left ? slot : L - 6 + slot;
    InvLine<S, T> ln{FluxSrc<S>::prim(B), o, st, B.npad, L};
    T fc[5];
    if (left) cascade_left<D, S, T>(B, ln, t, gamma, fc);
    else cascade_right<D, S, T>(B, ln, t, gamma, fc);
    const long long idx = o + (long long)(t + NG) * st;
    for (int m = 0; m < 5; ++m) {
      S* q = B.dq + m * B.npad + idx;
      *q = (S)((T)*q + fc[m]);
    }
  }
}

// The boundary rounds run in their own launch after k_inviscid<D>, over the
// same tiles, with CTAs sized to a tile's six outputs per line: inlined, their
// Roe fluxes need about 128 (FP32) or 250 (FP64) registers, against 48 and 80
// for the face loop.  On C3 the split took the inviscid stage from 3.61 to
// 3.25 ms mixed and from 12.2 to 11.9 ms plain (the FP64 face loop at three
// CTAs per SM).
template <int D, typename S, typename T>
__global__ void __launch_bounds__(256) k_inv_cascade(const BlockDev<S>* __restrict__ blocks,
                                                     const LineTile* __restrict__ tiles) {
  const LineTile tl = tiles[blockIdx.x];
  const BlockDev<S> B = blocks[tl.block];
  inv_boundary_rounds<D, S, T>(B, tl, dim_along(B, D), stride_along(B, D), T(B.prm.gamma));
}

template <int D, typename S, typename T>
__global__ void __launch_bounds__(256, LineMinBlocks<T>::inv) k_inviscid(const BlockDev<S>* __restrict__ blocks, const LineTile* __restrict__ tiles) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* fsh = reinterpret_cast<T*>(smem_raw);
  const LineTile tl = tiles[blockIdx.x];
  const BlockDev<S> B = blocks[tl.block];
  const ParamsDev& P = B.prm;
  const int L = dim_along(B, D);
  const int nf = L + 1;
  const long long st = stride_along(B, D);
  const T gamma = T(P.gamma);
  const int nitems = tl.count * nf;
  for (int it = threadIdx.x; it < nitems; it += blockDim.x) {
    int lane, f;
    tile_item<D>(it, tl.count, nf, lane, f);
    const long long o = line_origin(B, D, tl.first + lane);
    InvLine<S, T> ln{FluxSrc<S>::prim(B), o, st, B.npad, L};
    const bool fl = B.prim[o] < 1.0e-20;
    const bool fr = B.prim[o + (long long)(L + 5) * st] < 1.0e-20;
    T ql[5], qr[5], kx, ky, kz, fo[5];
    initial_states<S, T>(ln, f, fl, fr, ql, qr);
    face_metric<D, S, T>(B, o, st, f, L, kx, ky, kz);
    fallback_roe<S, T>(ln, f, ql, qr, kx, ky, kz, gamma, fo);
    T* dst = fsh + ((size_t)lane * nf + f) * 5;
    for (int m = 0; m < 5; ++m) dst[m] = fo[m];
  }
  __syncthreads();
  // regular points: flux difference of the face fluxes
  const int npts = tl.count * L;
  for (int it = threadIdx.x; it < npts; it += blockDim.x) {
    int lane, t;
    tile_item<D>(it, tl.count, L, lane, t);
    const long long o = line_origin(B, D, tl.first + lane);
    const bool fl = B.prim[o] < 1.0e-20;
    const bool fr = B.prim[o + (long long)(L + 5) * st] < 1.0e-20;
    if ((fl && t <= 2) || (fr && t >= L - 3)) continue;  // re-calculated below
    const long long idx = o + (long long)(t + NG) * st;
    const T* fb = fsh + (size_t)lane * nf * 5;
    for (int m = 0; m < 5; ++m) {
      S* q = B.dq + m * B.npad + idx;
      *q = (S)((T)*q + flux_diff<T>(fb + m, 5, t, L));
    }
  }

}


// ===========================================================================
// Interface residual averaging (HaloExchanger::average_interface_residuals,
// src/solver/HaloExchanger.cpp:186-398): pack dq/vol of every source window
// before any update, then each destination point applies its partners in
// region order: dq = 0.5 * (dens_t * vol + dq).
// ===========================================================================
template <typename S>
__global__ void k_iface_pack(const BlockDev<S>* __restrict__ blocks, const int* __restrict__ pk_block,
                             const long long* __restrict__ pk_idx, double* __restrict__ pack, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const BlockDev<S> B = blocks[pk_block[t]];
  const long long idx = pk_idx[t];
  const double vol = B.vol[idx];
  for (int m = 0; m < 5; ++m) pack[(long long)t * 5 + m] = (double)B.dq[m * B.npad + idx] / vol;
}

template <typename S>
__global__ void k_iface_apply(const BlockDev<S>* __restrict__ blocks, const int* __restrict__ ap_block,
                              const long long* __restrict__ ap_idx, const int* __restrict__ ap_off,
                              const int* __restrict__ ap_slot, const double* __restrict__ pack, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const BlockDev<S> B = blocks[ap_block[t]];
  const long long idx = ap_idx[t];
  const double vol_s = B.vol[idx];
  double q[5];
  for (int m = 0; m < 5; ++m) q[m] = (double)B.dq[m * B.npad + idx];
  for (int e = ap_off[t]; e < ap_off[t + 1]; ++e) {
    const long long sl = ap_slot[e];
    for (int m = 0; m < 5; ++m) {
      const double dens_t = pack[sl * 5 + m];
      q[m] = (double)(S)(0.5 * (dens_t * vol_s + q[m]));
    }
  }
  for (int m = 0; m < 5; ++m) B.dq[m * B.npad + idx] = (S)q[m];
}

// ===========================================================================
// LU-SGS / symmetric Gauss-Seidel (StateUpdater::update_solution,
// src/solver/StateUpdater.cpp:267-580) on the plane-major layout.
// Any order that visits a point after its lower face neighbours and before its
// upper ones reproduces the lexicographic sweeps exactly; the hyperplane order
// does, and each hyperplane is a contiguous, coalesced range here.
// ===========================================================================
template <typename S>
__device__ __forceinline__ int jlo_of(const BlockDev<S>& B, int s, int kk) {
  const int v = s - kk - (B.ni - 1);
  return v > 0 ? v : 0;
}

template <typename S>
__device__ __forceinline__ void decode_nat(const BlockDev<S>& B, int nat, int& ii, int& jj, int& kk) {
  const int i = nat % B.nx;
  const int r = nat / B.nx;
  ii = i - NG;
  jj = r % B.ny - NG;
  kk = r / B.ny - NG;
}

__device__ __forceinline__ double sqrt_s(double x) { return sqrt(x); }
__device__ __forceinline__ float sqrt_s(float x) { return sqrtf(x); }

// Static skewed operands (metrics, vol, unit normals): refreshed whenever they are uploaded.
// FP32 shadows of one block's metrics and vol (padded, ghosts included).
static __global__ void k_metric_shadow(const BlockDev<float>* __restrict__ blocks, int b) {
  const BlockDev<float>& B = blocks[b];
  const long long np = B.npad;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < np; idx += (long long)gridDim.x * blockDim.x) {
    for (int m = 0; m < 9; ++m) B.met_f[m * np + idx] = (float)B.metrics[m * np + idx];
    B.vol_f[idx] = (float)B.vol[idx];
  }
}

// FP32 shadow of one block's prim (after an upload or the initial state).
static __global__ void k_prim_shadow(const BlockDev<float>* __restrict__ blocks, int b) {
  const BlockDev<float>& B = blocks[b];
  const long long np = B.npad;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < np; idx += (long long)gridDim.x * blockDim.x)
    for (int m = 0; m < 6; ++m) B.prim_f[m * np + idx] = (float)B.prim[m * np + idx];
}

template <typename S>
__global__ void k_skew_static(const BlockDev<S>* __restrict__ blocks, int b) {
  const BlockDev<S> B = blocks[b];
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < B.ncomp; c += (long long)gridDim.x * blockDim.x) {
    const int nat = B.sk_nat[c];
    for (int m = 0; m < 9; ++m) B.sk_metrics[m * B.ncomp + c] = (S)B.metrics[m * B.npad + nat];
    B.sk_vol[c] = (S)B.vol[nat];
    // unit normals of compute_flux_splitting (StateUpdater.cpp:231-249), per direction
    for (int d = 0; d < 3; ++d) {
      const S nx = B.sk_metrics[(3 * d) * B.ncomp + c], ny = B.sk_metrics[(3 * d + 1) * B.ncomp + c],
              nz = B.sk_metrics[(3 * d + 2) * B.ncomp + c];
      S grad_mag = sqrt_s(nx * nx + ny * ny + nz * nz);
      if (grad_mag < S(1.0e-30)) grad_mag = S(1.0e-30);
      const S inv_mag = S(1) / grad_mag;
      B.sk_nrm[(3 * d) * B.ncomp + c] = nx * inv_mag;
      B.sk_nrm[(3 * d + 1) * B.ncomp + c] = ny * inv_mag;
      B.sk_nrm[(3 * d + 2) * B.ncomp + c] = nz * inv_mag;
      // the unclamped magnitude the spectral radius uses, and the reciprocal of the clamped one
      B.sk_gm[d * B.ncomp + c] = sqrt_s(nx * nx + ny * ny + nz * nz);
      B.sk_inv[d * B.ncomp + c] = inv_mag;
    }
  }
}

// Prep: gather prim, mu into the skewed layout; rhs = dq with physical-BC
// windows zeroed (set_boundary_dq_zero + the AoS copy, StateUpdater.cpp:447-570);
// diagonal coefficient 1/(1/dt + sum of radii) (get_diag_coeff :267-295), the
// same in all four sweeps.
template <typename S, typename T, bool PAIRS = true>
__global__ void __launch_bounds__(256, PointwiseMinBlocks<T>::n) k_lusgs_prep(const BlockDev<S>* __restrict__ blocks, const Chunk* __restrict__ chunks) {
  const Chunk ch = chunks[blockIdx.x];
  const BlockDev<S> B = blocks[ch.block];
  const ParamsDev& P = B.prm;
  const long long np = B.npad, nc = B.ncomp;
  const T gamma = T(P.gamma), reynolds = T(P.reynolds);
  for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
    const long long c = ch.start + t;
    const int nat = B.sk_nat[c];
    const bool masked = B.bcmask[nat] != 0;
    for (int m = 0; m < 5; ++m) B.sk_rhs[m * nc + c] = masked ? (S)0 : B.dq[m * np + nat];
    const S* pr = FluxSrc<S>::prim(B);
    const T rho = (T)pr[nat], u = (T)pr[np + nat], v = (T)pr[2 * np + nat], w = (T)pr[3 * np + nat],
            p = (T)pr[4 * np + nat];
    if (PAIRS) {  // the operands of k_sweep_pairs
      B.sk_prim[c] = (S)rho;
      B.sk_prim[nc + c] = (S)u;
      B.sk_prim[2 * nc + c] = (S)v;
      B.sk_prim[3 * nc + c] = (S)w;
      B.sk_prim[4 * nc + c] = (S)p;
    }
    T km[9];
    for (int m = 0; m < 9; ++m) km[m] = (T)B.sk_metrics[m * nc + c];
    const T ra = spectral_radius<T>(rho, u, v, w, p, gamma, km[0], km[1], km[2]);
    const T rb = spectral_radius<T>(rho, u, v, w, p, gamma, km[3], km[4], km[5]);
    const T rc = spectral_radius<T>(rho, u, v, w, p, gamma, km[6], km[7], km[8]);
    T rva = T(0), rvb = T(0), rvc = T(0);
    const T mu = (T)B.mu[nat];
    if (PAIRS) B.sk_mu[c] = (S)mu;
    T vcoef = T(0);
    if (P.nvis == 1) {
      T vol = (T)B.sk_vol[c];
      if (vol < T(1e-30)) vol = T(1e-30);
      {  // the neighbour factor of visc_spectral_radius (StateUpdater.cpp:194-207)
        T rc = rho;
        if (rc < T(1e-30)) rc = T(1e-30);
        const T rm_vol = rc * vol;
        vcoef = T(2) * mu / (tabs(reynolds) * rm_vol + T(1.0e-30));
      }
      rva = visc_spectral_radius<T>(rho, mu, vol, reynolds, km[0], km[1], km[2]);
      rvb = visc_spectral_radius<T>(rho, mu, vol, reynolds, km[3], km[4], km[5]);
      rvc = visc_spectral_radius<T>(rho, mu, vol, reynolds, km[6], km[7], km[8]);
    }
    const T rad_sum = ra + rb + rc + rva + rvb + rvc;
    const T term = (T(1) / (T)B.dt[nat]) + rad_sum;
    B.sk_coed[c] = (S)(T(1) / term);
    // the point's quantities as a neighbour in compute_flux_splitting (StateUpdater.cpp:217-253)
    {
      T rm = rho, pm = p;
      const T v2 = u * u + v * v + w * w;
      if (rm < T(1e-30)) rm = T(1e-30);
      if (pm < T(1e-30)) pm = T(1e-30);
      const T c2 = gamma * pm / rm;
      const T H = (gamma / (gamma - T(1))) * (pm / rm) + T(0.5) * v2;
      const T af = T(0.5) * (gamma - T(1)) * v2;
      B.sk_nbq[c] = (S)u;
      B.sk_nbq[nc + c] = (S)v;
      B.sk_nbq[2 * nc + c] = (S)w;
      B.sk_nbq[3 * nc + c] = (S)H;
      B.sk_nbq[4 * nc + c] = (S)c2;
      B.sk_nbq[5 * nc + c] = (S)af;
      B.sk_nbq[6 * nc + c] = (S)tsqrt(c2);
      B.sk_nbq[7 * nc + c] = (S)vcoef;
    }
  }
}

// Per face neighbour q of every point: the increment-independent coefficients of
// add_nb / add_nb_contrib (StateUpdater.cpp:326-343, 401-421): spectral radius of
// the neighbour with the point's metric, split eigenvalues l1 (and l4, l5 through
// x1, x2), ct_n, and half the viscous radius.  q = 0..2 lower i,j,k (sign +1),
// q = 3..5 upper (sign -1).
template <typename S, typename T>
__global__ void k_sweep_pairs(const BlockDev<S>* __restrict__ blocks, const Chunk* __restrict__ chunks) {
  const Chunk ch = chunks[blockIdx.x];
  const BlockDev<S> B = blocks[ch.block];
  const ParamsDev& P = B.prm;
  const long long nc = B.ncomp;
  const T gamma = T(P.gamma);
  for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
    const long long c = ch.start + t;
    int nb[6];
    for (int q = 0; q < 6; ++q) nb[q] = B.sk_nb[q * nc + c];
    for (int q = 0; q < 6; ++q) {
      if (nb[q] < 0) continue;
      const long long n = nb[q];
      const int d = q % 3;
      const T nx = (T)B.sk_metrics[(3 * d) * nc + c], ny = (T)B.sk_metrics[(3 * d + 1) * nc + c],
              nz = (T)B.sk_metrics[(3 * d + 2) * nc + c];
      const T rho = (T)B.sk_prim[n], um = (T)B.sk_prim[nc + n], vm = (T)B.sk_prim[2 * nc + n],
              wm = (T)B.sk_prim[3 * nc + n], p = (T)B.sk_prim[4 * nc + n];
      const T r = spectral_radius<T>(rho, um, vm, wm, p, gamma, nx, ny, nz);
      const T sign = q < 3 ? T(1) : T(-1);
      // compute_flux_splitting up to the increment-dependent part
      T rm = rho, pm = p;
      if (rm < T(1e-30)) rm = T(1e-30);
      if (pm < T(1e-30)) pm = T(1e-30);
      const T c2 = gamma * pm / rm;
      const T cm = tsqrt(c2);
      const T ct = nx * um + ny * vm + nz * wm + T(0);
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
      const T ct_n = (ct - T(0)) * inv_mag;
      T rvh = T(0);
      if (P.nvis == 1) {
        T vol_nb = (T)B.sk_vol[n];
        if (vol_nb < T(1e-30)) vol_nb = T(1e-30);
        const T rv = visc_spectral_radius<T>(rho, (T)B.sk_mu[n], vol_nb, T(P.reynolds), nx, ny, nz);
        rvh = T(0.5) * rv;
      }
      S* out = B.sk_pair + (long long)(5 * q) * nc + c;
      out[0] = (S)l1;
      out[nc] = (S)x1;
      out[2 * nc] = (S)x2;
      out[3 * nc] = (S)ct_n;
      out[4 * nc] = (S)rvh;
    }
  }
}

enum SweepMode { SW_LUSGS_FWD = 0, SW_LUSGS_BWD = 1, SW_GS = 2 };

// The cooperative-grid form (ORION_SWEEP_GRID): all four sweeps in one
// persistent cooperative launch, software-pipelined.
// Every CTA walks the hyperplane sequence; for each hyperplane a thread owns at
// most one point of its CTA's first chunk (further chunks are handled in place).
// The point's operands that do not change during the sweep (metrics, diagonal
// coefficient, RHS or its own earlier increment, neighbour indices) are loaded
// before the grid barrier that ends the previous hyperplane, so after the
// barrier one round of independent L2 loads (the neighbours' state and fresh
// increments) precedes the arithmetic.  The barrier's wait is bounded: after
// spin_limit polls the kernel records an error and every CTA returns (the host
// reports ORION_E_TIMEOUT) instead of spinning forever.
struct SweepCtl {
  unsigned int counter;
  int error;
};

__device__ __forceinline__ bool grid_barrier(SweepCtl* ctl, unsigned int target, long long spin_limit) {
  __syncthreads();
  __shared__ int s_abort;
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(&ctl->counter, 1u);
    long long it = 0;
    int abort = 0;
    while (true) {
      const unsigned int v = *(volatile unsigned int*)&ctl->counter;
      if (v >= target) break;
      if (*(volatile int*)&ctl->error) { abort = 1; break; }
      if (++it > spin_limit) {
        atomicExch(&ctl->error, 1);
        abort = 1;
        break;
      }
      __nanosleep(32);
    }
    __threadfence();
    s_abort = abort;
  }
  __syncthreads();
  return s_abort == 0;
}

template <typename T>
struct SweepOps {
  int block;     // -1: no point
  int c;         // compact index
  int nb[6];     // neighbour compact indices: lower i,j,k then upper i,j,k; -1 outside the interior
  T coed;
  T own[5];      // -rhs (forward LU-SGS, GS) or the point's forward increment (backward LU-SGS)
};

template <typename S, typename T, int MODE>
__device__ __forceinline__ void sweep_fetch(const BlockDev<S>& B, int block, int c, SweepOps<T>& o) {
  const long long nc = B.ncomp;
  o.block = block;
  o.c = c;
  for (int q = 0; q < 6; ++q) {
    const bool used = (q < 3) ? (MODE == SW_LUSGS_FWD || MODE == SW_GS) : (MODE == SW_LUSGS_BWD || MODE == SW_GS);
    o.nb[q] = used ? B.sk_nb[q * nc + c] : -1;
  }
  o.coed = (T)B.sk_coed[c];
  for (int m = 0; m < 5; ++m) {
    if (MODE == SW_LUSGS_BWD) o.own[m] = (T)__ldcg(B.sk_dq + m * nc + c);
    else o.own[m] = -(T)B.sk_rhs[m * nc + c];
  }
}

// The increment-dependent part of add_nb / add_nb_contrib for neighbour q
// (compute_flux_splitting from dc on, StateUpdater.cpp:255-264, and the viscous
// off-diagonal term :334-343 / :410-421), accumulated into rhs0 in the
// reference's order.
// The increment-dependent arithmetic of one neighbour term, from its loaded
// operands (dn: neighbour increment; nq: u, v, w, H, c2, af of the neighbour;
// pc: l1, x1, x2, ct_n, rv/2 of the pair; nrm: the point's unit normal).
template <typename T, int MODE>
__device__ __forceinline__ void split_flux(int q, T gm1, int nvis, const T dn[5], const T nq[6], const T pc[5],
                                           const T nrm[3], T fs[5]) {
  const T drm = dn[0], dum = dn[1], dvm = dn[2], dwm = dn[3], dEm = dn[4];
  const T um = nq[0], vm = nq[1], wm = nq[2], H = nq[3], c2 = nq[4], af = nq[5];
  const T nx_n = nrm[0], ny_n = nrm[1], nz_n = nrm[2];
  const T l1 = pc[0], x1 = pc[1], x2 = pc[2], ct_n = pc[3], rvh = pc[4];
  const T dc = ct_n * drm - (nx_n * dum + ny_n * dvm + nz_n * dwm);
  const T dh = af * drm - gm1 * (um * dum + vm * dvm + wm * dwm - dEm);
  const T c2dc = c2 * dc;
  fs[0] = l1 * drm - dh * x1 - dc * x2;
  fs[1] = l1 * dum + (nx_n * c2dc - um * dh) * x1 + (nx_n * dh - um * dc) * x2;
  fs[2] = l1 * dvm + (ny_n * c2dc - vm * dh) * x1 + (ny_n * dh - vm * dc) * x2;
  fs[3] = l1 * dwm + (nz_n * c2dc - wm * dh) * x1 + (nz_n * dh - wm * dc) * x2;
  fs[4] = l1 * dEm + (ct_n * c2dc - H * dh) * x1 + (ct_n * dh - H * dc) * x2;
  const T sgn = q < 3 ? T(1) : T(-1);
  if (nvis == 1) {
    if (MODE == SW_GS) {
      for (int m = 0; m < 5; ++m) fs[m] += rvh * dn[m] * sgn;
    } else {
      for (int m = 0; m < 5; ++m) fs[m] += rvh * dn[m];
    }
  }
}

template <typename T, int MODE>
__device__ __forceinline__ void split_accumulate(int q, const T fs[5], T rhs0[5]) {
  if (MODE == SW_GS && q >= 3) {
    for (int m = 0; m < 5; ++m) rhs0[m] -= fs[m];
  } else {
    for (int m = 0; m < 5; ++m) rhs0[m] += fs[m];
  }
}

template <typename T, int MODE>
__device__ __forceinline__ void split_term(int q, T gm1, int nvis, const T dn[5], const T nq[6], const T pc[5],
                                           const T nrm[3], T rhs0[5]) {
  T fs[5];
  split_flux<T, MODE>(q, gm1, nvis, dn, nq, pc, nrm, fs);
  split_accumulate<T, MODE>(q, fs, rhs0);
}

template <typename S, typename T, int MODE>
__device__ __forceinline__ void sweep_term(const BlockDev<S>& B, T gm1, int nvis, const SweepOps<T>& o, int q,
                                           T rhs0[5]) {
  const long long nc = B.ncomp;
  const long long n = o.nb[q];
  const long long c = o.c;
  const int d = q % 3;
  T dn[5], nq[6], pc[5], nrm[3];
  for (int m = 0; m < 5; ++m) dn[m] = (T)__ldcg(B.sk_dq + m * nc + n);
  for (int k = 0; k < 6; ++k) nq[k] = (T)B.sk_nbq[k * nc + n];
  for (int k = 0; k < 3; ++k) nrm[k] = (T)B.sk_nrm[(3 * d + k) * nc + c];
  for (int k = 0; k < 5; ++k) pc[k] = (T)B.sk_pair[(5 * q + k) * nc + c];
  split_term<T, MODE>(q, gm1, nvis, dn, nq, pc, nrm, rhs0);
}

template <typename S, typename T, int MODE>
__device__ __forceinline__ void sweep_apply(const BlockDev<S>& B, const ParamsDev& P, const SweepOps<T>& o) {
  const long long nc = B.ncomp;
  const T gm1 = T(P.gamma) - T(1);
  T rhs0[5] = {T(0), T(0), T(0), T(0), T(0)};
  // lower neighbours first (i, j, k), then upper (i, j, k): the reference's order
  for (int q = 0; q < 6; ++q)
    if (o.nb[q] >= 0) sweep_term<S, T, MODE>(B, gm1, P.nvis, o, q, rhs0);
  for (int m = 0; m < 5; ++m) {
    S* d = B.sk_dq + m * nc + o.c;
    if (MODE == SW_LUSGS_FWD) *d = (S)((o.own[m] + rhs0[m]) * o.coed);
    else if (MODE == SW_LUSGS_BWD) *d = (S)(o.own[m] - rhs0[m] * o.coed);
    else *d = (S)((rhs0[m] + o.own[m]) * o.coed);
  }
}

// One hyperplane of one sweep for every block; chunks list contiguous compact ranges.
// Launched as a programmatic dependent of the previous hyperplane's launch:
// before griddepcontrol.wait it reads what no earlier hyperplane writes (the
// neighbour indices, the diagonal coefficient, the RHS) and prefetches its
// splitting coefficients into L2, so the launch and those DRAM reads overlap
// the previous hyperplane; after the wait (the previous grid has completed
// and its writes are visible) it reads the neighbours' increments.  It lets
// its own dependent launch only after its wait, so at most one hyperplane
// ahead is resident.
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p)); }

// Threads per SM the per-hyperplane kernel is compiled for (register cap
// 65536 / this): 512 measured fastest on the 64-block 385x257x129 case.
#ifndef ORION_SWEEP_SM_THREADS
#define ORION_SWEEP_SM_THREADS 512
#endif
template <typename S, typename T, int MODE, int NT>
__global__ void __launch_bounds__(NT, ORION_SWEEP_SM_THREADS / NT) k_sweep_plane(const BlockDev<S>* __restrict__ blocks,
                                                    const Chunk* __restrict__ chunks) {
  constexpr int Q0 = MODE == SW_LUSGS_BWD ? 3 : 0;
  constexpr int Q1 = MODE == SW_LUSGS_FWD ? 3 : 6;
  constexpr bool PRELOAD = sizeof(T) == 4;  // FP32: every static operand in registers before the wait
  const Chunk ch = chunks[blockIdx.x];
  const bool active = (int)threadIdx.x < ch.count;
  const BlockDev<S>& B = blocks[ch.block];
  // the case's parameters, from the block's own descriptor: loaded with its
  // other fields and used only after the wait.  Work before the wait beyond
  // issuing loads lengthens the chain: it competes with the previous
  // hyperplane's launch, which is still running on the same SMs (forming a GS
  // pass's stale-side terms there, or even gamma - 1, made the step slower).
  const double gamma_ld = B.prm.gamma;
  const int nvis = B.prm.nvis;
  const long long nc = B.ncomp;
  const int c = (int)ch.start + threadIdx.x;
  // pointers into registers now: griddepcontrol.wait clobbers memory, so
  // anything read through B after it would be reloaded from global memory
  S* const skdq = B.sk_dq;
  const S* const sknbq = B.sk_nbq;
  const S* const skpair = B.sk_pair;
  const S* const sknrm = B.sk_nrm;
  int nb[6];
  T coed = T(0), own[5];
  T nq[6][6], pc[6][5], nrm[3][3];
  if (active) {
#pragma unroll
    for (int q = Q0; q < Q1; ++q) nb[q] = B.sk_nb[q * nc + c];
    coed = (T)B.sk_coed[c];
    if (MODE != SW_LUSGS_BWD)
#pragma unroll
      for (int m = 0; m < 5; ++m) own[m] = -(T)B.sk_rhs[m * nc + c];
#pragma unroll
    for (int q = Q0; q < Q1; ++q) {
      if (nb[q] < 0) continue;
      if (PRELOAD) {
#pragma unroll
        for (int k = 0; k < 6; ++k) nq[q][k] = (T)B.sk_nbq[k * nc + nb[q]];
#pragma unroll
        for (int k = 0; k < 5; ++k) pc[q][k] = (T)B.sk_pair[(5 * q + k) * nc + c];
      } else {
        for (int k = 0; k < 5; ++k) prefetch_l2(B.sk_pair + (long long)(5 * q + k) * nc + c);
        for (int k = 0; k < 6; ++k) prefetch_l2(B.sk_nbq + (long long)k * nc + nb[q]);
      }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (PRELOAD) {
#pragma unroll
        for (int k = 0; k < 3; ++k) nrm[d][k] = (T)B.sk_nrm[(3 * d + k) * nc + c];
      } else {
        for (int k = 0; k < 3; ++k) prefetch_l2(B.sk_nrm + (long long)(3 * d + k) * nc + c);
      }
    }
  }
  grid_dep_wait();
  grid_dep_launch();
  if (!active) return;
  if (MODE == SW_LUSGS_BWD)  // the forward increment: the launch just before may have written it
#pragma unroll
    for (int m = 0; m < 5; ++m) own[m] = (T)__ldcg(skdq + m * nc + c);
  // every neighbour increment in flight at once
  T dn[6][5];
#pragma unroll
  for (int q = Q0; q < Q1; ++q)
    if (nb[q] >= 0)
#pragma unroll
      for (int m = 0; m < 5; ++m) dn[q][m] = (T)__ldcg(skdq + m * nc + nb[q]);
  const T gm1 = T(gamma_ld) - T(1);
  T rhs0[5] = {T(0), T(0), T(0), T(0), T(0)};
  // lower neighbours first (i, j, k), then upper (i, j, k): the reference's order
#pragma unroll
  for (int q = Q0; q < Q1; ++q) {
    if (nb[q] < 0) continue;
    const int d = q % 3;
    if (!PRELOAD) {
      for (int k = 0; k < 6; ++k) nq[q][k] = (T)sknbq[k * nc + nb[q]];
      for (int k = 0; k < 5; ++k) pc[q][k] = (T)skpair[(5 * q + k) * nc + c];
      for (int k = 0; k < 3; ++k) nrm[d][k] = (T)sknrm[(3 * d + k) * nc + c];
    }
    split_term<T, MODE>(q, gm1, nvis, dn[q], nq[q], pc[q], nrm[d], rhs0);
  }
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    S* dst = skdq + m * nc + c;
    if (MODE == SW_LUSGS_FWD) *dst = (S)((own[m] + rhs0[m]) * coed);
    else if (MODE == SW_LUSGS_BWD) *dst = (S)(own[m] - rhs0[m] * coed);
    else *dst = (S)((rhs0[m] + own[m]) * coed);
  }
}

template <typename S, typename T, int MODE>
__device__ __forceinline__ bool persistent_pass(const BlockDev<S>* __restrict__ blocks, const Chunk* __restrict__ chunks,
                                                const int* __restrict__ off, int nlaunch, const ParamsDev& P,
                                                SweepCtl* ctl, unsigned int& target, long long spin_limit) {
  SweepOps<T> cur;
  cur.block = -1;
  // prefetch hyperplane 0
  {
    const int ci = off[0] + blockIdx.x;
    if (ci < off[1]) {
      const Chunk ch = chunks[ci];
      if ((int)threadIdx.x < ch.count)
        sweep_fetch<S, T, MODE>(blocks[ch.block], ch.block, (int)ch.start + threadIdx.x, cur);
    }
  }
  for (int t = 0; t < nlaunch; ++t) {
    if (cur.block >= 0) sweep_apply<S, T, MODE>(blocks[cur.block], P, cur);
    // further chunks of this hyperplane owned by this CTA (large hyperplanes only)
    for (int ci = off[t] + blockIdx.x + gridDim.x; ci < off[t + 1]; ci += gridDim.x) {
      const Chunk ch = chunks[ci];
      if ((int)threadIdx.x < ch.count) {
        SweepOps<T> x;
        sweep_fetch<S, T, MODE>(blocks[ch.block], ch.block, (int)ch.start + threadIdx.x, x);
        sweep_apply<S, T, MODE>(blocks[ch.block], P, x);
      }
    }
    // prefetch the next hyperplane's static operands, then wait for this one
    cur.block = -1;
    if (t + 1 < nlaunch) {
      const int ci = off[t + 1] + blockIdx.x;
      if (ci < off[t + 2]) {
        const Chunk ch = chunks[ci];
        if ((int)threadIdx.x < ch.count)
          sweep_fetch<S, T, MODE>(blocks[ch.block], ch.block, (int)ch.start + threadIdx.x, cur);
      }
    }
    target += gridDim.x;
    if (!grid_barrier(ctl, target, spin_limit)) return false;
  }
  return true;
}

template <typename S, typename T, int NT>
__global__ void __launch_bounds__(NT) k_sweeps_persistent(const BlockDev<S>* __restrict__ blocks,
                                                           const Chunk* __restrict__ fwd_chunks,
                                                           const int* __restrict__ fwd_off,
                                                           const Chunk* __restrict__ bwd_chunks,
                                                           const int* __restrict__ bwd_off, int nlaunch,
                                                           ParamsDev P, SweepCtl* ctl, long long spin_limit) {
  unsigned int target = 0;
  if (!persistent_pass<S, T, SW_LUSGS_FWD>(blocks, fwd_chunks, fwd_off, nlaunch, P, ctl, target, spin_limit)) return;
  if (!persistent_pass<S, T, SW_LUSGS_BWD>(blocks, bwd_chunks, bwd_off, nlaunch, P, ctl, target, spin_limit)) return;
  if (!persistent_pass<S, T, SW_GS>(blocks, fwd_chunks, fwd_off, nlaunch, P, ctl, target, spin_limit)) return;
  persistent_pass<S, T, SW_GS>(blocks, bwd_chunks, bwd_off, nlaunch, P, ctl, target, spin_limit);
}

// Cluster form of the four sweeps.  Mesh blocks are independent, so only the
// CTAs that share a block have to agree on hyperplane boundaries: each thread
// block cluster owns a group of mesh blocks and walks the hyperplanes of that
// group, separating consecutive hyperplanes with the hardware cluster barrier
// (release/acquire at cluster scope).  No cluster waits on another, so clusters
// may also run one after another.  Software-pipelined like the persistent form.
__device__ __forceinline__ void cluster_arrive() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n" ::: "memory");
}
__device__ __forceinline__ void cluster_wait() {
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}

// The fields of a block the sweeps touch, staged in shared memory so no
// hyperplane pays a global load for a pointer.
template <typename S>
struct SweepBlock {
  S* dq;
  const int* nb;
  const S* coed;
  const S* rhs;
  const S* nbq;
  const S* pair;
  const S* nrm;
  long long nc;
};

// A thread's share of one hyperplane: up to two chunks, staged per pass.
struct SweepSlot {
  int block;  // -1: none
  int start;
  int count;
};

// Static operands of point c: neighbour indices, diagonal coefficient and the
// RHS (or, backward, the forward increment) into registers; the splitting
// coefficients, neighbour states and normals prefetched to L2, so that after
// the barrier only the neighbours' fresh increments miss.
template <typename S, typename T, int MODE>
__device__ __forceinline__ void cl_fetch(const SweepBlock<S>& B, int block, int c, SweepOps<T>& o) {
  const long long nc = B.nc;
  o.block = block;
  o.c = c;
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    const bool used = (q < 3) ? (MODE == SW_LUSGS_FWD || MODE == SW_GS) : (MODE == SW_LUSGS_BWD || MODE == SW_GS);
    o.nb[q] = used ? __ldg(B.nb + q * nc + c) : -1;
  }
  o.coed = (T)B.coed[c];
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    if (MODE == SW_LUSGS_BWD) o.own[m] = (T)__ldcg(B.dq + m * nc + c);
    else o.own[m] = -(T)B.rhs[m * nc + c];
  }
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    if (o.nb[q] < 0) continue;
    for (int k = 0; k < 5; ++k) prefetch_l2(B.pair + (long long)(5 * q + k) * nc + c);
    for (int k = 0; k < 6; ++k) prefetch_l2(B.nbq + (long long)k * nc + o.nb[q]);
  }
  for (int k = 0; k < 9; ++k) prefetch_l2(B.nrm + (long long)k * nc + c);
}

// Every neighbour's increment in flight at once, then the terms in the
// reference's order (split_term: the same arithmetic as the other forms).
template <typename S, typename T, int MODE>
__device__ __forceinline__ void cl_apply(const SweepBlock<S>& B, T gm1, int nvis, const SweepOps<T>& o) {
  const long long nc = B.nc;
  const long long c = o.c;
  T dn[6][5];
#pragma unroll
  for (int q = 0; q < 6; ++q)
    if (o.nb[q] >= 0)
#pragma unroll
      for (int m = 0; m < 5; ++m) dn[q][m] = (T)__ldcg(B.dq + m * nc + o.nb[q]);
  T rhs0[5] = {T(0), T(0), T(0), T(0), T(0)};
#pragma unroll
  for (int q = 0; q < 6; ++q) {
    if (o.nb[q] < 0) continue;
    const int d = q % 3;
    T nq[6], pc[5], nrm[3];
    for (int k = 0; k < 6; ++k) nq[k] = (T)B.nbq[k * nc + o.nb[q]];
    for (int k = 0; k < 5; ++k) pc[k] = (T)B.pair[(5 * q + k) * nc + c];
    for (int k = 0; k < 3; ++k) nrm[k] = (T)B.nrm[(3 * d + k) * nc + c];
    split_term<T, MODE>(q, gm1, nvis, dn[q], nq, pc, nrm, rhs0);
  }
#pragma unroll
  for (int m = 0; m < 5; ++m) {
    S* d = B.dq + m * nc + c;
    if (MODE == SW_LUSGS_FWD) *d = (S)((o.own[m] + rhs0[m]) * o.coed);
    else if (MODE == SW_LUSGS_BWD) *d = (S)(o.own[m] - rhs0[m] * o.coed);
    else *d = (S)((rhs0[m] + o.own[m]) * o.coed);
  }
}

template <typename S, typename T, int MODE>
__device__ __forceinline__ void cluster_pass(const SweepBlock<S>* sb, const Chunk* __restrict__ chunks,
                                             const int* __restrict__ off, int nlaunch, int rank, int csize,
                                             const ParamsDev& P, SweepSlot* slots) {
  const T gm1 = T(P.gamma) - T(1);
  // stage this CTA's chunk of every hyperplane (two per hyperplane)
  __syncthreads();
  for (int x = threadIdx.x; x < 2 * nlaunch; x += blockDim.x) {
    const int t = x >> 1, r = x & 1;
    const int ci = off[t] + rank + r * csize;
    SweepSlot sl{-1, 0, 0};
    if (ci < off[t + 1]) {
      const Chunk ch = chunks[ci];
      sl = SweepSlot{ch.block, (int)ch.start, ch.count};
    }
    slots[x] = sl;
  }
  __syncthreads();
  SweepOps<T> cur[2];
  auto fetch = [&](int t) {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const SweepSlot sl = slots[2 * t + r];
      cur[r].block = -1;
      if (sl.block >= 0 && (int)threadIdx.x < sl.count)
        cl_fetch<S, T, MODE>(sb[sl.block], sl.block, sl.start + threadIdx.x, cur[r]);
    }
  };
  fetch(0);
  for (int t = 0; t < nlaunch; ++t) {
#pragma unroll
    for (int r = 0; r < 2; ++r)
      if (cur[r].block >= 0) cl_apply<S, T, MODE>(sb[cur[r].block], gm1, P.nvis, cur[r]);
    // chunks beyond the two staged ones (very large hyperplanes only)
    for (int ci = off[t] + rank + 2 * csize; ci < off[t + 1]; ci += csize) {
      const Chunk ch = chunks[ci];
      if ((int)threadIdx.x < ch.count) {
        SweepOps<T> x;
        cl_fetch<S, T, MODE>(sb[ch.block], ch.block, (int)ch.start + threadIdx.x, x);
        cl_apply<S, T, MODE>(sb[ch.block], gm1, P.nvis, x);
      }
    }
    // publish this hyperplane, fetch the next one's static operands, then wait
    cluster_arrive();
    if (t + 1 < nlaunch) fetch(t + 1);
    cluster_wait();
  }
}

template <typename S, typename T, int NT>
__global__ void __launch_bounds__(NT, 1) k_sweeps_cluster(const BlockDev<S>* __restrict__ blocks, int nblocks,
                                                          const Chunk* __restrict__ fwd_chunks,
                                                          const int* __restrict__ fwd_off,
                                                          const Chunk* __restrict__ bwd_chunks,
                                                          const int* __restrict__ bwd_off,
                                                          const int* __restrict__ grp_base,
                                                          const int* __restrict__ grp_nplanes, ParamsDev P) {
  namespace cg = cooperative_groups;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SweepBlock<S>* sb = reinterpret_cast<SweepBlock<S>*>(smem_raw);
  SweepSlot* slots = reinterpret_cast<SweepSlot*>(smem_raw + sizeof(SweepBlock<S>) * nblocks);
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
    const BlockDev<S>& B = blocks[b];
    sb[b] = SweepBlock<S>{B.sk_dq, B.sk_nb, B.sk_coed, B.sk_rhs, B.sk_nbq, B.sk_pair, B.sk_nrm, B.ncomp};
  }
  cg::cluster_group cl = cg::this_cluster();
  const int csize = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const int g = blockIdx.x / csize;
  const int base = grp_base[g], n = grp_nplanes[g];
  cluster_pass<S, T, SW_LUSGS_FWD>(sb, fwd_chunks, fwd_off + base, n, rank, csize, P, slots);
  cluster_pass<S, T, SW_LUSGS_BWD>(sb, bwd_chunks, bwd_off + base, n, rank, csize, P, slots);
  cluster_pass<S, T, SW_GS>(sb, fwd_chunks, fwd_off + base, n, rank, csize, P, slots);
  cluster_pass<S, T, SW_GS>(sb, bwd_chunks, bwd_off + base, n, rank, csize, P, slots);
}

// Finish, per interior point in natural order: zero the physical-BC windows
// (set_boundary_dq_zero), bring the swept increment back to the natural
// layout, limited update (update_limited) and, when DO_RES, the residual
// partials (ResidualMonitor::compute).
template <typename S>
__device__ __forceinline__ void limited_update(const BlockDev<S>& B, const ParamsDev& P, long long idx,
                                               const double dq[5]);
__device__ __forceinline__ void res_combine(double& sum, double& mx, long long& key, double osum, double omx,
                                            long long okey);
template <int NT>
__device__ __forceinline__ void block_reduce_res(double& sum, double& mx, long long& key);

// CTAs per SM the finish kernel is compiled for (register cap 65536 / (NT n)):
// on C3 four (64 registers, a few spilled) took the update stage from 7.43 to
// 7.04 ms mixed and 11.93 to 11.54 ms plain against no cap (105 registers).
#ifndef ORION_FINISH_MINB
#define ORION_FINISH_MINB 4
#endif
template <typename S, bool DO_RES, int NT>
__global__ void __launch_bounds__(NT, ORION_FINISH_MINB) k_sweep_finish(const BlockDev<S>* __restrict__ blocks,
                                                     const Chunk* __restrict__ chunks, ResPartial* __restrict__ partials) {
  // Natural order (interior index n = i + ni*(j + nj*k)): prim, dq, vol, dt
  // and the mask are read and written coalesced; only the swept increment is
  // gathered from the plane-major layout, at c = koff[s*nk + k] + (j - jlo(s,k)).
  const Chunk ch = chunks[blockIdx.x];
  const BlockDev<S> B = blocks[ch.block];
  const ParamsDev& P = B.prm;
  const long long np = B.npad, nc = B.ncomp;
  double sum = 0.0, mx = -1.0;
  long long key = (long long)0x7fffffffffffffffLL;
  for (int t = threadIdx.x; t < ch.count; t += NT) {
    const long long n = ch.start + t;
    const int n32 = (int)n, r32 = n32 / B.ni;
    const int ii = n32 - r32 * B.ni, jj = r32 % B.nj, kk = r32 / B.nj;
    const long long idx = lin(B, NG + ii, NG + jj, NG + kk);
    const int sp = ii + jj + kk;
    const int jlo = sp - kk - (B.ni - 1) > 0 ? sp - kk - (B.ni - 1) : 0;
    const long long c = (long long)__ldg(B.koff + (long long)sp * B.nk + kk) + (jj - jlo);
    double dq[5];
    const bool masked = B.bcmask[idx] != 0;
    for (int m = 0; m < 5; ++m) {
      const S v = masked ? (S)0 : __ldcs(B.sk_dq + m * nc + c);
      B.dq[m * np + idx] = v;
      dq[m] = (double)v;
    }
    limited_update(B, P, idx, dq);
    if (DO_RES) {
      double vol = B.vol[idx];
      double dt = (double)B.dt[idx];
      if (vol < 1e-30) vol = 1e-30;
      if (dt < 1e-30) dt = 1e-30;
      const double inv_factor = 1.0 / (dt * vol);
      const long long kbase = (B.int_base + n) * 5;
      for (int m = 0; m < 5; ++m) {
        const double res = fabs(dq[m]) * inv_factor;
        sum += res * res;
        if (res > mx || (res == mx && kbase + m < key)) {
          mx = res;
          key = kbase + m;
        }
      }
    }
  }
  if (DO_RES) {
    block_reduce_res<NT>(sum, mx, key);
    if (threadIdx.x == 0) partials[blockIdx.x] = ResPartial{sum, mx, key};
  }
}

// ===========================================================================
// Final update: set_boundary_dq_zero + update_limited (StateUpdater.cpp:447-542),
// optionally fused with the residual (ResidualMonitor::compute,
// src/solver/ResidualMonitor.cpp:11-137): per-CTA partial sums and maxima with
// the lexicographic location key; a single CTA combines them in fixed order.
// ===========================================================================
template <typename S>
__device__ __forceinline__ void limited_update(const BlockDev<S>& B, const ParamsDev& P, long long idx,
                                               const double dq[5]) {
  const long long np = B.npad;
  const double gm1 = P.gamma - 1.0;
  const double r = B.prim[idx], u = B.prim[np + idx], v = B.prim[2 * np + idx], w = B.prim[3 * np + idx],
               p = B.prim[4 * np + idx];
  const double E = p / gm1 + 0.5 * r * (u * u + v * v + w * w);
  double qn[5];
  qn[0] = r + dq[0];
  qn[1] = r * u + dq[1];
  qn[2] = r * v + dq[2];
  qn[3] = r * w + dq[3];
  qn[4] = E + dq[4];
  double r_n = qn[0];
  double inv_r = 1.0 / r_n;
  const double a = qn[1] * inv_r, b = qn[2] * inv_r, c = qn[3] * inv_r;
  const double p_n = gm1 * (qn[4] - 0.5 * r_n * (a * a + b * b + c * c));
  const double dp_p = fabs((p_n - p) / p);
  const double term = tmax(0.0, -0.3 + dp_p);
  const double Fa = 1.0 / (1.0 + 2.0 * term);
  double qf[5];
  qf[0] = r + dq[0] * Fa;
  qf[1] = r * u + dq[1] * Fa;
  qf[2] = r * v + dq[2] * Fa;
  qf[3] = r * w + dq[3] * Fa;
  qf[4] = E + dq[4] * Fa;
  r_n = qf[0];
  inv_r = 1.0 / r_n;
  const double u_n = qf[1] * inv_r, v_n = qf[2] * inv_r, w_n = qf[3] * inv_r;
  const double p_nf = gm1 * (qf[4] - 0.5 * r_n * (u_n * u_n + v_n * v_n + w_n * w_n));
  if (!(r_n <= 1e-6 || p_nf <= 1e-6)) {
    B.prim[idx] = r_n;
    B.prim[np + idx] = u_n;
    B.prim[2 * np + idx] = v_n;
    B.prim[3 * np + idx] = w_n;
    B.prim[4 * np + idx] = p_nf;
  }
}

__device__ __forceinline__ void res_combine(double& sum, double& mx, long long& key, double osum, double omx,
                                            long long okey) {
  sum += osum;
  if (omx > mx || (omx == mx && okey < key)) {
    mx = omx;
    key = okey;
  }
}

template <int NT>
__device__ __forceinline__ void block_reduce_res(double& sum, double& mx, long long& key) {
  // warp then CTA tree, fixed shape => deterministic
  for (int off = 16; off > 0; off >>= 1) {
    const double os = __shfl_down_sync(0xffffffffu, sum, off);
    const double om = __shfl_down_sync(0xffffffffu, mx, off);
    const long long ok = __shfl_down_sync(0xffffffffu, key, off);
    res_combine(sum, mx, key, os, om, ok);
  }
  __shared__ double s_sum[NT / 32];
  __shared__ double s_max[NT / 32];
  __shared__ long long s_key[NT / 32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    s_sum[w] = sum;
    s_max[w] = mx;
    s_key[w] = key;
  }
  __syncthreads();
  if (w == 0) {
    sum = (l < NT / 32) ? s_sum[l] : 0.0;
    mx = (l < NT / 32) ? s_max[l] : -1.0;
    key = (l < NT / 32) ? s_key[l] : (long long)0x7fffffffffffffffLL;
    for (int off = 16; off > 0; off >>= 1) {
      const double os = __shfl_down_sync(0xffffffffu, sum, off);
      const double om = __shfl_down_sync(0xffffffffu, mx, off);
      const long long ok = __shfl_down_sync(0xffffffffu, key, off);
      res_combine(sum, mx, key, os, om, ok);
    }
  }
}

template <typename S, bool DO_UPDATE, bool DO_RES, int NT>
__global__ void __launch_bounds__(NT) k_update_res(const BlockDev<S>* __restrict__ blocks, const Chunk* __restrict__ chunks,
                                                    ResPartial* __restrict__ partials) {
  const Chunk ch = chunks[blockIdx.x];
  const BlockDev<S> B = blocks[ch.block];
  const ParamsDev& P = B.prm;
  const long long np = B.npad;
  double sum = 0.0, mx = -1.0;
  long long key = (long long)0x7fffffffffffffffLL;
  for (int t = threadIdx.x; t < ch.count; t += NT) {
    const long long n = ch.start + t;
    const int n32 = (int)n, r32 = n32 / B.ni;
    const int ii = n32 - r32 * B.ni, jj = r32 % B.nj, kk = r32 / B.nj;
    const long long idx = lin(B, NG + ii, NG + jj, NG + kk);
    double dq[5];
    if (DO_UPDATE && B.bcmask[idx]) {
      for (int m = 0; m < 5; ++m) {
        B.dq[m * np + idx] = (S)0;
        dq[m] = 0.0;
      }
    } else {
      for (int m = 0; m < 5; ++m) dq[m] = (double)B.dq[m * np + idx];
    }
    if (DO_UPDATE) limited_update(B, P, idx, dq);
    if (DO_RES) {
      double vol = B.vol[idx];
      double dt = (double)B.dt[idx];
      if (vol < 1e-30) vol = 1e-30;
      if (dt < 1e-30) dt = 1e-30;
      const double inv_factor = 1.0 / (dt * vol);
      const long long kbase = (B.int_base + n) * 5;
      for (int m = 0; m < 5; ++m) {
        const double res = fabs(dq[m]) * inv_factor;
        sum += res * res;
        if (res > mx || (res == mx && kbase + m < key)) {
          mx = res;
          key = kbase + m;
        }
      }
    }
  }
  if (DO_RES) {
    block_reduce_res<NT>(sum, mx, key);
    if (threadIdx.x == 0) partials[blockIdx.x] = ResPartial{sum, mx, key};
  }
}

template <typename S>
__device__ __forceinline__ void res_final_body(const BlockDev<S>* __restrict__ blocks, int nblocks,
                                               const ResPartial* __restrict__ partials, int npart,
                                               long long total_points, const unsigned long long* dtmin_bits,
                                               ResidualOut* __restrict__ hist, int* __restrict__ counter,
                                               int capacity, ResPartial* __restrict__ total);

template <typename S>
__global__ void __launch_bounds__(1024) k_res_final(const BlockDev<S>* __restrict__ blocks, int nblocks,
                                                     const ResPartial* __restrict__ partials, int npart,
                                                     long long total_points, const unsigned long long* dtmin_bits,
                                                     ResidualOut* __restrict__ hist, int* __restrict__ counter,
                                                     int capacity, ResPartial* __restrict__ total) {
  res_final_body<S>(blocks, nblocks, partials, npart, total_points, dtmin_bits, hist, counter, capacity, total);
}

// One CTA per case of a group: that case's minimum time step (dt_part) or
// residual statistics (partials) over its own range, in the same order as
// the case's own launches, into the case's own result slots.
static __global__ void __launch_bounds__(1024) k_dtmin_group(const GroupMember* __restrict__ members,
                                                             const double* __restrict__ dt_part) {
  const GroupMember& m = members[blockIdx.x];
  dtmin_final_body(dt_part + m.pad_off, m.pad_n, m.dtmin);
}

template <typename S>
__global__ void __launch_bounds__(1024) k_res_final_group(const GroupMember* __restrict__ members,
                                                           const ResPartial* __restrict__ partials, int capacity) {
  const GroupMember& m = members[blockIdx.x];
  res_final_body<S>(static_cast<const BlockDev<S>*>(m.blocks), m.nblocks, partials + m.part_off, m.part_n,
                    m.total_points, m.dtmin, m.hist, m.counter, capacity, m.total);
}

template <typename S>
__device__ __forceinline__ void res_final_body(const BlockDev<S>* __restrict__ blocks, int nblocks,
                                               const ResPartial* __restrict__ partials, int npart,
                                               long long total_points, const unsigned long long* dtmin_bits,
                                               ResidualOut* __restrict__ hist, int* __restrict__ counter,
                                               int capacity, ResPartial* __restrict__ total) {
  double sum = 0.0, mx = -1.0;
  long long key = (long long)0x7fffffffffffffffLL;
  for (int t = threadIdx.x; t < npart; t += 1024) {
    const ResPartial p = partials[t];
    res_combine(sum, mx, key, p.sum, p.max, p.key);
  }
  block_reduce_res<1024>(sum, mx, key);
  if (threadIdx.x == 0) {
    if (total) *total = ResPartial{sum, mx, key};
    ResidualOut r;
    r.rms = total_points > 0 ? sqrt(sum / (double)total_points) : 0.0;
    r.max = mx;
    const long long pt = key / 5;
    int b = 0;
    for (int q = 0; q < nblocks; ++q) {
      const BlockDev<S>& B = blocks[q];
      if (pt >= B.int_base && pt < B.int_base + (long long)B.ni * B.nj * B.nk) b = q;
    }
    const BlockDev<S>& B = blocks[b];
    const long long n = pt - B.int_base;
    r.loc[0] = b;
    r.loc[1] = (int)(n % B.ni) + 1;
    r.loc[2] = (int)((n / B.ni) % B.nj) + 1;
    r.loc[3] = (int)(n / ((long long)B.ni * B.nj)) + 1;
    r.loc[4] = (int)(key % 5) + 1;
    r.pad = 0;
    r.phydtime = __longlong_as_double((long long)*dtmin_bits);
    const int c = *counter;
    hist[c % capacity] = r;
    *counter = c + 1;
  }
}

// ===========================================================================
// Initial flow on the device: freestream + splitmix64 noise + EOS temperature
// (initialize_flow / update_temperature, src/preprocess/InitialCondition.cpp:7-147).
// ===========================================================================
__device__ __forceinline__ double splitmix_uniform(unsigned long long seed, unsigned long long n) {
  unsigned long long z = seed + n * 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z = z ^ (z >> 31);
  return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

template <typename S>
__global__ void k_init_flow(const BlockDev<S>* __restrict__ blocks, const Chunk* __restrict__ chunks,
                            const long long* __restrict__ pad_base, unsigned long long seed, double amp) {
  const Chunk ch = chunks[blockIdx.x];
  const BlockDev<S> B = blocks[ch.block];
  const ParamsDev& P = B.prm;
  const long long np = B.npad;
  for (int t = threadIdx.x; t < ch.count; t += blockDim.x) {
    const long long idx = ch.start + t;
    const unsigned long long n = (unsigned long long)(pad_base[ch.block] + idx);
    double rho = P.roo, u = P.uoo;
    if (amp != 0.0) {
      const double r1 = splitmix_uniform(seed, 2 * n + 1);
      const double r2 = splitmix_uniform(seed, 2 * n + 2);
      rho = rho * (1.0 + amp * (2.0 * r1 - 1.0));
      u = u * (1.0 + amp * (2.0 * r2 - 1.0));
    }
    const double p = P.poo;
    B.prim[idx] = rho;
    B.prim[np + idx] = u;
    B.prim[2 * np + idx] = P.voo;
    B.prim[3 * np + idx] = P.woo;
    B.prim[4 * np + idx] = p;
    double T = P.too;
    if (P.nvis == 1) {
      double r = rho;
      if (r < 1.0e-30) r = 1.0e-30;
      const double a2 = P.gamma * p / r;
      T = (P.moo * P.moo) * a2;
    }
    B.prim[5 * np + idx] = T;
    B.q[idx] = P.roo;
    B.q[np + idx] = P.roo * P.uoo;
    B.q[2 * np + idx] = P.roo * P.voo;
    B.q[3 * np + idx] = P.roo * P.woo;
    const double v2 = P.uoo * P.uoo + P.voo * P.voo + P.woo * P.woo;
    B.q[4 * np + idx] = P.poo / (P.gamma - 1.0) + 0.5 * P.roo * v2;
    for (int m = 0; m < 5; ++m) B.dq[m * np + idx] = (S)0;
  }
}

}  // namespace orion
