// Solution output fields of one block (write_block_vts_binary,
// src/postprocess/PostProcess.cpp:116-243): density, pressure, temperature,
// Mach and velocity at the interior points, i fastest, as Float32.  Mach is
// formed in FP64 in the reference's order and then rounded, like the
// reference; compiled in the strict FP64 translation unit.
#pragma once
#include <cuda_runtime.h>

namespace orion {
namespace out {

// dst: 7 arrays of n floats: rho, p, T, Mach, u, v, w.
__global__ void k_pack_output(const double* __restrict__ prim, long long np, int ni, int nj, int nk, int nx, int ny,
                              double gamma, float* __restrict__ dst) {
  const long long n = (long long)ni * nj * nk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(t % ni), r = (int)(t / ni);
    const int j = r % nj, k = r / nj;
    const long long idx = (i + 3) + (long long)nx * ((j + 3) + (long long)ny * (k + 3));
    const double rho = prim[idx], u = prim[np + idx], v = prim[2 * np + idx], w = prim[3 * np + idx],
                 p = prim[4 * np + idx], T = prim[5 * np + idx];
    const double v2 = u * u + v * v + w * w;
    const double c2 = gamma * p / rho;
    const double mach = (c2 > 1e-30) ? sqrt(v2 / c2) : 0.0;
    dst[t] = (float)rho;
    dst[n + t] = (float)p;
    dst[2 * n + t] = (float)T;
    dst[3 * n + t] = (float)mach;
    dst[4 * n + t] = (float)u;
    dst[5 * n + t] = (float)v;
    dst[6 * n + t] = (float)w;
  }
}

}  // namespace out
}  // namespace orion
