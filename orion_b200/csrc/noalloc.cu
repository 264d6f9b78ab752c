// Residual norm of one block without any device allocation.
//
// Some callers cannot call cudaMalloc at the point where they need a residual:
// a host solver that reserves its whole device-memory budget at start-up and
// hands out nothing afterwards, a time loop running inside another framework's
// stream-ordered pool, or a driver that must not let an allocation synchronize
// the device between two kernels of a step.  orion_residual_block_noalloc
// serves them: the caller passes the block's fields and receives the
// statistics, and the only scratch the reduction needs (one partial per CTA
// and the final result) lives in a fixed-size array in this file's device
// memory, which every GPU that loads the library holds until the process exits.
#include <cuda_runtime.h>

#include <string>

#include "kernels.cuh"
#include "orion_gpu.h"

namespace orion {
int set_error(int code, const std::string& msg);  // orion_last_error() reports it
}

using namespace orion;

namespace {

constexpr int kNaThreads = 256;
constexpr int kNaChunk = 1024;  // interior points per CTA
constexpr int kNaMaxPartials = ORION_NOALLOC_MAX_POINTS / kNaChunk;

struct NoAllocScratch {
  ResPartial partial[kNaMaxPartials];
  ResidualOut result;
};

}  // namespace

// Shared by every call on a device: partials are fully rewritten by each call
// before they are read, the result slot likewise.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

namespace {

// Per-CTA partial sums and maxima of |dq| / (dt * vol) over a chunk of interior
// points (the arithmetic of ResidualMonitor::compute, src/solver/ResidualMonitor.cpp:11-137).
__global__ void __launch_bounds__(kNaThreads) k_noalloc_partials(const double* __restrict__ dq,
                                                                 const double* __restrict__ vol,
                                                                 const double* __restrict__ dt, int ni, int nj,
                                                                 int nk, NoAllocScratch* __restrict__ scr) {
  const int nx = ni + 2 * NG, ny = nj + 2 * NG, nz = nk + 2 * NG;
  const long long np = (long long)nx * ny * nz;
  const long long ntot = (long long)ni * nj * nk;
  const long long start = (long long)blockIdx.x * kNaChunk;
  double sum = 0.0, mx = -1.0;
  long long key = (long long)0x7fffffffffffffffLL;
  for (int t = threadIdx.x; t < kNaChunk; t += kNaThreads) {
    const long long n = start + t;
    if (n >= ntot) break;
    const int ii = (int)(n % ni), jj = (int)((n / ni) % nj), kk = (int)(n / ((long long)ni * nj));
    const long long idx = (long long)(ii + NG) + (long long)nx * ((jj + NG) + (long long)ny * (kk + NG));
    double v = vol[idx];
    double d = dt[idx];
    if (v < 1e-30) v = 1e-30;
    if (d < 1e-30) d = 1e-30;
    const double inv_factor = 1.0 / (d * v);
    for (int m = 0; m < 5; ++m) {
      const double res = fabs(dq[m * np + idx]) * inv_factor;
      sum += res * res;
      if (res > mx || (res == mx && n * 5 + m < key)) {
        mx = res;
        key = n * 5 + m;
      }
    }
  }
  block_reduce_res<kNaThreads>(sum, mx, key);
  if (threadIdx.x == 0) scr->partial[blockIdx.x] = ResPartial{sum, mx, key};
}

__global__ void __launch_bounds__(1024) k_noalloc_final(NoAllocScratch* __restrict__ scr, int npart, int ni, int nj) {
  double sum = 0.0, mx = -1.0;
  long long key = (long long)0x7fffffffffffffffLL;
  for (int t = threadIdx.x; t < npart; t += 1024) {
    const ResPartial p = scr->partial[t];
    res_combine(sum, mx, key, p.sum, p.max, p.key);
  }
  block_reduce_res<1024>(sum, mx, key);
  if (threadIdx.x == 0) {
    ResidualOut r;
    r.max = mx;
    r.rms = sum;  // sum of squares; the host divides by the point count
    const long long pt = key / 5;
    r.loc[0] = 0;
    r.loc[1] = (int)(pt % ni) + 1;
    r.loc[2] = (int)((pt / ni) % nj) + 1;
    r.loc[3] = (int)(pt / ((long long)ni * nj)) + 1;
    r.loc[4] = (int)(key % 5) + 1;
    r.pad = 0;
    r.phydtime = 0.0;
    scr->result = r;
  }
}

int na_fail(int code, const std::string& msg) { return orion::set_error(code, msg); }

}  // namespace

extern "C" int orion_residual_block_noalloc(const double* dq, const double* vol, const double* dt, int idim, int jdim,
                                            int kdim, void* stream, orion_residual_t* out) {
  if (!dq || !vol || !dt || !out) return na_fail(ORION_E_INVALID, "null pointer argument");
  if (idim < 1 || jdim < 1 || kdim < 1) return na_fail(ORION_E_INVALID, "block extents must be positive");
  const long long ntot = (long long)idim * jdim * kdim;
  if (ntot > (long long)ORION_NOALLOC_MAX_POINTS)
    return na_fail(ORION_E_INVALID, "block has " + std::to_string(ntot) + " interior points; the allocation-free "
                                    "residual accepts at most " + std::to_string(ORION_NOALLOC_MAX_POINTS));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // The call ends with a stream synchronisation, which a capturing stream
  // cannot take: refuse instead of invalidating the caller's capture.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess)
    return na_fail(ORION_E_CUDA, "cudaStreamIsCapturing failed on the given stream");
  if (cap != cudaStreamCaptureStatusNone)
    return na_fail(ORION_E_INVALID, "orion_residual_block_noalloc waits for its stream and cannot run on a "
                                    "capturing stream");
  // The device address of the static array in the current context, looked up
  // on every call (it allocates nothing, and a cached address would outlive a
  // device reset or a new primary context).
  NoAllocScratch* scr = nullptr;
  {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return na_fail(ORION_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    scr = static_cast<NoAllocScratch*>(p);
  }
  const int npart = (int)((ntot + kNaChunk - 1) / kNaChunk);
  k_noalloc_partials<<<npart, kNaThreads, 0, s>>>(dq, vol, dt, idim, jdim, kdim, scr);
  k_noalloc_final<<<1, 1024, 0, s>>>(scr, npart, idim, jdim);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return na_fail(ORION_E_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  ResidualOut r;
  e = cudaMemcpyAsync(&r, &scr->result, sizeof(r), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return na_fail(ORION_E_CUDA, std::string("result copy: ") + cudaGetErrorString(e));
  out->rms = sqrt(r.rms / (double)(ntot * 5));
  out->max = r.max;
  for (int m = 0; m < 5; ++m) out->max_loc[m] = r.loc[m];
  out->pad = 0;
  out->phydtime = 0.0;  // not computed here: it is the time-step stage's minimum, not a residual statistic
  return 0;
}
