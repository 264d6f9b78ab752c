// Device side of the block-sharded step: the shard's outgoing interface data
// gathered into a contiguous buffer, and a received buffer scattered into
// place.  Exchange buffers are FP64 in both precisions (the primitive state
// and the packed dq/vol are FP64).
#pragma once
#include <cuda_runtime.h>

namespace orion {

// out[t] = base[idx[t]]: the primitive elements a peer's ghosts take.
static __global__ void k_shard_gather(const double* __restrict__ base, const long long* __restrict__ idx,
                                      double* __restrict__ out, long long n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) out[t] = base[idx[t]];
}

// base[idx[t]] = in[t]: a peer's elements into this shard's ghosts.
static __global__ void k_shard_scatter(double* __restrict__ base, const long long* __restrict__ idx,
                                       const double* __restrict__ in, long long n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) base[idx[t]] = in[t];
}

// out[5 s + m] = pack[5 slots[s] + m]: packed dq/vol slots a peer averages with.
static __global__ void k_shard_gather_slots(const double* __restrict__ pack, const int* __restrict__ slots,
                                            double* __restrict__ out, long long nslots) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nslots * 5) return;
  const long long s = t / 5;
  out[t] = pack[(long long)slots[s] * 5 + (t - s * 5)];
}

}  // namespace orion
