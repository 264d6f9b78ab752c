// Tile wavefront form of the LU-SGS / symmetric Gauss-Seidel sweeps
// (StateUpdater::lusgs_sweep and gs_pr_sweep, src/solver/StateUpdater.cpp:297-445).
//
// The increment-independent coefficients of every neighbour term (the
// neighbour's spectral radius through this point's metric, the split
// eigenvalues, the viscous radius) are formed in place from the neighbour's
// prepared state (u, v, w, H, c^2, af, c, viscous factor) and this point's
// static metric magnitudes, so a pass reads per point only its own operands,
// its neighbours' prepared state and increments, and writes its increment.
//
// One launch per pass.  A CTA owns a tile of 32 x TK grid lines along i of one
// block (32 consecutive j, TK consecutive k) and walks it: at local step t the
// thread of line (tj, tk) updates the point i = t - tj - tk (mirrored on the
// backward passes).  All points a CTA touches at one step lie on one i+j+k
// hyperplane, and within a k row they are consecutive in the plane-major
// layout, so every warp reads and writes 32 consecutive elements.
//
// Dependencies are the reference's lexicographic order exactly: a point reads
// its "behind" neighbours (lower i, j, k on forward passes, upper on backward
// ones) after they were updated in this pass, and its "ahead" neighbours
// before.  Inside a tile the behind-j and behind-k neighbours were updated one
// step earlier by the adjacent threads (shared memory, one barrier per step),
// the behind-i neighbour by the same thread (registers).  Across tiles a CTA
// waits on the progress counter of its upstream neighbour tile in j and in k,
// which runs 32 (resp. TK) steps ahead; the ahead neighbours are only updated
// by the downstream tiles after this tile has published that it read them.
//
// Tiles are claimed through a ticket counter in a dependency-respecting order,
// so a CTA only ever waits on tiles held by CTAs that are already running:
// the launch needs no co-residency guarantee.  Every wait is bounded: after
// spin_limit polls it raises the shared error word and the CTA returns; every
// other waiting CTA sees the word and returns too (the host reports
// ORION_E_TIMEOUT).
#pragma once

#include <cstddef>

#include "kernels.cuh"

namespace orion {

// One tile of one pass.  (jb, kb) is the tile's first line in sweep order:
// the lowest (j, k) on forward passes, the highest on backward passes.
struct SweepTile {
  int block;
  int jb, kb;
  int up_j, up_k;  // ticket slots of the upstream tiles in j and k (-1: none)
  int pad[3];
};

// Per-launch control: ticket counter then one progress word per tile slot
// (steps completed), zeroed before every pass.
struct TileCtl {
  unsigned int ticket;
  unsigned int pad;
  unsigned int progress[1];
};

// Polls are plain volatile loads: an acquire load at GPU scope would discard
// the SM's L1 contents at every poll.  Nothing a tile reads through L1 is
// written during the pass; the increments other tiles write are read with
// ld.global.cg (L2, the point of coherence), and the producer publishes its
// progress only after a fence that makes them visible there.
__device__ __forceinline__ unsigned int ld_poll_u32(const unsigned int* p) { return *(const volatile unsigned int*)p; }

__device__ __forceinline__ void publish_u32(unsigned int* p, unsigned int v) {
  __threadfence();
  *(volatile unsigned int*)p = v;
}

// Waits (bounded) until *p >= need; `known` caches the last value seen.
// Returns false when this wait or another CTA's gave up.
__device__ __forceinline__ bool tile_wait(const unsigned int* p, unsigned int need, unsigned int& known, int* err,
                                          long long spin_limit) {
  if (known >= need) return true;
  long long it = 0;
  while (true) {
    const unsigned int v = ld_poll_u32(p);
    if (v >= need) {
      known = v;
      return true;
    }
    if (*(volatile int*)err) return false;
    if (++it > spin_limit) {
      atomicExch(err, 1);
      return false;
    }
    __nanosleep(32);
  }
}

// Compact index of (s, kk, jj) is row_base(s, kk) + jj.
__device__ __forceinline__ long long row_base(const int* __restrict__ koff, int ni, int nk, int s, int kk) {
  const int v = s - kk - (ni - 1);
  return (long long)__ldg(koff + (long long)s * nk + kk) - (v > 0 ? v : 0);
}

// Bound of a compute warp's wait for the control warp (about four seconds).
constexpr long long kComputeWaitCycles = 8000000000LL;

__device__ __forceinline__ void compute_barrier(int nthreads) {
  asm volatile("bar.sync 1, %0;\n" ::"r"(nthreads) : "memory");
}

// Prefetch distance (steps) and tile height of each precision: FP32 tiles are
// 32 x 4 lines and read their operands three steps ahead, FP64 tiles 32 x 2
// lines two steps ahead (the prefetch buffers live in shared memory).
#ifndef ORION_TILE_K_F32
#define ORION_TILE_K_F32 4
#endif
#ifndef ORION_TILE_PD_F32
#define ORION_TILE_PD_F32 3
#endif
#ifndef ORION_TILE_K_F64
#define ORION_TILE_K_F64 2
#endif
#ifndef ORION_TILE_PD_F64
#define ORION_TILE_PD_F64 2
#endif
template <typename T> struct TileShape;
template <> struct TileShape<float> { static constexpr int TK = ORION_TILE_K_F32, PD = ORION_TILE_PD_F32; };
template <> struct TileShape<double> { static constexpr int TK = ORION_TILE_K_F64, PD = ORION_TILE_PD_F64; };

// Fields a point's owner prefetches: static operands (coed, own: rhs or the
// forward increment, metrics 9, |grad| 3, 1/|grad| 3) for itself, and the
// neighbour-visible state (u, v, w, H, c^2, af, c, viscous factor, and on the
// GS passes the old increment) for the adjacent threads.
constexpr int kTileStatics = 21;
template <int MODE> __host__ __device__ constexpr int tile_ring_fields() { return MODE == SW_GS ? 13 : 8; }

// Dynamic shared memory of one tile CTA with `npl` hyperplanes at most.
// Edge records: the state (8) and increment (5) of a neighbour in another
// tile, per step slot, for the first and last lane of every k row (j edges)
// and every lane of the first and last k row (k edges).
constexpr int kTileEdgeFields = 13;
template <int TK> __host__ __device__ constexpr int tile_edge_records() { return 2 * TK + 64; }

template <typename T, int MODE>
constexpr size_t tile_smem_bytes(int npl) {
  constexpr int TK = TileShape<T>::TK, PD = TileShape<T>::PD;
  return (size_t)((PD + 1) * kTileStatics + (PD + 2) * tile_ring_fields<MODE>()) * TK * 32 * sizeof(T) +
         (size_t)(PD + 1) * tile_edge_records<TK>() * kTileEdgeFields * sizeof(T) +
         (size_t)(TK + 2) * npl * sizeof(int);
}

template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
  const unsigned int s = (unsigned int)__cvta_generic_to_shared(smem);
  if (sizeof(T) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// MODE: SW_LUSGS_FWD (forward, behind = lower, uses q 0..2), SW_LUSGS_BWD
// (backward, behind = upper, uses q 3..5), SW_GS with DIR +1 / -1 (all six).
//
// 32*TK compute threads and one control warp.  The compute warps separate
// their steps with a named barrier of their own; before step t they wait (in
// shared memory) until the control warp has seen the upstream tiles far
// enough along.  The control warp publishes the compute warps' completed
// steps (fence, then the progress word) and polls the upstream progress, so
// neither the fence nor the polls are on the compute warps' path.  When a
// wait gives up, the control warp raises the error word and releases every
// remaining step: the compute warps finish the tile on whatever data is there
// (every access stays in bounds) and the host reports ORION_E_TIMEOUT.
//
// Each compute thread copies its own points' operands PD steps ahead with
// cp.async into shared memory: the static operands into a (PD+1)-slot buffer
// of its own, the neighbour-visible state into a (PD+2)-slot ring the adjacent
// threads read at step t from slot t-1 (behind neighbours) and t+1 (ahead).
// New increments of the behind neighbours come from the previous step
// (registers for i, s_dq for j and k).  Neighbours in other tiles are
// prefetched with the same lead into per-step edge records; a step's operands
// are fetched only once the upstream tiles allow that step, so the compute of
// a step never waits on memory.  The row bases of the tile's k rows (and the
// rows on either side) are cached in shared memory for every hyperplane.
template <typename S, typename T, int MODE, int DIR>
__global__ void __launch_bounds__(32 * TileShape<T>::TK + 32) k_sweep_tiles(const BlockDev<S>* __restrict__ blocks,
                                                                           const SweepTile* __restrict__ tiles,
                                                                           int ntiles, TileCtl* __restrict__ ctl,
                                                                           int* __restrict__ err, long long spin_limit) {
  static_assert(sizeof(S) == sizeof(T), "the tile sweeps keep operands in their storage precision");
  constexpr int TJ = 32, TK = TileShape<T>::TK, PD = TileShape<T>::PD;
  constexpr int NSS = PD + 1, NSR = PD + 2, NR = tile_ring_fields<MODE>(), NS = kTileStatics;
  constexpr int Q0 = MODE == SW_LUSGS_BWD ? 3 : 0;
  constexpr int Q1 = MODE == SW_LUSGS_FWD ? 3 : 6;
  // behind neighbours (updated in this pass) are q = QB .. QB+2
  constexpr int QB = DIR > 0 ? 0 : 3;
  __shared__ int s_slot;
  __shared__ int s_ready;  // steps whose upstream data is ready (control -> compute)
  __shared__ int s_done;   // steps the compute warps have completed (compute -> control)
  __shared__ T s_dq[2][5][TK][TJ];  // each thread's increment of the last two steps
  const int tj = threadIdx.x & 31, tk = threadIdx.x >> 5;
  if (threadIdx.x == 0) {
    s_slot = (int)atomicAdd(&ctl->ticket, 1u);
    s_ready = 0;
    s_done = 0;
  }
  __syncthreads();
  const int slot = s_slot;
  if (slot >= ntiles) return;
  const SweepTile W = tiles[slot];
  const BlockDev<S>& Bd = blocks[W.block];
  const ParamsDev& P = Bd.prm;
  const int ni = Bd.ni;
  const int nsteps = ni + TJ + TK - 2;

  if (tk == TK) {  // ---------------- control warp ----------------
    if (tj != 0) return;
    const int up_j = W.up_j, up_k = W.up_k;
    unsigned int* const mine = &ctl->progress[slot];
    // steps allowed by an upstream tile that has completed p steps and runs `lag` ahead
    auto allowed = [&](int up, int lag) -> int {
      if (up < 0) return nsteps;
      const int p = (int)ld_poll_u32(&ctl->progress[up]);
      return p >= nsteps ? nsteps : max(0, p - lag + 1);
    };
    int ready = 0, published = 0;
    long long idle = 0;
    while (published < nsteps) {
      bool moved = false;
      if (ready < nsteps) {
        const int r = min(allowed(up_j, TJ), allowed(up_k, TK));
        if (r > ready) {
          ready = r;
          *(volatile int*)&s_ready = ready;
          moved = true;
        }
      }
      const int d = *(volatile int*)&s_done;
      if (d > published) {
        publish_u32(mine, (unsigned int)d);
        published = d;
        moved = true;
      }
      if (moved) {
        idle = 0;
        continue;
      }
      if (*(volatile int*)err || ++idle > spin_limit) {  // give up: release the compute warps, stop publishing
        if (!*(volatile int*)err) atomicExch(err, 1);
        *(volatile int*)&s_ready = nsteps;
        return;
      }
      __nanosleep(32);
    }
    return;
  }

  // ---------------- compute warps ----------------
  extern __shared__ __align__(16) unsigned char tile_smem[];
  T(*s_stat)[NS][TK][TJ] = reinterpret_cast<T(*)[NS][TK][TJ]>(tile_smem);
  T(*s_ring)[NR][TK][TJ] = reinterpret_cast<T(*)[NR][TK][TJ]>(tile_smem + sizeof(T) * NSS * NS * TK * TJ);
  constexpr int NE = tile_edge_records<TK>(), NEF = kTileEdgeFields;
  T(*s_edge)[NE][NEF] = reinterpret_cast<T(*)[NE][NEF]>(tile_smem + sizeof(T) * (NSS * NS + NSR * NR) * TK * TJ);
  int* s_rowb = reinterpret_cast<int*>(tile_smem + sizeof(T) * ((NSS * NS + NSR * NR) * TK * TJ + NSS * NE * NEF));
  const long long nc = Bd.ncomp;
  const int nj = Bd.nj, nk = Bd.nk, npl = Bd.nplanes;
  S* const skdq = Bd.sk_dq;
  const S* const skcoed = Bd.sk_coed;
  const S* const skrhs = Bd.sk_rhs;
  const S* const sknbq = Bd.sk_nbq;
  const S* const skmet = Bd.sk_metrics;
  const S* const skgm = Bd.sk_gm;
  const S* const skinv = Bd.sk_inv;
  const int jj = W.jb + DIR * tj, kk = W.kb + DIR * tk;
  const bool row = jj >= 0 && jj < nj && kk >= 0 && kk < nk;
  const T gm1 = T(P.gamma) - T(1);
  const int nvis = P.nvis;
  // row bases of k rows kb - DIR .. kb + DIR*TK: compact index of (s, kk_r, jj) = s_rowb[r * npl + s] + jj
  {
    const int* const koff = Bd.koff;
    for (int e = threadIdx.x; e < (TK + 2) * npl; e += 32 * TK) {
      const int r = e / npl, sp = e - r * npl;
      const int kr = W.kb + DIR * (r - 1);
      s_rowb[e] = (kr >= 0 && kr < nk) ? (int)row_base(koff, ni, nk, sp, kr) : 0;
    }
  }
  // rows of this thread (r = tk + 1) and its k neighbours (r = tk, tk + 2)
  const int* const rb_own = s_rowb + (tk + 1) * npl;
  const int* const rb_lo = s_rowb + (DIR > 0 ? tk : tk + 2) * npl;  // row kk - 1
  const int* const rb_hi = s_rowb + (DIR > 0 ? tk + 2 : tk) * npl;  // row kk + 1
  auto valid = [&](int u) { return row && u >= 0 && u < ni; };
  auto ii_of = [&](int u) { return DIR > 0 ? u : ni - 1 - u; };
  compute_barrier(32 * TK);  // row bases ready

  // edge increments in flight: loaded at prefetch time, stored to the edge
  // record at the end of the step
  T edq[4][5];
  T* edq_dst[4] = {nullptr, nullptr, nullptr, nullptr};
  // waits (bounded) until the upstream tiles allow step x
  auto wait_ready = [&](int x) {
    if (*(volatile int*)&s_ready <= x) {  // bounded: the control warp releases or gives up well before this
      const long long t0 = clock64();
      while (*(volatile int*)&s_ready <= x) {
        if (clock64() - t0 > kComputeWaitCycles) {
          atomicExch(err, 1);
          break;
        }
      }
    }
  };
  // copies the operands of this thread's point at sweep position u into the
  // buffers of step slot `step` (the upstream tiles must allow that step)
  auto prefetch = [&](int u, int step) {
    if (!valid(u)) return;
    const int ii = ii_of(u);
    const long long c = (long long)rb_own[ii + jj + kk] + jj;
    T(*st)[TK][TJ] = s_stat[step % NSS];
    T(*rg)[TK][TJ] = s_ring[step % NSR];
    cp_async_elem(&st[0][tk][tj], skcoed + c);
#pragma unroll
    for (int m = 0; m < 5; ++m)
      cp_async_elem(&st[1 + m][tk][tj], (MODE == SW_LUSGS_BWD ? (const S*)skdq : skrhs) + m * nc + c);
#pragma unroll
    for (int m = 0; m < 9; ++m) cp_async_elem(&st[6 + m][tk][tj], skmet + m * nc + c);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      cp_async_elem(&st[15 + d][tk][tj], skgm + d * nc + c);
      cp_async_elem(&st[18 + d][tk][tj], skinv + d * nc + c);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) cp_async_elem(&rg[k][tk][tj], sknbq + k * nc + c);
    if (MODE == SW_GS) {
#pragma unroll
      for (int m = 0; m < 5; ++m) cp_async_elem(&rg[8 + m][tk][tj], (const S*)skdq + m * nc + c);
    }
    // neighbours in other tiles: state by cp.async, increment (written during
    // this pass by the upstream tile, or not yet by the downstream one) from
    // L2 into registers, stored at the end of the step
    const int s = ii + jj + kk;
    T(*ed)[NEF] = s_edge[step % NSS];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      // e: 0 behind-j, 1 ahead-j, 2 behind-k, 3 ahead-k
      const bool isj = e < 2, behind = (e & 1) == 0;
      if (isj ? (behind ? tj != 0 : tj != TJ - 1) : (behind ? tk != 0 : tk != TK - 1)) continue;
      if (MODE == SW_LUSGS_FWD && !behind) continue;  // these passes read behind neighbours only
      if (MODE == SW_LUSGS_BWD && !behind) continue;
      const bool lower = behind == (DIR > 0);  // natural lower neighbour (j-1 or k-1)
      const int nd = isj ? jj + (lower ? -1 : 1) : kk + (lower ? -1 : 1);
      if (nd < 0 || nd >= (isj ? nj : nk)) continue;
      const int sn = lower ? s - 1 : s + 1;
      const long long n = isj ? (long long)rb_own[sn] + nd : (long long)(lower ? rb_lo : rb_hi)[sn] + jj;
      const int rec = isj ? (behind ? 0 : 1) * TK + tk : 2 * TK + (behind ? 0 : 1) * 32 + tj;
#pragma unroll
      for (int k = 0; k < 8; ++k) cp_async_elem(&ed[rec][k], sknbq + k * nc + n);
      T* const slotp = &ed[rec][8];
#pragma unroll
      for (int m = 0; m < 5; ++m) edq[e][m] = (T)__ldcg(skdq + m * nc + n);
      edq_dst[e] = slotp;
    }
  };
  auto store_edges = [&]() {
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (!edq_dst[e]) continue;
#pragma unroll
      for (int m = 0; m < 5; ++m) edq_dst[e][m] = edq[e][m];
      edq_dst[e] = nullptr;
    }
  };
  {
    const int u0 = -tj - tk;
    wait_ready(min(PD, nsteps) - 1);
#pragma unroll
    for (int p = 0; p < PD; ++p) {
      prefetch(u0 + p, p);
      cp_async_commit();
      store_edges();
    }
  }

  T prev[5] = {T(0), T(0), T(0), T(0), T(0)};  // this thread's increment of the previous step (behind-i)
  for (int t = 0; t < nsteps; ++t) {
    cp_async_wait<PD - 2>();   // this thread's copies up to step t+1 have landed
    compute_barrier(32 * TK);  // everybody's copies up to step t+1 and step t-1's increments are visible
    if (threadIdx.x == 0 && t > 0) {
      __threadfence_block();
      *(volatile int*)&s_done = t;
    }
    const int u = t - tj - tk;  // position along i in sweep order
    if (t + PD < nsteps) {
      wait_ready(t + PD);
      prefetch(u + PD, t + PD);
    }
    cp_async_commit();
    if (valid(u)) {
      const T(*st)[TK][TJ] = s_stat[t % NSS];
      const int ii = ii_of(u);
      const int s = ii + jj + kk;
      const long long c = (long long)rb_own[s] + jj;
      bool has[6];
      has[0] = ii > 0;
      has[1] = jj > 0;
      has[2] = kk > 0;
      has[3] = ii < ni - 1;
      has[4] = jj < nj - 1;
      has[5] = kk < nk - 1;
      const int pb = (t - 1) & 1;
      const T(*rgb)[TK][TJ] = s_ring[(t + NSR - 1) % NSR];
      const T(*rga)[TK][TJ] = s_ring[(t + 1) % NSR];
      T rhs0[5] = {T(0), T(0), T(0), T(0), T(0)};
      // lower neighbours first (i, j, k), then upper (i, j, k): the reference's order
#pragma unroll
      for (int q = Q0; q < Q1; ++q) {
        if (!has[q]) continue;
        const int d = q % 3;
        const bool behind = q >= QB && q < QB + 3;
        T dn[5], nq[8];
        // source of the neighbour: this thread (i), the adjacent thread (j, k)
        // in this tile, or another tile (global memory)
        const bool in_tile = d == 0 || (d == 1 ? (behind ? tj > 0 : tj < TJ - 1) : (behind ? tk > 0 : tk < TK - 1));
        if (in_tile) {
          const int sj = d == 1 ? (behind ? tj - 1 : tj + 1) : tj;
          const int sk = d == 2 ? (behind ? tk - 1 : tk + 1) : tk;
          const T(*rg)[TK][TJ] = behind ? rgb : rga;
#pragma unroll
          for (int k = 0; k < 8; ++k) nq[k] = rg[k][sk][sj];
          if (behind) {
            if (d == 0) {
#pragma unroll
              for (int m = 0; m < 5; ++m) dn[m] = prev[m];
            } else {
#pragma unroll
              for (int m = 0; m < 5; ++m) dn[m] = s_dq[pb][m][sk][sj];
            }
          } else {
#pragma unroll
            for (int m = 0; m < 5; ++m) dn[m] = rg[8 + m][sk][sj];
          }
        } else {
          // neighbour in another tile: its record, prefetched with this step's operands
          const int rec = d == 1 ? (behind ? 0 : 1) * TK + tk : 2 * TK + (behind ? 0 : 1) * 32 + tj;
          const T* ed = s_edge[t % NSS][rec];
#pragma unroll
          for (int k = 0; k < 8; ++k) nq[k] = ed[k];
#pragma unroll
          for (int m = 0; m < 5; ++m) dn[m] = ed[8 + m];
        }
        // the neighbour's state as seen through this point's metric: spectral
        // radius, split eigenvalues and viscous radius (calc_spectral_radius,
        // compute_flux_splitting, calc_visc_spectral_radius,
        // StateUpdater.cpp:175-265), in the reference's operation order
        T pc[5], nrm[3];
        const T kx = st[6 + 3 * d][tk][tj], ky = st[7 + 3 * d][tk][tj], kz = st[8 + 3 * d][tk][tj];
        const T gmr = st[15 + d][tk][tj], inv = st[18 + d][tk][tj];
        const T c2 = nq[4], cm = nq[6];
        const T ct = nq[0] * kx + nq[1] * ky + nq[2] * kz + T(0);
        const T r = tabs(ct) + cm * gmr;
        const T gmc = gmr < T(1.0e-30) ? T(1.0e-30) : gmr;
        const T sign = q < 3 ? T(1) : T(-1);
        T l1 = ct;
        T l4 = ct + cm * gmc;
        T l5 = ct - cm * gmc;
        l1 = T(0.5) * (l1 + sign * r);
        l4 = T(0.5) * (l4 + sign * r);
        l5 = T(0.5) * (l5 + sign * r);
        pc[0] = l1;
        pc[1] = (T(2) * l1 - l4 - l5) / (T(2) * c2);
        pc[2] = (l4 - l5) / (T(2) * cm);
        pc[3] = (ct - T(0)) * inv;
        pc[4] = nvis == 1 ? T(0.5) * (nq[7] * (kx * kx + ky * ky + kz * kz)) : T(0);
        nrm[0] = kx * inv;
        nrm[1] = ky * inv;
        nrm[2] = kz * inv;
        split_term<T, MODE>(q, gm1, nvis, dn, nq, pc, nrm, rhs0);
      }
      const T coed = st[0][tk][tj];
#pragma unroll
      for (int m = 0; m < 5; ++m) {
        const T ownv = st[1 + m][tk][tj];
        const T own = MODE == SW_LUSGS_BWD ? ownv : -ownv;
        S v;
        if (MODE == SW_LUSGS_FWD) v = (S)((own + rhs0[m]) * coed);
        else if (MODE == SW_LUSGS_BWD) v = (S)(own - rhs0[m] * coed);
        else v = (S)((rhs0[m] + own) * coed);
        skdq[m * nc + c] = v;
        s_dq[t & 1][m][tk][tj] = (T)v;
        prev[m] = (T)v;
      }
    }
    store_edges();
  }
  cp_async_wait<0>();
  compute_barrier(32 * TK);
  if (threadIdx.x == 0) {
    __threadfence_block();
    *(volatile int*)&s_done = nsteps;
  }
}

}  // namespace orion
