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

// Dynamic shared memory of one tile CTA: the 4-slot ring of neighbour-visible
// state (8 values per point, 13 on the GS passes).
template <typename T, int MODE, int TK>
constexpr size_t tile_ring_bytes() {
  return (size_t)4 * (MODE == SW_GS ? 13 : 8) * TK * 32 * sizeof(T);
}

__device__ __forceinline__ void compute_barrier(int nthreads) {
  asm volatile("bar.sync 1, %0;\n" ::"r"(nthreads) : "memory");
}

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
template <typename S, typename T, int MODE, int DIR, int TK>
__global__ void __launch_bounds__(32 * TK + 32) k_sweep_tiles(const BlockDev<S>* __restrict__ blocks,
                                                              const SweepTile* __restrict__ tiles, int ntiles,
                                                              TileCtl* __restrict__ ctl, int* __restrict__ err,
                                                              ParamsDev P, long long spin_limit) {
  constexpr int TJ = 32;
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
  // Each thread prefetches its own coming points only: the static operands of
  // its next point (registers) and the neighbour-visible state (u, v, w, H,
  // c^2, af, c, viscous factor; on the GS passes also the old increment) of
  // the point after that, which it writes to a 4-slot ring in shared memory.
  // At step t a point finds its in-tile neighbours' state in slot t-1
  // (behind) and t+1 (ahead), their new increments in s_dq; only neighbours
  // in other tiles are read from global memory.
  constexpr int NR = MODE == SW_GS ? 13 : 8;  // ring fields per point
  constexpr bool PF_STATIC = sizeof(T) == 4;   // FP32: prefetch the static operands a step ahead too
  // dynamic shared memory: tile_ring_bytes<T, MODE, TK>()
  extern __shared__ __align__(16) unsigned char tile_smem[];
  T(*s_ring)[NR][TK][TJ] = reinterpret_cast<T(*)[NR][TK][TJ]>(tile_smem);
  const long long nc = Bd.ncomp;
  const int nj = Bd.nj, nk = Bd.nk;
  const int* const koff = Bd.koff;
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
  auto valid = [&](int u) { return row && u >= 0 && u < ni; };
  auto ii_of = [&](int u) { return DIR > 0 ? u : ni - 1 - u; };
  auto cidx = [&](int u) {  // compact index of this thread's point at sweep position u
    const int ii = ii_of(u);
    return row_base(koff, ni, nk, ii + jj + kk, kk) + jj;
  };
  // static operands: coed, own (rhs, or the forward increment on the backward
  // LU-SGS pass), metrics 9, |grad| 3, 1/|grad| 3
  constexpr int NS = 21;
  auto load_static = [&](long long c, T v[NS]) {
    v[0] = (T)skcoed[c];
#pragma unroll
    for (int m = 0; m < 5; ++m) v[1 + m] = MODE == SW_LUSGS_BWD ? (T)__ldcg(skdq + m * nc + c) : (T)skrhs[m * nc + c];
#pragma unroll
    for (int m = 0; m < 9; ++m) v[6 + m] = (T)skmet[m * nc + c];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      v[15 + d] = (T)skgm[d * nc + c];
      v[18 + d] = (T)skinv[d * nc + c];
    }
  };
  auto load_ring = [&](long long c, T v[NR]) {
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] = (T)sknbq[k * nc + c];
    if (MODE == SW_GS) {
#pragma unroll
      for (int m = 0; m < 5; ++m) v[8 + m] = (T)__ldcg(skdq + m * nc + c);
    }
  };
  auto store_ring = [&](int slot, const T v[NR]) {
#pragma unroll
    for (int k = 0; k < NR; ++k) s_ring[slot][k][tk][tj] = v[k];
  };

  T st_cur[NS], st_next[NS], rg_next[NR];
  // prologue: ring slots of steps 0 and 1, static operands of step 0
  {
    const int u0 = -tj - tk;
    if (valid(u0)) {
      load_ring(cidx(u0), rg_next);
      store_ring(0, rg_next);
    }
    if (valid(u0 + 1)) {
      load_ring(cidx(u0 + 1), rg_next);
      store_ring(1, rg_next);
    }
    if (valid(u0)) load_static(cidx(u0), st_cur);
  }
  compute_barrier(32 * TK);

  T prev[5] = {T(0), T(0), T(0), T(0), T(0)};  // this thread's increment of the previous step (behind-i)
  for (int t = 0; t < nsteps; ++t) {
    const int u = t - tj - tk;  // position along i in sweep order
    // prefetch (independent of the upstream tiles: nobody else writes these)
    const bool nxt1 = valid(u + 1), nxt2 = valid(u + 2);
    if (PF_STATIC && nxt1) load_static(cidx(u + 1), st_next);
    if (nxt2) load_ring(cidx(u + 2), rg_next);
    if (*(volatile int*)&s_ready <= t) {  // bounded: the control warp releases or gives up well before this
      const long long t0 = clock64();
      while (*(volatile int*)&s_ready <= t) {
        if (clock64() - t0 > kComputeWaitCycles) {
          atomicExch(err, 1);
          break;
        }
      }
    }
    if (valid(u)) {
      if (!PF_STATIC) load_static(cidx(u), st_cur);
      const int ii = ii_of(u);
      const int s = ii + jj + kk;
      const long long c = row_base(koff, ni, nk, s, kk) + jj;
      bool has[6];
      has[0] = ii > 0;
      has[1] = jj > 0;
      has[2] = kk > 0;
      has[3] = ii < ni - 1;
      has[4] = jj < nj - 1;
      has[5] = kk < nk - 1;
      const int pb = (t - 1) & 1, rb = (t - 1) & 3, ra = (t + 1) & 3;
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
          const int slot = behind ? rb : ra;
#pragma unroll
          for (int k = 0; k < 8; ++k) nq[k] = s_ring[slot][k][sk][sj];
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
            for (int m = 0; m < 5; ++m) dn[m] = s_ring[slot][8 + m][sk][sj];
          }
        } else {
          // neighbour in another tile: (ii, jj +- 1, kk) on plane s +- 1 or (ii, jj, kk +- 1)
          const bool lower = q < 3;
          const int sn = lower ? s - 1 : s + 1;
          const long long n = d == 1 ? row_base(koff, ni, nk, sn, kk) + (lower ? jj - 1 : jj + 1)
                                     : row_base(koff, ni, nk, sn, lower ? kk - 1 : kk + 1) + jj;
#pragma unroll
          for (int k = 0; k < 8; ++k) nq[k] = (T)sknbq[k * nc + n];
#pragma unroll
          for (int m = 0; m < 5; ++m) dn[m] = (T)__ldcg(skdq + m * nc + n);
        }
        // the neighbour's state as seen through this point's metric: spectral
        // radius, split eigenvalues and viscous radius (calc_spectral_radius,
        // compute_flux_splitting, calc_visc_spectral_radius,
        // StateUpdater.cpp:175-265), in the reference's operation order
        T pc[5], nrm[3];
        const T kx = st_cur[6 + 3 * d], ky = st_cur[7 + 3 * d], kz = st_cur[8 + 3 * d];
        const T gmr = st_cur[15 + d], inv = st_cur[18 + d];
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
      const T coed = st_cur[0];
#pragma unroll
      for (int m = 0; m < 5; ++m) {
        const T own = MODE == SW_LUSGS_BWD ? st_cur[1 + m] : -st_cur[1 + m];
        S v;
        if (MODE == SW_LUSGS_FWD) v = (S)((own + rhs0[m]) * coed);
        else if (MODE == SW_LUSGS_BWD) v = (S)(own - rhs0[m] * coed);
        else v = (S)((rhs0[m] + own) * coed);
        skdq[m * nc + c] = v;
        s_dq[t & 1][m][tk][tj] = (T)v;
        prev[m] = (T)v;
      }
    }
    if (nxt2) store_ring((t + 2) & 3, rg_next);
    if (PF_STATIC && nxt1) {
#pragma unroll
      for (int k = 0; k < NS; ++k) st_cur[k] = st_next[k];
    }
    compute_barrier(32 * TK);  // step t's writes (shared and global) are done
    if (threadIdx.x == 0) {
      __threadfence_block();
      *(volatile int*)&s_done = t + 1;
    }
  }
}

}  // namespace orion
