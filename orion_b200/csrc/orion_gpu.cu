// C-ABI runtime of the B200 per-step path: case lifetime, work lists, stage
// launchers and the graph-captured step.  See include/orion_gpu.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <mutex>
#include <vector>

#include "case.hpp"
#include "metrics_dev.cuh"
#include "output_dev.cuh"
#include "shard_dev.cuh"
#include "sweep_tiles.cuh"

using namespace orion;

namespace orion {
thread_local std::string g_last_error;
int set_error(int code, const std::string& msg) { return fail(code, msg); }
}  // namespace orion


namespace {

template <typename T>
int dev_upload(orion_case_t c, T** dptr, const std::vector<T>& v, bool keep = false) {
  *dptr = nullptr;
  if (v.empty()) return 0;
  void* p = nullptr;
  if (cudaMallocAsync(&p, v.size() * sizeof(T), c->stream) != cudaSuccess)
    return fail(ORION_E_NOMEM, "cudaMallocAsync (work list)");
  c->allocs.push_back(p);
  CUDA_TRY(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, c->stream));
  if (keep) {  // a list a group is built from
    const auto* bytes = reinterpret_cast<const unsigned char*>(v.data());
    c->list_mirror[p].assign(bytes, bytes + v.size() * sizeof(T));
  }
  *dptr = static_cast<T*>(p);
  return 0;
}

template <typename T>
int dev_alloc(orion_case_t c, T** dptr, size_t n) {
  void* p = nullptr;
  if (cudaMallocAsync(&p, std::max<size_t>(n, 1) * sizeof(T), c->stream) != cudaSuccess)
    return fail(ORION_E_NOMEM, "cudaMallocAsync");
  c->allocs.push_back(p);
  CUDA_TRY(cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * sizeof(T), c->stream));
  *dptr = static_cast<T*>(p);
  return 0;
}

// Bytes of one block's fields for storage size ssz.
size_t block_bytes(const HostBlock& b, size_t ssz) {
  const size_t np = (size_t)b.npad;
  size_t s = 0;
  auto add = [&](size_t bytes) { s = align_up(s, 256) + bytes; };
  add(6 * np * 8);    // prim
  add(5 * np * 8);    // q
  add(5 * np * ssz);  // dq
  add(9 * np * 8);    // metrics
  add(np * 8);        // vol
  add(np * ssz);      // dt
  add(np * ssz);      // c
  add(np * ssz);      // mu
  add(12 * np * ssz); // duvwt
  add(np);            // bcmask
  if (ssz == 4) {     // FP32 shadows: prim 6, metrics 9, vol
    add(6 * np * 4);
    add(9 * np * 4);
    add(np * 4);
  }
  const size_t nc = (size_t)b.idim * b.jdim * b.kdim;
  const size_t npl = (size_t)(b.idim + b.jdim + b.kdim - 2);
  add((npl * b.kdim + 1) * 4);  // koff
  add(nc * 4);                  // sk_nat
  add(6 * nc * 4);              // sk_nb
  add(80 * nc * ssz);           // sk_metrics 9, sk_vol, sk_prim 5, sk_mu, sk_coed, sk_rhs 5, sk_dq 5, sk_nrm 9, sk_nbq 8,
                                // sk_pair 30, sk_gm 3, sk_inv 3
  return align_up(s, 256);
}

template <typename S>
void carve_block(char* base, const HostBlock& b, BlockDev<S>& d) {
  const size_t np = (size_t)b.npad;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    off = align_up(off, 256);
    char* p = base + off;
    off += bytes;
    return p;
  };
  d.prim = reinterpret_cast<double*>(take(6 * np * 8));
  d.q = reinterpret_cast<double*>(take(5 * np * 8));
  d.dq = reinterpret_cast<S*>(take(5 * np * sizeof(S)));
  d.metrics = reinterpret_cast<double*>(take(9 * np * 8));
  d.vol = reinterpret_cast<double*>(take(np * 8));
  d.dt = reinterpret_cast<S*>(take(np * sizeof(S)));
  d.c = reinterpret_cast<S*>(take(np * sizeof(S)));
  d.mu = reinterpret_cast<S*>(take(np * sizeof(S)));
  d.duvwt = reinterpret_cast<S*>(take(12 * np * sizeof(S)));
  d.bcmask = reinterpret_cast<uint8_t*>(take(np));
  d.prim_f = d.met_f = d.vol_f = nullptr;
  if (sizeof(S) == 4) {  // FP32 shadows of prim, metrics, vol for the mixed path's flux kernels
    d.prim_f = reinterpret_cast<float*>(take(6 * np * 4));
    d.met_f = reinterpret_cast<float*>(take(9 * np * 4));
    d.vol_f = reinterpret_cast<float*>(take(np * 4));
  }
  const size_t nc = (size_t)b.idim * b.jdim * b.kdim;
  const int npl = b.idim + b.jdim + b.kdim - 2;
  d.nplanes = npl;
  d.ncomp = (long long)nc;
  d.koff = reinterpret_cast<int*>(take(((size_t)npl * b.kdim + 1) * 4));
  d.sk_nat = reinterpret_cast<int*>(take(nc * 4));
  d.sk_nb = reinterpret_cast<int*>(take(6 * nc * 4));
  S* sk = reinterpret_cast<S*>(take(80 * nc * sizeof(S)));
  d.sk_metrics = sk;
  d.sk_vol = sk + 9 * nc;
  d.sk_prim = sk + 10 * nc;
  d.sk_mu = sk + 15 * nc;
  d.sk_coed = sk + 16 * nc;
  d.sk_rhs = sk + 17 * nc;
  d.sk_dq = sk + 22 * nc;
  d.sk_nrm = sk + 27 * nc;
  d.sk_nbq = sk + 36 * nc;
  d.sk_pair = sk + 44 * nc;
  d.sk_gm = sk + 74 * nc;
  d.sk_inv = sk + 77 * nc;
  d.prm = ParamsDev{};  // set by the caller: the case's parameters
  d.ni = b.idim;
  d.nj = b.jdim;
  d.nk = b.kdim;
  d.nx = b.nx;
  d.ny = b.ny;
  d.nz = b.nz;
  d.npad = b.npad;
}

int validate_blocks(int nblocks, const orion_block_desc_t* blocks) {
  if (nblocks <= 0 || !blocks) return fail(ORION_E_INVALID, "nblocks must be positive");
  for (int b = 0; b < nblocks; ++b) {
    const auto& d = blocks[b];
    if (d.idim < 12 || d.jdim < 12 || d.kdim < 12)
      return fail(ORION_E_UNSUPPORTED, "block " + std::to_string(b) + ": every extent must be >= 12 points");
    // interior point indices within a block are 32-bit in several kernels
    if ((long long)(d.idim + 2 * NG) * (d.jdim + 2 * NG) * (d.kdim + 2 * NG) >= (1LL << 31))
      return fail(ORION_E_UNSUPPORTED, "block " + std::to_string(b) + ": more than 2^31 padded points");
    if (d.nregions < 0 || (d.nregions > 0 && !d.regions))
      return fail(ORION_E_INVALID, "block " + std::to_string(b) + ": bad region list");
    for (int r = 0; r < d.nregions; ++r) {
      const auto& g = d.regions[r];
      if (g.bctype < 0 && (g.nbt < 1 || g.nbt > nblocks || g.ibcwin < 1))
        return fail(ORION_E_INVALID, "block " + std::to_string(b) + " region " + std::to_string(r) +
                                         ": interface target out of range");
    }
  }
  return 0;
}

// Plane-major order of a block's interior points: hyperplane s = ii+jj+kk, then
// kk, then jj.  koff[s*nk + kk] is the start of the (s, kk) run.
void plane_major_maps(const HostBlock& h, std::vector<int>& koff, std::vector<int>& nat) {
  const int ni = h.idim, nj = h.jdim, nk = h.kdim;
  const int npl = ni + nj + nk - 2;
  koff.assign((size_t)npl * nk + 1, 0);
  nat.clear();
  nat.reserve((size_t)ni * nj * nk);
  for (int s = 0; s < npl; ++s)
    for (int kk = 0; kk < nk; ++kk) {
      koff[(size_t)s * nk + kk] = (int)nat.size();
      const int jlo = std::max(0, s - kk - (ni - 1));
      const int jhi = std::min(nj - 1, s - kk);
      for (int jj = jlo; jj <= jhi; ++jj) {
        const int ii = s - jj - kk;
        nat.push_back((ii + NG) + h.nx * ((jj + NG) + h.ny * (kk + NG)));
      }
    }
  koff[(size_t)npl * nk] = (int)nat.size();
}

// Compact indices of the six face neighbours of every compact point (component
// stride ncomp): lower i, j, k then upper i, j, k; -1 where the neighbour is a ghost.
void plane_major_neighbours(const HostBlock& h, const std::vector<int>& koff, const std::vector<int>& nat,
                            std::vector<int>& nb) {
  const int ni = h.idim, nj = h.jdim, nk = h.kdim;
  const size_t nc = nat.size();
  nb.assign(6 * nc, -1);
  auto jlo = [&](int s, int kk) { return std::max(0, s - kk - (ni - 1)); };
  for (size_t c = 0; c < nc; ++c) {
    const int v = nat[c];
    const int i = v % h.nx, r = v / h.nx;
    const int ii = i - NG, jj = r % h.ny - NG, kk = r / h.ny - NG;
    const int s = ii + jj + kk;
    if (ii > 0) nb[0 * nc + c] = koff[(size_t)(s - 1) * nk + kk] + (jj - jlo(s - 1, kk));
    if (jj > 0) nb[1 * nc + c] = koff[(size_t)(s - 1) * nk + kk] + (jj - 1 - jlo(s - 1, kk));
    if (kk > 0) nb[2 * nc + c] = koff[(size_t)(s - 1) * nk + kk - 1] + (jj - jlo(s - 1, kk - 1));
    if (ii < ni - 1) nb[3 * nc + c] = koff[(size_t)(s + 1) * nk + kk] + (jj - jlo(s + 1, kk));
    if (jj < nj - 1) nb[4 * nc + c] = koff[(size_t)(s + 1) * nk + kk] + (jj + 1 - jlo(s + 1, kk));
    if (kk < nk - 1) nb[5 * nc + c] = koff[(size_t)(s + 1) * nk + kk + 1] + (jj - jlo(s + 1, kk + 1));
  }
}

}  // namespace

int orion::build_cluster_lists(orion_case_t c, int nclusters) {
  auto& L = c->L;
  const int nb = c->nblocks;
  nclusters = std::max(1, std::min(nclusters, nb));
  std::vector<int> order(nb);
  for (int b = 0; b < nb; ++b) order[b] = b;
  std::sort(order.begin(), order.end(), [&](int a, int b) {
    const auto& ha = c->hb[a];
    const auto& hb = c->hb[b];
    return (long long)ha.idim * ha.jdim * ha.kdim > (long long)hb.idim * hb.jdim * hb.kdim;
  });
  std::vector<std::vector<int>> groups(nclusters);
  std::vector<long long> load(nclusters, 0);
  for (int b : order) {
    const int g = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    groups[g].push_back(b);
    load[g] += (long long)c->hb[b].idim * c->hb[b].jdim * c->hb[b].kdim;
  }
  std::vector<std::vector<int>> koffs(nb);
  for (int b = 0; b < nb; ++b) {
    std::vector<int> nat;
    plane_major_maps(c->hb[b], koffs[b], nat);
  }
  const int nt = L.sweep_nt;
  std::vector<int> base, npl;
  for (int dir = 0; dir < 2; ++dir) {
    std::vector<Chunk> ch;
    std::vector<int> off;
    base.clear();
    npl.clear();
    for (int g = 0; g < nclusters; ++g) {
      int pmax = 0;
      for (int b : groups[g]) pmax = std::max(pmax, c->hb[b].idim + c->hb[b].jdim + c->hb[b].kdim - 2);
      base.push_back((int)off.size());
      npl.push_back(pmax);
      for (int t = 0; t < pmax; ++t) {
        off.push_back((int)ch.size());
        for (int b : groups[g]) {
          const auto& h = c->hb[b];
          const int np_b = h.idim + h.jdim + h.kdim - 2;
          if (t >= np_b) continue;
          const int sp = dir == 0 ? t : np_b - 1 - t;
          const int lo = koffs[b][(size_t)sp * h.kdim], hi = koffs[b][(size_t)(sp + 1) * h.kdim];
          for (int x = lo; x < hi; x += nt) ch.push_back(Chunk{b, std::min(nt, hi - x), (long long)x});
        }
      }
      off.push_back((int)ch.size());
    }
    int rc;
    if ((rc = dev_upload(c, &L.cl_chunks[dir], ch))) return rc;
    if ((rc = dev_upload(c, &L.cl_off[dir], off))) return rc;
  }
  int rc;
  if ((rc = dev_upload(c, &L.cl_base, base))) return rc;
  if ((rc = dev_upload(c, &L.cl_nplanes, npl))) return rc;
  L.cl_count = nclusters;
  return 0;
}

namespace {

// --------------------------------------------------------------------------
// work-list builders
// --------------------------------------------------------------------------
// Line tiles per direction: up to L.lanes_cap grid lines per CTA, fewer where
// the face fluxes of the longest line would not fit the shared-memory budget.
int build_line_tiles(orion_case_t c) {
  auto& L = c->L;
  const int nb = c->nblocks;
  const size_t tsz = (c->prec == ORION_PREC_FP64) ? 8 : 4;
  int rc;
  for (int d = 0; d < 3; ++d) {
    int lmax = 0;
    for (auto& h : c->hb) lmax = std::max(lmax, d == 0 ? h.idim : (d == 1 ? h.jdim : h.kdim));
    L.lmax[d] = lmax;
    int lanes = (int)std::min<size_t>((size_t)L.lanes_cap, kLineSmemBudget / ((size_t)(lmax + 1) * 5 * tsz));
    if (lanes < 1) return fail(ORION_E_UNSUPPORTED, "grid line too long for the line kernels");
    if (d > 0 && lanes >= 8) lanes = lanes / 8 * 8;
    L.lanes[d] = lanes;
    L.line_units[d] = lanes * (lmax + 1);
    std::vector<LineTile> tiles;
    for (int b = 0; b < nb; ++b) {
      const auto& h = c->hb[b];
      const int nlines = d == 0 ? h.jdim * h.kdim : (d == 1 ? h.idim * h.kdim : h.idim * h.jdim);
      for (int s = 0; s < nlines; s += lanes) tiles.push_back(LineTile{b, s, std::min(lanes, nlines - s), 0});
    }
    if ((rc = dev_upload(c, &L.tiles[d], tiles, true))) return rc;
    L.n_tiles[d] = (int)tiles.size();
  }
  return 0;
}

// Tile wavefront sweeps: tiles of 32 x TK grid lines (TK per precision,
// TileShape), per direction in ticket order.  A tile's start in steps is
// 32 J + TK K behind its
// block's first tile, and its upstream tiles (J-1, K) and (J, K-1) start
// strictly earlier, so ordering by start offset (ties by block, then J) is a
// dependency-respecting order for every block at once.
int build_sweep_tiles(orion_case_t c) {
  auto& L = c->L;
  constexpr int TJ = 32;
  const int TK = c->prec == ORION_PREC_FP64 ? TileShape<double>::TK : TileShape<float>::TK;
  L.tile_k = TK;
  int maxn = 0;
  for (int dir = 0; dir < 2; ++dir) {
    struct Item {
      int start, block, J, K;
    };
    std::vector<Item> items;
    std::vector<int> first(c->nblocks + 1, 0);
    for (int b = 0; b < c->nblocks; ++b) {
      const auto& h = c->hb[b];
      const int nJ = (h.jdim + TJ - 1) / TJ, nK = (h.kdim + TK - 1) / TK;
      for (int K = 0; K < nK; ++K)
        for (int J = 0; J < nJ; ++J) items.push_back(Item{TJ * J + TK * K, b, J, K});
    }
    std::stable_sort(items.begin(), items.end(), [](const Item& a, const Item& b) {
      if (a.start != b.start) return a.start < b.start;
      if (a.block != b.block) return a.block < b.block;
      return a.J < b.J;
    });
    // slot of (block, J, K)
    std::vector<long long> base(c->nblocks + 1, 0);
    std::vector<int> nJs(c->nblocks);
    for (int b = 0; b < c->nblocks; ++b) {
      const auto& h = c->hb[b];
      nJs[b] = (h.jdim + TJ - 1) / TJ;
      base[b + 1] = base[b] + (long long)nJs[b] * ((h.kdim + TK - 1) / TK);
    }
    std::vector<int> slot_of((size_t)base[c->nblocks], -1);
    for (size_t q = 0; q < items.size(); ++q)
      slot_of[(size_t)(base[items[q].block] + (long long)items[q].K * nJs[items[q].block] + items[q].J)] = (int)q;
    std::vector<SweepTile> tiles(items.size());
    for (size_t q = 0; q < items.size(); ++q) {
      const Item& it = items[q];
      const auto& h = c->hb[it.block];
      SweepTile& w = tiles[q];
      w = SweepTile{};
      w.block = it.block;
      w.jb = dir == 0 ? it.J * TJ : h.jdim - 1 - it.J * TJ;
      w.kb = dir == 0 ? it.K * TK : h.kdim - 1 - it.K * TK;
      const long long bb = base[it.block];
      w.up_j = it.J > 0 ? slot_of[(size_t)(bb + (long long)it.K * nJs[it.block] + it.J - 1)] : -1;
      w.up_k = it.K > 0 ? slot_of[(size_t)(bb + (long long)(it.K - 1) * nJs[it.block] + it.J)] : -1;
      if ((w.up_j >= 0 && w.up_j >= (int)q) || (w.up_k >= 0 && w.up_k >= (int)q))
        return fail(ORION_E_INVALID, "sweep tile order does not respect the dependencies");
    }
    int rc;
    SweepTile* d = nullptr;
    if ((rc = dev_upload(c, &d, tiles, true))) return rc;
    L.sweep_tiles[dir] = d;
    L.n_sweep_tiles[dir] = (int)tiles.size();
    maxn = std::max(maxn, (int)tiles.size());
  }
  L.tile_ctl_bytes = offsetof(TileCtl, progress) + sizeof(unsigned int) * (size_t)maxn;
  unsigned char* ctl = nullptr;
  int rc;
  if ((rc = dev_alloc(c, &ctl, L.tile_ctl_bytes))) return rc;
  L.tile_ctl = ctl;
  return 0;
}

int build_lists(orion_case_t c, const std::vector<long long>& prim_off, const ExchangePlan& plan) {
  auto& L = c->L;
  const int nb = c->nblocks;
  // pointwise chunks over padded and interior index spaces
  std::vector<Chunk> pad, itr;
  for (int b = 0; b < nb; ++b) {
    const auto& h = c->hb[b];
    for (long long s = 0; s < h.npad; s += kChunk) pad.push_back(Chunk{b, (int)std::min<long long>(kChunk, h.npad - s), s});
    const long long ni = (long long)h.idim * h.jdim * h.kdim;
    for (long long s = 0; s < ni; s += kChunk) itr.push_back(Chunk{b, (int)std::min<long long>(kChunk, ni - s), s});
  }
  int rc;
  if ((rc = dev_upload(c, &L.pad_chunks, pad, true))) return rc;
  L.n_pad_chunks = (int)pad.size();
  if ((rc = dev_upload(c, &L.int_chunks, itr, true))) return rc;
  L.n_int_chunks = (int)itr.size();
  if ((rc = dev_upload(c, &L.pad_base, c->shard.pad_base))) return rc;

  // line-kernel tiles: 16 grid lines per CTA in FP32, 32 in FP64 (autotuned defaults)
  L.lanes_cap = c->prec == ORION_PREC_FP64 ? 32 : 16;
  if ((rc = build_line_tiles(c))) return rc;

  // wavefront launches: launch t of the forward sweeps covers hyperplane t of
  // every block, launch t of the backward sweeps hyperplane nplanes-1-t.
  {
    L.max_planes = 0;
    std::vector<std::vector<int>> koffs(nb);
    for (int b = 0; b < nb; ++b) {
      const auto& h = c->hb[b];
      L.max_planes = std::max(L.max_planes, h.idim + h.jdim + h.kdim - 2);
      std::vector<int> nat;
      plane_major_maps(h, koffs[b], nat);
      const BlockDev<double>* b64 = c->bd64.empty() ? nullptr : &c->bd64[b];
      const BlockDev<float>* b32 = c->bd32.empty() ? nullptr : &c->bd32[b];
      void* dk = b64 ? (void*)b64->koff : (void*)b32->koff;
      void* dn = b64 ? (void*)b64->sk_nat : (void*)b32->sk_nat;
      CUDA_TRY(cudaMemcpyAsync(dk, koffs[b].data(), koffs[b].size() * 4, cudaMemcpyHostToDevice, c->stream));
      CUDA_TRY(cudaMemcpyAsync(dn, nat.data(), nat.size() * 4, cudaMemcpyHostToDevice, c->stream));
      std::vector<int> nbv;
      plane_major_neighbours(h, koffs[b], nat, nbv);
      void* dnb = b64 ? (void*)b64->sk_nb : (void*)b32->sk_nb;
      CUDA_TRY(cudaMemcpyAsync(dnb, nbv.data(), nbv.size() * 4, cudaMemcpyHostToDevice, c->stream));
    }
    // kSweepThreads points per sweep chunk, one per thread
    const int nt = kSweepThreads;
    L.sweep_nt = nt;
    for (int dir = 0; dir < 2; ++dir) {
      std::vector<Chunk> ch;
      std::vector<int> off{0};
      for (int t = 0; t < L.max_planes; ++t) {
        for (int b = 0; b < nb; ++b) {
          const auto& h = c->hb[b];
          const int npl = h.idim + h.jdim + h.kdim - 2;
          if (t >= npl) continue;
          const int sp = dir == 0 ? t : npl - 1 - t;
          const int lo = koffs[b][(size_t)sp * h.kdim], hi = koffs[b][(size_t)(sp + 1) * h.kdim];
          for (int x = lo; x < hi; x += nt) ch.push_back(Chunk{b, std::min(nt, hi - x), (long long)x});
        }
        off.push_back((int)ch.size());
      }
      if ((rc = dev_upload(c, &L.sweep_chunks[dir], ch, true))) return rc;
      if ((rc = dev_upload(c, &L.sweep_off_dev[dir], off))) return rc;
      L.sweep_off[dir] = off;
    }
  }

  // ---------------- halo copy (exchange_bc) ----------------
  // pairs inside this case as arena offsets; pairs with other shards as gather
  // (send) and scatter (receive) lists per peer
  {
    auto off = [&](const ElemRef& e) { return prim_off[e.block] + e.elem; };
    std::vector<long long> hs, hd;
    hs.reserve(plan.halo_src.size());
    hd.reserve(plan.halo_dst.size());
    for (size_t q = 0; q < plan.halo_dst.size(); ++q) {
      hd.push_back(off(plan.halo_dst[q]));
      hs.push_back(off(plan.halo_src[q]));
    }
    if ((rc = dev_upload(c, &L.halo_src, hs))) return rc;
    if ((rc = dev_upload(c, &L.halo_dst, hd))) return rc;
    L.n_halo = (int)hd.size();
    auto& X = c->shard;
    X.halo_send.assign(plan.nranks, nullptr);
    X.halo_recv.assign(plan.nranks, nullptr);
    X.n_halo_send.assign(plan.nranks, 0);
    X.n_halo_recv.assign(plan.nranks, 0);
    for (int r = 0; r < plan.nranks; ++r) {
      std::vector<long long> snd, rcv;
      for (const auto& e : plan.halo_send[r]) snd.push_back(off(e));
      for (const auto& e : plan.halo_recv[r]) rcv.push_back(off(e));
      if ((rc = dev_upload(c, &X.halo_send[r], snd))) return rc;
      if ((rc = dev_upload(c, &X.halo_recv[r], rcv))) return rc;
      X.n_halo_send[r] = (long long)snd.size();
      X.n_halo_recv[r] = (long long)rcv.size();
    }
  }

  // ---------------- physical BC phases ----------------
  {
    std::vector<std::vector<RegionDev>> per_block(nb);
    for (int b = 0; b < nb; ++b) {
      const auto& h = c->hb[b];
      for (const auto& hr : h.regions) {
        if (hr.r.bctype < 0) continue;
        RegionDev R{};
        R.block = b;
        R.type = hr.r.bctype;
        R.s_nd = hr.s_nd;
        R.dir = hr.s_nd - 1;
        R.lr = hr.s_lr;
        if (R.dir < 0) return fail(ORION_E_UNSUPPORTED, "physical BC region is not a face");
        for (int m = 0; m < 3; ++m) {
          R.lo[m] = hr.r.s_st[m] - 1 + NG;
          R.hi[m] = hr.r.s_ed[m] - 1 + NG;
        }
        const long long npts = (long long)std::max(0, R.hi[0] - R.lo[0] + 1) * std::max(0, R.hi[1] - R.lo[1] + 1) *
                               std::max(0, R.hi[2] - R.lo[2] + 1);
        R.npts = (int)npts;
        R.is2d = (R.type == 3 && R.dir != 2 && h.kdim <= 2) ? 1 : 0;
        per_block[b].push_back(R);
      }
    }
    std::vector<RegionDev> regs;
    std::vector<int> phase_list;
    size_t nphase = 0;
    for (auto& v : per_block) nphase = std::max(nphase, v.size());
    L.phase_off.assign(1, 0);
    L.phase_maxpts.clear();
    for (size_t p = 0; p < nphase; ++p) {
      int maxpts = 0;
      for (int b = 0; b < nb; ++b) {
        if (p < per_block[b].size()) {
          phase_list.push_back((int)regs.size());
          regs.push_back(per_block[b][p]);
          maxpts = std::max(maxpts, per_block[b][p].npts);
        }
      }
      L.phase_off.push_back((int)phase_list.size());
      L.phase_maxpts.push_back(maxpts);
    }
    if ((rc = dev_upload(c, &L.regions, regs, true))) return rc;
    if ((rc = dev_upload(c, &L.phase_regions, phase_list, true))) return rc;
  }

  // ---------------- interface residual averaging ----------------
  // own slots are packed here; the slots of other shards arrive after them
  {
    if ((rc = dev_upload(c, &L.pk_block, plan.pk_block, true))) return rc;
    if ((rc = dev_upload(c, &L.pk_idx, plan.pk_idx, true))) return rc;
    L.n_pack = (int)plan.pk_block.size();
    if ((rc = dev_alloc(c, &L.pack, (size_t)plan.n_slots * 5))) return rc;
    if ((rc = dev_upload(c, &L.ap_block, plan.ap_block, true))) return rc;
    if ((rc = dev_upload(c, &L.ap_idx, plan.ap_idx, true))) return rc;
    if ((rc = dev_upload(c, &L.ap_off, plan.ap_off, true))) return rc;
    if ((rc = dev_upload(c, &L.ap_slot, plan.ap_slot, true))) return rc;
    L.n_ap = (int)plan.ap_block.size();
    auto& X = c->shard;
    X.iface_send.assign(plan.nranks, nullptr);
    X.n_iface_send.assign(plan.nranks, 0);
    for (int r = 0; r < plan.nranks; ++r) {
      if ((rc = dev_upload(c, &X.iface_send[r], plan.iface_send[r]))) return rc;
      X.n_iface_send[r] = (long long)plan.iface_send[r].size();
    }
    X.iface_recv_base = plan.iface_recv_base;
    X.iface_recv_n = plan.iface_recv_n;
  }

  if ((rc = dev_alloc(c, &L.partials, (size_t)L.n_int_chunks))) return rc;
  if ((rc = dev_alloc(c, &L.hist, (size_t)kHistCap))) return rc;
  if ((rc = dev_alloc(c, &L.counter, 1))) return rc;
  if ((rc = dev_alloc(c, &L.dtmin, 1))) return rc;
  if ((rc = dev_alloc(c, &L.res_total, 1))) return rc;
  if ((rc = dev_alloc(c, &L.dt_part, (size_t)std::max(L.n_pad_chunks, L.n_int_chunks)))) return rc;
  {
    int* ctl = nullptr;
    if ((rc = dev_alloc(c, &ctl, 4))) return rc;
    L.sweep_ctl = ctl;
  }
  if ((rc = build_sweep_tiles(c))) return rc;
  return 0;
}

const StageOps& ops_for(int precision) { return precision == ORION_PREC_FP64 ? plain_ops() : mixed_ops(); }

template <typename F>
int dispatch(orion_case_t c, F fn) {
  if (!c) return fail(ORION_E_INVALID, "null case");
  int rc = fn(ops_for(c->prec));
  if (rc) return rc;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(ORION_E_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return 0;
}

// Pinned host rings for orion_step_submit, kept for the life of the process:
// freeing pinned memory may synchronise the device, which a request loop that
// retires one case while others run must not do.
static std::mutex g_ring_mu;

// Graph capture, schedule and parameter changes are serialised across host
// threads (a request loop builds cases on some threads while it steps others
// on another); case creation, launches and copies are not: each case has its
// own stream, memory and lists, and process-wide kernel attributes are set
// once (std::call_once).
static std::mutex g_struct_mu;
static std::vector<ResidualOut*> g_free_rings;

static ResidualOut* acquire_hist_ring() {
  {
    std::lock_guard<std::mutex> lk(g_ring_mu);
    if (!g_free_rings.empty()) {
      ResidualOut* r = g_free_rings.back();
      g_free_rings.pop_back();
      return r;
    }
  }
  ResidualOut* r = nullptr;
  if (cudaMallocHost((void**)&r, sizeof(ResidualOut) * kHistCap) != cudaSuccess) return nullptr;
  return r;
}

static void release_hist_ring(ResidualOut* r) {
  std::lock_guard<std::mutex> lk(g_ring_mu);
  g_free_rings.push_back(r);
}

void io_release(orion_case_t c);

void destroy_case(orion_case_t c) {
  if (!c) return;
  if (c->graph) cudaGraphExecDestroy(c->graph);
  io_release(c);
  // stream-ordered frees: no device-wide synchronisation while other cases run
  for (void* p : c->allocs) cudaFreeAsync(p, c->stream);
  if (c->arena) cudaFreeAsync(c->arena, c->stream);
  if (c->d_blocks) cudaFreeAsync(c->d_blocks, c->stream);
  if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
  if (c->hist_host) release_hist_ring(c->hist_host);
  delete c;
}

int field_info(orion_case_t c, int block, int field, void** dptr, int* ncomp, bool* is_storage) {
  if (!c || block < 0 || block >= c->nblocks) return fail(ORION_E_INVALID, "bad block index");
  *is_storage = false;
  const bool f64 = c->prec == ORION_PREC_FP64;
  auto pick = [&](auto& bd) -> int {
    auto& b = bd[block];
    switch (field) {
      case ORION_FIELD_PRIM: *dptr = b.prim; *ncomp = 6; return 0;
      case ORION_FIELD_Q: *dptr = b.q; *ncomp = 5; return 0;
      case ORION_FIELD_DQ: *dptr = b.dq; *ncomp = 5; *is_storage = true; return 0;
      case ORION_FIELD_METRICS: *dptr = (void*)b.metrics; *ncomp = 9; return 0;
      case ORION_FIELD_VOL: *dptr = (void*)b.vol; *ncomp = 1; return 0;
      case ORION_FIELD_DT: *dptr = b.dt; *ncomp = 1; *is_storage = true; return 0;
      case ORION_FIELD_C: *dptr = b.c; *ncomp = 1; *is_storage = true; return 0;
      case ORION_FIELD_MU: *dptr = b.mu; *ncomp = 1; *is_storage = true; return 0;
      default: return fail(ORION_E_INVALID, "bad field id");
    }
  };
  return f64 ? pick(c->bd64) : pick(c->bd32);
}

}  // namespace

// ============================================================================
// C ABI
// ============================================================================
static int capture_step(orion_case_t c, cudaGraph_t* g) {
  CUDA_TRY(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  int rc = ops_for(c->prec).step(c, c->prec == ORION_PREC_FP64);
  cudaError_t e = cudaStreamEndCapture(c->stream, g);
  if (rc) return rc;
  if (e != cudaSuccess) return fail(ORION_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  return 0;
}

static int ensure_graph(orion_case_t c) {
  if (c->graph) return 0;
  std::lock_guard<std::mutex> lk(g_struct_mu);
  cudaGraph_t g;
  int rc = capture_step(c, &g);
  if (rc && (c->L.persist_grid > 0 || c->L.cl_size > 0)) {
    // the cluster / cooperative sweep launch could not be captured: per-hyperplane launches
    cudaGetLastError();
    c->L.persist_grid = 0;
    c->L.cl_size = 0;
    rc = capture_step(c, &g);
  }
  if (rc) return rc;
  size_t nodes = 0;
  cudaGraphGetNodes(g, nullptr, &nodes);
  c->step_launches = (int)nodes;
  cudaError_t e = cudaGraphInstantiate(&c->graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    c->graph = nullptr;
    return fail(ORION_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
  }
  return 0;
}


static void set_params_dev(ParamsDev& P, const orion_params_t& p) {
  P.gamma = p.gamma;
  P.moo = p.moo;
  P.reynolds = p.reynolds;
  P.prl = p.prl;
  P.cfl = p.cfl;
  P.twall = p.twall;
  P.tref = p.tref;
  P.visc = p.visc;
  P.roo = p.roo;
  P.uoo = p.uoo;
  P.voo = p.voo;
  P.woo = p.woo;
  P.poo = p.poo;
  P.too = p.too;
  P.csrv = (double)p.csrv;
  P.nvis = p.nvis;
  P.method = p.method;
}

// Host blocks of a descriptor list, regions classified.
static int host_blocks(int nblocks, const orion_block_desc_t* blocks, std::vector<HostBlock>& hb) {
  hb.assign(nblocks, HostBlock{});
  for (int b = 0; b < nblocks; ++b) {
    auto& h = hb[b];
    h.idim = blocks[b].idim;
    h.jdim = blocks[b].jdim;
    h.kdim = blocks[b].kdim;
    h.nx = h.idim + 2 * NG;
    h.ny = h.jdim + 2 * NG;
    h.nz = h.kdim + 2 * NG;
    h.npad = (long long)h.nx * h.ny * h.nz;
    const int dims[3] = {h.idim, h.jdim, h.kdim};
    for (int r = 0; r < blocks[b].nregions; ++r) {
      HostRegion hr;
      hr.r = blocks[b].regions[r];
      classify_region(hr, dims);
      if (hr.r.bctype < 0 && hr.s_nd == 0) return fail(ORION_E_INVALID, "interface region is not a plane");
      h.regions.push_back(hr);
    }
  }
  return 0;
}

// A case of the blocks `owner[b] == rank` of the global list (owner NULL: all
// blocks, rank 0).  Residual keys and the initial noise use global block
// offsets, so every shard's blocks are numbered as in the whole case.
static int create_case(int nglobal, const orion_block_desc_t* blocks, const int* owner, int rank,
                       const orion_params_t* params, int precision, orion_case_t* out) {
  if (!out || !params) return fail(ORION_E_INVALID, "null argument");
  *out = nullptr;
  if (precision != ORION_PREC_FP64 && precision != ORION_PREC_MIXED) return fail(ORION_E_INVALID, "bad precision");
  int rc = validate_blocks(nglobal, blocks);
  if (rc) return rc;
  std::vector<HostBlock> gb;
  if ((rc = host_blocks(nglobal, blocks, gb))) return rc;
  ExchangePlan plan;
  {
    const std::vector<int> own = owner ? std::vector<int>(owner, owner + nglobal) : std::vector<int>();
    const std::string err = build_exchange_plan(gb, own, rank, plan, NG);
    if (!err.empty()) return fail(ORION_E_INVALID, err);
  }
  if (plan.local.empty()) return fail(ORION_E_INVALID, "shard " + std::to_string(rank) + " owns no block");
  const int nblocks = (int)plan.local.size();
  // every early return below releases what was made so far (stream, arena, lists)
  struct CaseGuard {
    void operator()(orion_case_s* p) const { destroy_case(p); }
  };
  std::unique_ptr<orion_case_s, CaseGuard> c(new orion_case_s());
  c->nblocks = nblocks;
  c->prec = precision;
  CUDA_TRY(cudaGetDevice(&c->device));
  set_params_dev(c->P, *params);
  // The case's own stream first: its memory is allocated and freed in stream
  // order on it, so making or freeing a case never waits for other cases' work.
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(ORION_E_CUDA, "cudaStreamCreate");
  c->own_stream = true;

  // global offsets of every block's interior and padded points
  std::vector<long long> gint(nglobal), gpad(nglobal);
  long long ti = 0, tp = 0;
  for (int g = 0; g < nglobal; ++g) {
    gint[g] = ti;
    gpad[g] = tp;
    ti += (long long)gb[g].idim * gb[g].jdim * gb[g].kdim;
    tp += gb[g].npad;
  }
  auto& X = c->shard;
  X.rank = plan.rank;
  X.nranks = plan.nranks;
  X.global_ids = plan.local;
  X.total_interior_global = ti;
  long long tot = 0;
  for (int g : plan.local) {
    c->hb.push_back(gb[g]);
    X.pad_base.push_back(gpad[g]);
    tot += (long long)gb[g].idim * gb[g].jdim * gb[g].kdim;
  }
  c->total_interior = tot;

  // arena
  const size_t ssz = precision == ORION_PREC_FP64 ? 8 : 4;
  std::vector<size_t> boff(nblocks);
  size_t total = 0;
  for (int b = 0; b < nblocks; ++b) {
    boff[b] = total;
    total += block_bytes(c->hb[b], ssz);
  }
  if (cudaMallocAsync(&c->arena, total, c->stream) != cudaSuccess) {
    cudaGetLastError();
    return fail(ORION_E_NOMEM, "device arena of " + std::to_string(total) + " bytes");
  }
  c->arena_bytes = total;
  CUDA_TRY(cudaMemsetAsync(c->arena, 0, total, c->stream));
  std::vector<long long> prim_off(nblocks);
  if (precision == ORION_PREC_FP64) {
    c->bd64.resize(nblocks);
    for (int b = 0; b < nblocks; ++b) {
      carve_block(static_cast<char*>(c->arena) + boff[b], c->hb[b], c->bd64[b]);
      c->bd64[b].prm = c->P;  // every kernel reads its case's parameters from its block's descriptor
      c->bd64[b].int_base = gint[plan.local[b]];
      prim_off[b] = (c->bd64[b].prim - static_cast<double*>(c->arena));
    }
    CUDA_TRY(cudaMallocAsync(&c->d_blocks, sizeof(BlockDev<double>) * nblocks, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->d_blocks, c->bd64.data(), sizeof(BlockDev<double>) * nblocks, cudaMemcpyHostToDevice,
                             c->stream));
  } else {
    c->bd32.resize(nblocks);
    for (int b = 0; b < nblocks; ++b) {
      carve_block(static_cast<char*>(c->arena) + boff[b], c->hb[b], c->bd32[b]);
      c->bd32[b].prm = c->P;  // every kernel reads its case's parameters from its block's descriptor
      c->bd32[b].int_base = gint[plan.local[b]];
      prim_off[b] = (c->bd32[b].prim - static_cast<double*>(c->arena));
    }
    CUDA_TRY(cudaMallocAsync(&c->d_blocks, sizeof(BlockDev<float>) * nblocks, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->d_blocks, c->bd32.data(), sizeof(BlockDev<float>) * nblocks, cudaMemcpyHostToDevice,
                             c->stream));
  }

  // physical-BC dq mask (set_boundary_dq_zero windows, StateUpdater.cpp:447-468)
  for (int b = 0; b < nblocks; ++b) {
    const auto& h = c->hb[b];
    std::vector<uint8_t> mask((size_t)h.npad, 0);
    for (const auto& hr : h.regions) {
      if (hr.r.bctype <= 0) continue;
      for (int k = hr.r.s_st[2] - 1 + NG; k <= hr.r.s_ed[2] - 1 + NG; ++k)
        for (int j = hr.r.s_st[1] - 1 + NG; j <= hr.r.s_ed[1] - 1 + NG; ++j)
          for (int i = hr.r.s_st[0] - 1 + NG; i <= hr.r.s_ed[0] - 1 + NG; ++i)
            if (i >= 0 && j >= 0 && k >= 0 && i < h.nx && j < h.ny && k < h.nz)
              mask[(size_t)i + (size_t)h.nx * ((size_t)j + (size_t)h.ny * k)] = 1;
    }
    const uint8_t* dmask = precision == ORION_PREC_FP64 ? c->bd64[b].bcmask : c->bd32[b].bcmask;
    CUDA_TRY(cudaMemcpyAsync((void*)dmask, mask.data(), mask.size(), cudaMemcpyHostToDevice, c->stream));
  }

  if ((rc = build_lists(c.get(), prim_off, plan))) return rc;
  rc = ops_for(precision).set_attributes();
  if (!rc) rc = ops_for(precision).persistent_grid(c.get());
  if (rc) return rc;
  // creation-time copies and memsets are ordered on the case's stream
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  *out = c.release();
  return 0;
}

extern "C" {

const char* orion_last_error(void) { return g_last_error.c_str(); }
int orion_abi_version(void) { return ORION_GPU_ABI_VERSION; }

int orion_gpu_init(int device) {
  int n = 0;
  CUDA_TRY(cudaGetDeviceCount(&n));
  if (device < 0 || device >= n) return fail(ORION_E_INVALID, "no such CUDA device");
  CUDA_TRY(cudaSetDevice(device));
  cudaDeviceProp prop;
  CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) return fail(ORION_E_UNSUPPORTED, "this library is built for sm_100a (B200)");
  return 0;
}

size_t orion_footprint_estimate(int nblocks, const orion_block_desc_t* blocks, int precision) {
  if (nblocks <= 0 || !blocks) return 0;
  const size_t ssz = precision == ORION_PREC_FP64 ? 8 : 4;
  size_t s = 0;
  for (int b = 0; b < nblocks; ++b) {
    HostBlock h;
    h.idim = blocks[b].idim;
    h.jdim = blocks[b].jdim;
    h.kdim = blocks[b].kdim;
    h.nx = h.idim + 2 * NG;
    h.ny = h.jdim + 2 * NG;
    h.nz = h.kdim + 2 * NG;
    h.npad = (long long)h.nx * h.ny * h.nz;
    s += block_bytes(h, ssz);
  }
  return s + (s / 64);  // work lists and buffers are a small fraction
}

int orion_case_create(int nblocks, const orion_block_desc_t* blocks, const orion_params_t* params, int precision,
                      orion_case_t* out) {
  return create_case(nblocks, blocks, nullptr, 0, params, precision, out);
}

int orion_case_create_shard(int nblocks, const orion_block_desc_t* blocks, const int* owner, int rank,
                            const orion_params_t* params, int precision, orion_case_t* out) {
  if (!owner) return fail(ORION_E_INVALID, "null owner list");
  return create_case(nblocks, blocks, owner, rank, params, precision, out);
}

int orion_case_destroy(orion_case_t c) {
  if (!c) return 0;
  if (c->group) return fail(ORION_E_INVALID, "the case belongs to a group: destroy the group first");
  cudaStreamSynchronize(c->stream);
  destroy_case(c);
  return 0;
}

int orion_case_set_stream(orion_case_t c, void* stream) {
  if (!c) return fail(ORION_E_INVALID, "null case");
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (c->own_stream) cudaStreamDestroy(c->stream);
  if (stream) {
    c->stream = static_cast<cudaStream_t>(stream);
    c->own_stream = false;
  } else {
    CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    c->own_stream = true;
  }
  if (c->graph) {
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  return 0;
}

}  // extern "C"

namespace {

template <typename S>
int refresh_blocks(orion_case_t c, std::vector<BlockDev<S>>& bd) {
  for (auto& b : bd) b.prm = c->P;
  if (bd.empty()) return 0;
  CUDA_TRY(cudaMemcpyAsync(c->d_blocks, bd.data(), sizeof(BlockDev<S>) * bd.size(), cudaMemcpyHostToDevice, c->stream));
  if (c->group) {
    const auto& mem = c->group->members;
    const size_t m = std::find(mem.begin(), mem.end(), c) - mem.begin();
    auto* gb = static_cast<BlockDev<S>*>(c->group->proxy->d_blocks) + c->group->block_off[m];
    CUDA_TRY(cudaMemcpyAsync(gb, bd.data(), sizeof(BlockDev<S>) * bd.size(), cudaMemcpyHostToDevice, c->stream));
  }
  return 0;
}

int refresh_block_params(orion_case_t c) {
  return c->prec == ORION_PREC_FP64 ? refresh_blocks<double>(c, c->bd64) : refresh_blocks<float>(c, c->bd32);
}

}  // namespace

extern "C" {

int orion_case_set_params(orion_case_t c, const orion_params_t* params) {
  if (!c || !params) return fail(ORION_E_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(g_struct_mu);
  set_params_dev(c->P, *params);
  // the copies in the block descriptors the kernels read (the case's, and its
  // group's), after the launches already enqueued
  int rc = refresh_block_params(c);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (c->graph) {  // the captured step holds the old values: capture again on the next step
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  return 0;
}

static void current_schedule(orion_case_t c, orion_schedule_t* s) {
  s->sweep_form = c->L.tiles_on ? ORION_SWEEP_TILES
                  : c->L.cl_size > 0 ? ORION_SWEEP_CLUSTER
                  : (c->L.persist_grid > 0 ? ORION_SWEEP_GRID : ORION_SWEEP_PLANES);
  s->cluster_size = c->L.cl_size;
  s->lanes = c->L.lanes_cap;
  s->ms_per_step = 0.f;
}

static int apply_schedule(orion_case_t c, const orion_schedule_t& s) {
  if (s.lanes < 1 || s.lanes > 32) return fail(ORION_E_INVALID, "lanes must be 1..32");
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (c->graph) {
    cudaGraphExecDestroy(c->graph);
    c->graph = nullptr;
  }
  int rc = 0;
  if (s.lanes != c->L.lanes_cap) {
    c->L.lanes_cap = s.lanes;
    if ((rc = build_line_tiles(c))) return rc;
  }
  rc = ops_for(c->prec).schedule(c, s.sweep_form, s.cluster_size);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return rc;
}

int orion_case_set_schedule(orion_case_t c, const orion_schedule_t* s) {
  if (!c || !s) return fail(ORION_E_INVALID, "null argument");
  std::lock_guard<std::mutex> lk(g_struct_mu);
  return apply_schedule(c, *s);
}

int orion_case_get_schedule(orion_case_t c, orion_schedule_t* s) {
  if (!c || !s) return fail(ORION_E_INVALID, "null argument");
  current_schedule(c, s);
  return 0;
}

static int launch_steps(orion_case_t c, int nsteps);
static int sweep_status(orion_case_t c);
static int enqueue_hist_copy(orion_case_t c, int nsteps, cudaStream_t st = nullptr);

int orion_case_autotune(orion_case_t c, int steps_per_trial, orion_schedule_t* trials, int cap, int* ntrials,
                        orion_schedule_t* best) {
  if (!c || !ntrials || !best || steps_per_trial < 1 || (cap > 0 && !trials))
    return fail(ORION_E_INVALID, "bad arguments");
  if (c->pending_n > 0) return fail(ORION_E_INVALID, "submitted steps have not been polled");
  *ntrials = 0;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  // the state between steps is prim (every other field is recomputed from it)
  std::vector<double*> prim(c->nblocks);
  size_t tot = 0;
  for (int b = 0; b < c->nblocks; ++b) {
    void* d;
    int nc;
    bool st;
    int rc = field_info(c, b, ORION_FIELD_PRIM, &d, &nc, &st);
    if (rc) return rc;
    prim[b] = static_cast<double*>(d);
    tot += (size_t)6 * c->hb[b].npad;
  }
  double* save = nullptr;
  if (cudaMallocAsync((void**)&save, tot * sizeof(double), c->stream) != cudaSuccess) {
    cudaGetLastError();
    return fail(ORION_E_NOMEM, "autotune state copy");
  }
  auto copy_state = [&](bool out) -> int {
    size_t o = 0;
    for (int b = 0; b < c->nblocks; ++b) {
      const size_t n = (size_t)6 * c->hb[b].npad;
      CUDA_TRY(cudaMemcpyAsync(out ? save + o : prim[b], out ? prim[b] : save + o, n * sizeof(double),
                               cudaMemcpyDeviceToDevice, c->stream));
      o += n;
    }
    return 0;
  };
  int counter = 0;
  CUDA_TRY(cudaMemcpy(&counter, c->L.counter, sizeof(int), cudaMemcpyDeviceToHost));
  const long long steps_done = c->steps_done, hist_count = c->hist_count;
  int rc = copy_state(true);
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));

  auto trial = [&](orion_schedule_t s) -> int {
    int r;
    {
      std::lock_guard<std::mutex> lk(g_struct_mu);
      r = apply_schedule(c, s);
    }
    if (r) return r;
    if ((r = launch_steps(c, 1))) return r;  // capture + warm-up
    if ((r = copy_state(false))) return r;
    CUDA_TRY(cudaEventRecord(e0, c->stream));
    if ((r = launch_steps(c, steps_per_trial))) return r;
    CUDA_TRY(cudaEventRecord(e1, c->stream));
    CUDA_TRY(cudaEventSynchronize(e1));
    if ((r = sweep_status(c))) return r;
    float ms = 0.f;
    CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
    if ((r = copy_state(false))) return r;
    s.ms_per_step = ms / steps_per_trial;
    if (*ntrials < cap) trials[*ntrials] = s;
    ++*ntrials;
    if (best->ms_per_step <= 0.f || s.ms_per_step < best->ms_per_step) *best = s;
    return 0;
  };
  orion_schedule_t start;
  current_schedule(c, &start);
  best->ms_per_step = 0.f;
  // phase 1: grid lines per CTA of the line kernels, with the current sweep form
  for (int lanes : {8, 16, 32}) {
    if (rc) break;
    orion_schedule_t s = start;
    s.lanes = lanes;
    rc = trial(s);
  }
  // phase 2: every sweep form, with the best lanes
  const orion_schedule_t forms[5] = {{ORION_SWEEP_TILES, 0, 0, 0.f}, {ORION_SWEEP_CLUSTER, 16, 0, 0.f},
                                     {ORION_SWEEP_CLUSTER, 8, 0, 0.f}, {ORION_SWEEP_GRID, 0, 0, 0.f},
                                     {ORION_SWEEP_PLANES, 0, 0, 0.f}};
  for (const auto& f : forms) {
    if (rc) break;
    if (f.sweep_form == start.sweep_form && (f.sweep_form != ORION_SWEEP_CLUSTER || f.cluster_size == start.cluster_size))
      continue;  // timed in phase 1
    orion_schedule_t s = f;
    s.lanes = best->lanes;
    const int r = trial(s);
    if (r == ORION_E_UNSUPPORTED) continue;  // this device cannot hold that form
    rc = r;
  }
  // keep the fastest; the solution is where it was before tuning
  if (!rc) {
    std::lock_guard<std::mutex> lk(g_struct_mu);
    rc = apply_schedule(c, *best);
  }
  if (!rc) rc = copy_state(false);
  if (!rc) {
    cudaMemcpyAsync(c->L.counter, &counter, sizeof(int), cudaMemcpyHostToDevice, c->stream);
    cudaStreamSynchronize(c->stream);
  }
  c->steps_done = steps_done;
  c->hist_count = hist_count;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(save, c->stream);
  cudaStreamSynchronize(c->stream);
  return rc;
}

int orion_case_sync(orion_case_t c) {
  if (!c) return fail(ORION_E_INVALID, "null case");
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return 0;
}

int orion_case_stream(orion_case_t c, void** stream) {
  if (!c || !stream) return fail(ORION_E_INVALID, "null argument");
  *stream = (void*)c->stream;
  return 0;
}

int orion_case_step_launches(orion_case_t c, int* n) {
  if (!c || !n) return fail(ORION_E_INVALID, "null argument");
  int rc = ensure_graph(c);
  if (rc) return rc;
  *n = c->step_launches;
  return 0;
}

int orion_case_sweep_schedule(orion_case_t c, int out[5]) {
  if (!c || !out) return fail(ORION_E_INVALID, "null argument");
  const auto& L = c->L;
  out[0] = L.tiles_on ? 3 : (L.cl_size > 0 ? 2 : (L.persist_grid > 0 ? 1 : 0));
  out[1] = L.tiles_on ? L.n_sweep_tiles[0] : (L.cl_size > 0 ? L.cl_count : L.persist_grid);
  out[2] = L.cl_size;
  out[3] = L.tiles_on ? 32 * L.tile_k : L.sweep_nt;
  out[4] = L.max_planes;
  return 0;
}

int orion_case_footprint(orion_case_t c, size_t* bytes) {
  if (!c || !bytes) return fail(ORION_E_INVALID, "null argument");
  *bytes = c->arena_bytes;
  return 0;
}

int orion_case_upload(orion_case_t c, int block, int field, const double* host) {
  void* d;
  int nc;
  bool st;
  int rc = field_info(c, block, field, &d, &nc, &st);
  if (rc) return rc;
  if (!host) return fail(ORION_E_INVALID, "null host pointer");
  const size_t n = (size_t)c->hb[block].npad * nc;
  // Copies go on the case's own stream: a cudaMemcpy from pageable memory on
  // the legacy stream may return before the data reach the device, and kernels
  // on the case's (non-blocking) stream would not be ordered after it.
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  if (st && c->prec != ORION_PREC_FP64) {
    std::vector<float> tmp(n);
    for (size_t i = 0; i < n; ++i) tmp[i] = (float)host[i];
    CUDA_TRY(cudaMemcpyAsync(d, tmp.data(), n * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
  } else {
    CUDA_TRY(cudaMemcpyAsync(d, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  }
  if (field == ORION_FIELD_METRICS || field == ORION_FIELD_VOL) {
    rc = dispatch(c, [&](const StageOps& o) { return o.skew_static(c, block); });
    if (rc) return rc;
  }
  if (field == ORION_FIELD_PRIM) {
    rc = dispatch(c, [&](const StageOps& o) { return o.prim_shadow(c, block); });
    if (rc) return rc;
  }
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return 0;
}

int orion_case_download(orion_case_t c, int block, int field, double* host) {
  void* d;
  int nc;
  bool st;
  int rc = field_info(c, block, field, &d, &nc, &st);
  if (rc) return rc;
  if (!host) return fail(ORION_E_INVALID, "null host pointer");
  const size_t n = (size_t)c->hb[block].npad * nc;
  if (st && c->prec != ORION_PREC_FP64) {
    std::vector<float> tmp(n);
    CUDA_TRY(cudaMemcpyAsync(tmp.data(), d, n * sizeof(float), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (size_t i = 0; i < n; ++i) host[i] = (double)tmp[i];
  } else {
    CUDA_TRY(cudaMemcpyAsync(host, d, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
  }
  return 0;
}

int orion_case_grid_metrics(orion_case_t c, int block, const double* x, const double* y, const double* z, int gcl) {
  if (!c || block < 0 || block >= c->nblocks || !x || !y || !z) return fail(ORION_E_INVALID, "bad arguments");
  const auto& h = c->hb[block];
  const long long n = (long long)h.idim * h.jdim * h.kdim;
  void* dmet;
  void* dvol;
  int nc;
  bool st;
  int rc = field_info(c, block, ORION_FIELD_METRICS, &dmet, &nc, &st);
  if (!rc) rc = field_info(c, block, ORION_FIELD_VOL, &dvol, &nc, &st);
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  double* dxyz = nullptr;
  double* dD = nullptr;
  if (cudaMallocAsync((void**)&dxyz, sizeof(double) * 3 * n, c->stream) != cudaSuccess ||
      cudaMallocAsync((void**)&dD, sizeof(double) * 9 * n, c->stream) != cudaSuccess) {
    cudaGetLastError();
    if (dxyz) cudaFreeAsync(dxyz, c->stream);
    return fail(ORION_E_NOMEM, "grid metrics scratch");
  }
  CUDA_TRY(cudaMemcpyAsync(dxyz, x, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(cudaMemcpyAsync(dxyz + n, y, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(cudaMemcpyAsync(dxyz + 2 * n, z, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  CUDA_TRY(cudaMemsetAsync(dmet, 0, sizeof(double) * 9 * (size_t)h.npad, c->stream));  // ghosts stay zero
  CUDA_TRY(cudaMemsetAsync(dvol, 0, sizeof(double) * (size_t)h.npad, c->stream));
  const gm::GridDims G{h.idim, h.jdim, h.kdim, n};
  const int nblk = (int)((n + kThreads - 1) / kThreads);
  gm::k_coord_derivs<<<nblk, kThreads, 0, c->stream>>>(G, dxyz, dD);
  gm::k_metrics_final<<<nblk, kThreads, 0, c->stream>>>(G, h.nx, h.ny, h.npad, gcl, dxyz, dD,
                                                       static_cast<double*>(dmet), static_cast<double*>(dvol));
  CUDA_TRY(cudaGetLastError());
  cudaFreeAsync(dxyz, c->stream);
  cudaFreeAsync(dD, c->stream);
  rc = dispatch(c, [&](const StageOps& o) { return o.skew_static(c, block); });
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return 0;
}

int orion_case_pack_output(orion_case_t c, int block, float* host) {
  if (!c || block < 0 || block >= c->nblocks || !host) return fail(ORION_E_INVALID, "bad arguments");
  const auto& h = c->hb[block];
  const long long n = (long long)h.idim * h.jdim * h.kdim;
  void* dprim;
  int nc;
  bool st;
  int rc = field_info(c, block, ORION_FIELD_PRIM, &dprim, &nc, &st);
  if (rc) return rc;
  float* stage = nullptr;
  if (cudaMallocAsync((void**)&stage, sizeof(float) * 7 * n, c->stream) != cudaSuccess) {
    cudaGetLastError();
    return fail(ORION_E_NOMEM, "output staging buffer");
  }
  out::k_pack_output<<<148 * 4, kThreads, 0, c->stream>>>(static_cast<const double*>(dprim), h.npad, h.idim, h.jdim,
                                                          h.kdim, h.nx, h.ny, c->P.gamma, stage);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(host, stage, sizeof(float) * 7 * n, cudaMemcpyDeviceToHost, c->stream);
  cudaFreeAsync(stage, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return fail(ORION_E_CUDA, std::string("pack output: ") + cudaGetErrorString(e));
  return 0;
}

int orion_case_init_flow(orion_case_t c, uint64_t seed, double amp) {
  return dispatch(c, [&](const StageOps& o) {
    int rc = o.init_flow(c, seed, amp);
    for (int b = 0; !rc && b < c->nblocks; ++b) rc = o.prim_shadow(c, b);
    return rc;
  });
}

int orion_exchange_bc(orion_case_t c) {
  return dispatch(c, [&](const StageOps& o) { return o.exchange(c); });
}
int orion_apply_physical_bc(orion_case_t c) {
  return dispatch(c, [&](const StageOps& o) { return o.bc(c); });
}
int orion_update_flow_states(orion_case_t c) {
  return dispatch(c, [&](const StageOps& o) { return o.state(c, false, true); });
}
int orion_calculate_time_step(orion_case_t c) {
  return dispatch(c, [&](const StageOps& o) { return o.timestep(c); });
}
int orion_compute_viscous_rhs(orion_case_t c) {
  return dispatch(c, [&](const StageOps& o) { return o.viscous(c); });
}
int orion_average_interface_residuals(orion_case_t c) {
  if (c && c->shard.nranks > 1)
    return fail(ORION_E_INVALID, "a shard averages with orion_shard_average_begin, the exchange and orion_shard_average_end");
  return dispatch(c, [&](const StageOps& o) { return o.average(c); });
}
int orion_compute_inviscid_rhs(orion_case_t c) {
  return dispatch(c, [&](const StageOps& o) { return o.inviscid(c); });
}
int orion_update_solution(orion_case_t c) {
  return dispatch(c, [&](const StageOps& o) { return o.update(c, false); });
}

static int read_hist(orion_case_t c, long long first, int n, orion_residual_t* out) {
  std::vector<ResidualOut> h(kHistCap);
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  CUDA_TRY(cudaMemcpy(h.data(), c->L.hist, sizeof(ResidualOut) * kHistCap, cudaMemcpyDeviceToHost));
  for (int s = 0; s < n; ++s) {
    const ResidualOut& r = h[(size_t)((first + s) % kHistCap)];
    out[s].rms = r.rms;
    out[s].max = r.max;
    for (int m = 0; m < 5; ++m) out[s].max_loc[m] = r.loc[m];
    out[s].pad = 0;
    out[s].phydtime = r.phydtime;
  }
  return 0;
}

int orion_residual_compute(orion_case_t c, orion_residual_t* out) {
  if (!c || !out) return fail(ORION_E_INVALID, "null argument");
  if (c->shard.nranks > 1) return fail(ORION_E_INVALID, "a shard's residual is orion_shard_residual, reduced over the shards");
  int cnt = 0;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  CUDA_TRY(cudaMemcpy(&cnt, c->L.counter, sizeof(int), cudaMemcpyDeviceToHost));
  int rc = dispatch(c, [&](const StageOps& o) { return o.residual(c); });
  if (rc) return rc;
  c->hist_count = cnt + 1;
  return read_hist(c, cnt, 1, out);
}

int orion_phydtime(orion_case_t c, double* out) {
  if (!c || !out) return fail(ORION_E_INVALID, "null argument");
  unsigned long long bits = 0;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  CUDA_TRY(cudaMemcpy(&bits, c->L.dtmin, sizeof(bits), cudaMemcpyDeviceToHost));
  double v;
  std::memcpy(&v, &bits, sizeof(v));
  *out = v;
  return 0;
}

static int launch_steps(orion_case_t c, int nsteps) {
  if (c->shard.nranks > 1)
    return fail(ORION_E_INVALID, "a shard steps through the per-stage entry points and the shard exchanges");
  int rc = ensure_graph(c);
  if (rc) return rc;
  for (int s = 0; s < nsteps; ++s) CUDA_TRY(cudaGraphLaunch(c->graph, c->stream));
  c->steps_done += nsteps;
  return 0;
}

int orion_step_async(orion_case_t c, int nsteps) {
  if (!c || nsteps < 0) return fail(ORION_E_INVALID, "bad arguments");
  int rc = launch_steps(c, nsteps);
  if (rc) return rc;
  if (c->hist_count >= 0) c->hist_count += nsteps;
  return 0;
}

// Reads the sweep barrier's error flag (the stream is idle).
static int sweep_status(orion_case_t c) {
  if (!c->L.sweep_ctl) return 0;
  int ctl[2] = {0, 0};
  CUDA_TRY(cudaMemcpy(ctl, c->L.sweep_ctl, sizeof(ctl), cudaMemcpyDeviceToHost));
  if (ctl[1]) {
    CUDA_TRY(cudaMemsetAsync(c->L.sweep_ctl, 0, sizeof(ctl), c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return fail(ORION_E_TIMEOUT, "a bounded wait of the implicit sweeps (grid barrier or tile progress) gave up waiting");
  }
  return 0;
}

int orion_step(orion_case_t c, int nsteps, orion_residual_t* hist) {
  if (!c || nsteps < 0) return fail(ORION_E_INVALID, "bad arguments");
  int cnt = 0;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  CUDA_TRY(cudaMemcpy(&cnt, c->L.counter, sizeof(int), cudaMemcpyDeviceToHost));
  int done = 0;
  while (done < nsteps) {
    const int n = std::min(nsteps - done, kHistCap);
    int rc = launch_steps(c, n);
    if (rc) return rc;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    rc = sweep_status(c);
    if (rc) return rc;
    if (hist) {
      rc = read_hist(c, (long long)cnt + done, n, hist + done);
      if (rc) return rc;
    }
    done += n;
  }
  c->hist_count = (long long)cnt + nsteps;
  CUDA_TRY(cudaGetLastError());
  return 0;
}

int orion_step_submit(orion_case_t c, int nsteps) {
  if (!c || nsteps < 0) return fail(ORION_E_INVALID, "bad arguments");
  if (c->pending_n + nsteps > kHistCap)
    return fail(ORION_E_INVALID, "more unpolled steps than the history ring holds (4096)");
  if (!c->hist_host && !(c->hist_host = acquire_hist_ring()))
    return fail(ORION_E_NOMEM, "pinned history ring");
  if (c->hist_count < 0) {  // once: learn the device counter
    int cnt = 0;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    CUDA_TRY(cudaMemcpy(&cnt, c->L.counter, sizeof(int), cudaMemcpyDeviceToHost));
    c->hist_count = cnt;
  }
  if (nsteps == 0) return 0;
  int rc = launch_steps(c, nsteps);
  if (rc) return rc;
  return enqueue_hist_copy(c, nsteps);
}

// Copies the history entries of the last nsteps steps (enqueued on the case's
// stream) into the case's pinned ring and records them as pending.
static int enqueue_hist_copy(orion_case_t c, int nsteps, cudaStream_t st) {
  // on the case's stream unless another stream ordered after the steps is given;
  // the new entries sit at ring positions [first, first + nsteps) mod kHistCap
  const long long first = c->hist_count;
  long long pos = first % kHistCap;
  int left = nsteps;
  while (left > 0) {
    const int n = (int)std::min<long long>(left, kHistCap - pos);
    CUDA_TRY(cudaMemcpyAsync(c->hist_host + pos, c->L.hist + pos, sizeof(ResidualOut) * n, cudaMemcpyDeviceToHost,
                             st ? st : c->stream));
    left -= n;
    pos = 0;
  }
  if (c->pending_n == 0) c->pending_first = first;
  c->pending_n += nsteps;
  c->hist_count += nsteps;
  return 0;
}

int orion_case_poll(orion_case_t c, orion_residual_t* out, int cap, int* n) {
  if (!c || !n || (cap > 0 && !out)) return fail(ORION_E_INVALID, "null argument");
  *n = 0;
  if (c->io) {  // pipelined I/O copies the history on the output copy stream
    const cudaError_t qo = cudaStreamQuery(c->io->out);
    if (qo == cudaErrorNotReady) return 0;
    if (qo != cudaSuccess) {
      cudaGetLastError();
      return fail(ORION_E_CUDA, std::string("output copy stream: ") + cudaGetErrorString(qo));
    }
  }
  const cudaError_t q = cudaStreamQuery(c->stream);
  if (q == cudaErrorNotReady) return 0;
  if (q != cudaSuccess) {
    cudaGetLastError();
    return fail(ORION_E_CUDA, std::string("case stream: ") + cudaGetErrorString(q));
  }
  int rc = sweep_status(c->group ? c->group->proxy : c);
  if (rc) return rc;
  const int take = std::min(cap, c->pending_n);
  for (int s = 0; s < take; ++s) {
    const ResidualOut& r = c->hist_host[(c->pending_first + s) % kHistCap];
    out[s].rms = r.rms;
    out[s].max = r.max;
    for (int m = 0; m < 5; ++m) out[s].max_loc[m] = r.loc[m];
    out[s].pad = 0;
    out[s].phydtime = r.phydtime;
  }
  c->pending_first += take;
  c->pending_n -= take;
  *n = take;
  return 1;
}

}  // extern "C"

// ---- pipelined host I/O (orion_io_*) -------------------------------------
namespace {

// Staging copies on the SMs, every block's in one launch (blockIdx.y is the
// block): a cudaMemcpyAsync between device buffers would queue on the copy
// engines behind the host copies of the neighbouring steps, and one launch
// per block left the SMs mostly idle between small copies.  Installing an
// input also writes the mixed path's FP32 prim shadow from the same loads
// (the values k_prim_shadow writes).  Spans start 16-byte aligned.
__global__ void k_io_copy(const IoSpan* __restrict__ spans) {
  const IoSpan sp = spans[blockIdx.y];
  const long long n2 = sp.n / 2;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const double2* src = reinterpret_cast<const double2*>(sp.src);
  double2* dst = reinterpret_cast<double2*>(sp.dst);
  float2* sh = reinterpret_cast<float2*>(sp.shadow);
  for (long long i = t; i < n2; i += stride) {
    const double2 v = src[i];
    dst[i] = v;
    if (sh) sh[i] = make_float2((float)v.x, (float)v.y);
  }
  if (t == 0 && (sp.n & 1)) {
    const double v = sp.src[sp.n - 1];
    sp.dst[sp.n - 1] = v;
    if (sp.shadow) sp.shadow[sp.n - 1] = (float)v;
  }
}

int io_copy(const IoSpan* spans, int nspans, long long max_n, cudaStream_t st) {
  if (nspans <= 0) return 0;
  const long long want = (max_n / 2 + 255) / 256;
  const int gx = (int)std::max<long long>(1, std::min<long long>(want, std::max(1, 148 * 16 / nspans)));
  k_io_copy<<<dim3(gx, nspans), 256, 0, st>>>(spans);
  CUDA_TRY(cudaGetLastError());
  return 0;
}

void io_free_buffers(IoPipe* io) {
  for (int k = 0; k < 2; ++k) {
    if (io->stage_in[k]) cudaFree(io->stage_in[k]);
    if (io->stage_out[k]) cudaFree(io->stage_out[k]);
    if (io->spans_in[k]) cudaFree(io->spans_in[k]);
    if (io->spans_out[k]) cudaFree(io->spans_out[k]);
    io->stage_in[k] = io->stage_out[k] = nullptr;
    io->spans_in[k] = io->spans_out[k] = nullptr;
  }
}

int io_pipe(orion_case_t c, IoPipe** out) {
  if (c->io) {
    *out = c->io;
    return 0;
  }
  if (c->group) return fail(ORION_E_UNSUPPORTED, "a grouped case steps through its group");
  if (c->shard.nranks > 1) return fail(ORION_E_UNSUPPORTED, "a shard exchanges through its own calls");
  auto io = std::make_unique<IoPipe>();
  size_t total = 0;
  for (int b = 0; b < c->nblocks; ++b) {
    io->off.push_back(total);
    total += ((size_t)c->hb[b].npad * 6 + 1) / 2 * 2;  // 16-byte aligned starts
  }
  io->put.assign(c->nblocks, 0);
  std::vector<void*> prim(c->nblocks);
  for (int b = 0; b < c->nblocks; ++b) {
    int nc;
    bool st;
    int rc = field_info(c, b, ORION_FIELD_PRIM, &prim[b], &nc, &st);
    if (rc) return rc;
    io->max_n = std::max(io->max_n, 6 * (long long)c->hb[b].npad);
  }
  for (int k = 0; k < 2; ++k) {
    if (cudaMalloc((void**)&io->stage_in[k], total * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&io->stage_out[k], total * sizeof(double)) != cudaSuccess ||
        cudaMalloc((void**)&io->spans_in[k], sizeof(IoSpan) * c->nblocks) != cudaSuccess ||
        cudaMalloc((void**)&io->spans_out[k], sizeof(IoSpan) * c->nblocks) != cudaSuccess) {
      cudaGetLastError();
      io_free_buffers(io.get());
      return fail(ORION_E_NOMEM, "pipelined I/O staging");
    }
    std::vector<IoSpan> sin(c->nblocks), sout(c->nblocks);
    for (int b = 0; b < c->nblocks; ++b) {
      const long long n = 6 * (long long)c->hb[b].npad;
      float* sh = c->prec == ORION_PREC_FP64 ? nullptr : c->bd32[b].prim_f;
      sin[b] = IoSpan{io->stage_in[k] + io->off[b], static_cast<double*>(prim[b]), sh, n};
      sout[b] = IoSpan{static_cast<const double*>(prim[b]), io->stage_out[k] + io->off[b], nullptr, n};
    }
    CUDA_TRY(cudaMemcpy(io->spans_in[k], sin.data(), sizeof(IoSpan) * c->nblocks, cudaMemcpyHostToDevice));
    CUDA_TRY(cudaMemcpy(io->spans_out[k], sout.data(), sizeof(IoSpan) * c->nblocks, cudaMemcpyHostToDevice));
    for (cudaEvent_t* e : {&io->in_ready[k], &io->in_free[k], &io->out_ready[k], &io->out_free[k]})
      CUDA_TRY(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  }
  CUDA_TRY(cudaStreamCreateWithFlags(&io->in, cudaStreamNonBlocking));
  CUDA_TRY(cudaStreamCreateWithFlags(&io->out, cudaStreamNonBlocking));
  c->io = io.release();
  *out = c->io;
  return 0;
}

void io_release(orion_case_t c) {
  IoPipe* io = c->io;
  if (!io) return;
  if (io->in) cudaStreamSynchronize(io->in);
  if (io->out) cudaStreamSynchronize(io->out);
  if (c->stream) cudaStreamSynchronize(c->stream);
  io_free_buffers(io);
  for (int k = 0; k < 2; ++k)
    for (cudaEvent_t e : {io->in_ready[k], io->in_free[k], io->out_ready[k], io->out_free[k]})
      if (e) cudaEventDestroy(e);
  if (io->in) cudaStreamDestroy(io->in);
  if (io->out) cudaStreamDestroy(io->out);
  delete io;
  c->io = nullptr;
}

}  // namespace

extern "C" {

int orion_last_residual(orion_case_t c, orion_residual_t* out) {
  if (!c || !out) return fail(ORION_E_INVALID, "null argument");
  int cnt = 0;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  CUDA_TRY(cudaMemcpy(&cnt, c->L.counter, sizeof(int), cudaMemcpyDeviceToHost));
  if (cnt <= 0) return fail(ORION_E_INVALID, "no step has run");
  return read_hist(c, cnt - 1, 1, out);
}


int orion_io_put(orion_case_t c, int block, const double* host) {
  if (!c || !host || block < 0 || block >= c->nblocks) return fail(ORION_E_INVALID, "bad arguments");
  IoPipe* io = nullptr;
  int rc = io_pipe(c, &io);
  if (rc) return rc;
  const int k = io->put_buf;
  if (io->put_waits[k]) {  // the io step that installed this buffer last must be done with it
    CUDA_TRY(cudaStreamWaitEvent(io->in, io->in_free[k], 0));
    io->put_waits[k] = false;
  }
  CUDA_TRY(cudaMemcpyAsync(io->stage_in[k] + io->off[block], host, sizeof(double) * 6 * (size_t)c->hb[block].npad,
                           cudaMemcpyHostToDevice, io->in));
  io->put[block] = 1;
  return 0;
}

int orion_io_step(orion_case_t c, int nsteps) {
  if (!c || nsteps < 0) return fail(ORION_E_INVALID, "bad arguments");
  IoPipe* io = nullptr;
  int rc = io_pipe(c, &io);
  if (rc) return rc;
  if (c->pending_n + nsteps > kHistCap)
    return fail(ORION_E_INVALID, "more unpolled steps than the history ring holds (4096)");
  // install the blocks put since the last io step, from the input buffer they filled
  bool any = false;
  for (int b = 0; b < c->nblocks; ++b) any = any || io->put[b];
  if (any) {
    const int k = io->put_buf;
    CUDA_TRY(cudaEventRecord(io->in_ready[k], io->in));
    CUDA_TRY(cudaStreamWaitEvent(c->stream, io->in_ready[k], 0));
    // runs of consecutive put blocks, one launch each (one launch when all were put)
    for (int b = 0; b < c->nblocks;) {
      if (!io->put[b]) {
        ++b;
        continue;
      }
      int e = b;
      while (e < c->nblocks && io->put[e]) io->put[e++] = 0;
      if ((rc = io_copy(io->spans_in[k] + b, e - b, io->max_n, c->stream))) return rc;
      b = e;
    }
    CUDA_TRY(cudaEventRecord(io->in_free[k], c->stream));
    io->put_waits[k] = true;
    io->put_buf = k ^ 1;  // the next puts fill the other buffer while this step runs
  }
  if (!c->hist_host && !(c->hist_host = acquire_hist_ring())) return fail(ORION_E_NOMEM, "pinned history ring");
  if (c->hist_count < 0) {  // once: learn the device counter
    int cnt = 0;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    CUDA_TRY(cudaMemcpy(&cnt, c->L.counter, sizeof(int), cudaMemcpyDeviceToHost));
    c->hist_count = cnt;
  }
  if (nsteps > 0 && (rc = launch_steps(c, nsteps))) return rc;
  // the gets issued so far from the last filled buffer end where out_free says
  if (io->get_buf >= 0 && io->got[io->get_buf]) {
    CUDA_TRY(cudaEventRecord(io->out_free[io->get_buf], io->out));
    io->step_waits[io->get_buf] = true;
    io->got[io->get_buf] = false;
  }
  // the result into the other output buffer, once its own last gets have read it
  const int j = io->out_buf;
  if (io->step_waits[j]) {
    CUDA_TRY(cudaStreamWaitEvent(c->stream, io->out_free[j], 0));
    io->step_waits[j] = false;
  }
  if ((rc = io_copy(io->spans_out[j], c->nblocks, io->max_n, c->stream))) return rc;
  CUDA_TRY(cudaEventRecord(io->out_ready[j], c->stream));
  // the residual history leaves with the state, on the output copy stream: on
  // the case's stream that small copy would queue on the copy engine behind
  // the previous state's copy to the host and hold up the next step
  CUDA_TRY(cudaStreamWaitEvent(io->out, io->out_ready[j], 0));
  if (nsteps > 0 && (rc = enqueue_hist_copy(c, nsteps, io->out))) return rc;
  io->get_buf = j;
  io->out_buf = j ^ 1;
  return 0;
}

int orion_io_get(orion_case_t c, int block, double* host) {
  if (!c || !host || block < 0 || block >= c->nblocks) return fail(ORION_E_INVALID, "bad arguments");
  IoPipe* io = c->io;
  if (!io || io->get_buf < 0) return fail(ORION_E_INVALID, "no io step has run");
  const int j = io->get_buf;  // the output stream already waits for this buffer's staging
  CUDA_TRY(cudaMemcpyAsync(host, io->stage_out[j] + io->off[block], sizeof(double) * 6 * (size_t)c->hb[block].npad,
                           cudaMemcpyDeviceToHost, io->out));
  io->got[j] = true;
  return 0;
}

int orion_io_wait(orion_case_t c) {
  if (!c) return fail(ORION_E_INVALID, "null case");
  if (c->io) {
    CUDA_TRY(cudaStreamSynchronize(c->io->in));
    CUDA_TRY(cudaStreamSynchronize(c->io->out));
  }
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  return sweep_status(c);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Groups: several cases stepped together, one launch per stage over the blocks
// of every member.  The group's lists are the members' lists concatenated,
// with block indices (and tile slots, pack slots, partial ranges) shifted by
// the members before; every member keeps its own chunks, tiles and reduction
// order, so its results are the same as when it steps alone.
// ---------------------------------------------------------------------------
namespace {

// A member's list: its set-up copy when it has one, else read back.
template <typename T>
int download(orion_case_t c, std::vector<T>& v, const T* d, size_t n) {
  v.resize(n);
  if (!n) return 0;
  auto it = c->list_mirror.find(static_cast<const void*>(d));
  if (it != c->list_mirror.end() && it->second.size() >= n * sizeof(T)) {
    std::memcpy(v.data(), it->second.data(), n * sizeof(T));
    return 0;
  }
  CUDA_TRY(cudaMemcpy(v.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost));
  return 0;
}

template <typename S>
std::vector<BlockDev<S>>& host_blocks(orion_case_t c);
template <>
std::vector<BlockDev<double>>& host_blocks<double>(orion_case_t c) { return c->bd64; }
template <>
std::vector<BlockDev<float>>& host_blocks<float>(orion_case_t c) { return c->bd32; }

template <typename S>
int build_group(orion_group_t g, orion_case_t px) {
  auto& L = px->L;
  auto& mem = g->members;
  const int nm = (int)mem.size();
  int rc;
  // block descriptors: the members' own
  std::vector<BlockDev<S>> blocks;
  std::vector<int> boff(nm + 1, 0);
  for (int m = 0; m < nm; ++m) {
    for (const auto& b : host_blocks<S>(mem[m])) blocks.push_back(b);  // each points at its case's parameters
    boff[m + 1] = (int)blocks.size();
  }
  BlockDev<S>* d_blocks = nullptr;
  CUDA_TRY(cudaMallocAsync((void**)&d_blocks, sizeof(BlockDev<S>) * blocks.size(), px->stream));
  px->d_blocks = d_blocks;  // freed with the proxy
  CUDA_TRY(cudaMemcpyAsync(d_blocks, blocks.data(), sizeof(BlockDev<S>) * blocks.size(), cudaMemcpyHostToDevice,
                           px->stream));
  px->nblocks = (int)blocks.size();

  std::vector<GroupMember> gm(nm);
  std::vector<Chunk> pad, itr;
  std::vector<LineTile> tl[3];
  std::vector<RegionDev> regs;
  std::vector<std::vector<int>> phases;
  std::vector<int> pk_block, ap_block, ap_off{0}, ap_slot;
  std::vector<long long> pk_idx, ap_idx;
  std::vector<std::vector<Chunk>> planes[2];
  std::vector<SweepTile> stiles[2];
  int max_planes = 0;
  for (int m = 0; m < nm; ++m) {
    orion_case_t c = mem[m];
    const auto& M = c->L;
    const int bo = boff[m];
    std::vector<Chunk> v;
    // padded and interior chunks; the member's partial ranges
    if ((rc = download(c, v, M.pad_chunks, M.n_pad_chunks))) return rc;
    gm[m].pad_off = (int)pad.size();
    gm[m].pad_n = M.n_pad_chunks;
    for (auto ch : v) { ch.block += bo; pad.push_back(ch); }
    if ((rc = download(c, v, M.int_chunks, M.n_int_chunks))) return rc;
    gm[m].part_off = (int)itr.size();
    gm[m].part_n = M.n_int_chunks;
    for (auto ch : v) { ch.block += bo; itr.push_back(ch); }
    gm[m].blocks = d_blocks + bo;
    gm[m].nblocks = c->nblocks;
    gm[m].total_points = c->total_interior * 5;
    gm[m].dtmin = M.dtmin;
    gm[m].hist = M.hist;
    gm[m].counter = M.counter;
    gm[m].total = M.res_total;
    // line tiles
    for (int d = 0; d < 3; ++d) {
      std::vector<LineTile> t;
      if ((rc = download(c, t, M.tiles[d], M.n_tiles[d]))) return rc;
      for (auto x : t) { x.block += bo; tl[d].push_back(x); }
      L.lanes[d] = std::max(L.lanes[d], M.lanes[d]);
      L.lmax[d] = std::max(L.lmax[d], M.lmax[d]);
      L.line_units[d] = std::max(L.line_units[d], M.line_units[d]);
    }
    // halo copy: the member's own list, read in place
    gm[m].arena = static_cast<double*>(c->arena);
    gm[m].halo_src = M.halo_src;
    gm[m].halo_dst = M.halo_dst;
    gm[m].n_halo = M.n_halo;
    g->run.max_halo = std::max(g->run.max_halo, M.n_halo);
    // physical BC phases: the p-th region of every block of every member
    {
      std::vector<RegionDev> r;
      std::vector<int> pl;
      const int nreg = M.phase_off.empty() ? 0 : M.phase_off.back();
      if ((rc = download(c, pl, M.phase_regions, (size_t)nreg))) return rc;
      int maxr = 0;
      for (int x : pl) maxr = std::max(maxr, x + 1);
      if ((rc = download(c, r, M.regions, (size_t)maxr))) return rc;
      const int rbase = (int)regs.size();
      for (auto x : r) { x.block += bo; regs.push_back(x); }
      for (size_t p = 0; p + 1 < M.phase_off.size(); ++p) {
        if (phases.size() <= p) phases.resize(p + 1);
        for (int q = M.phase_off[p]; q < M.phase_off[p + 1]; ++q) phases[p].push_back(rbase + pl[q]);
      }
    }
    // interface averaging: own slots packed in member order
    {
      std::vector<int> pb, ab, ao, as;
      std::vector<long long> pi, ai;
      if ((rc = download(c, pb, M.pk_block, M.n_pack)) || (rc = download(c, pi, M.pk_idx, M.n_pack))) return rc;
      if ((rc = download(c, ab, M.ap_block, M.n_ap)) || (rc = download(c, ai, M.ap_idx, M.n_ap))) return rc;
      if ((rc = download(c, ao, M.ap_off, M.n_ap ? (size_t)M.n_ap + 1 : 0))) return rc;
      if ((rc = download(c, as, M.ap_slot, M.n_ap ? (size_t)ao.back() : 0))) return rc;
      const int slot_base = (int)pk_block.size(), ent_base = (int)ap_slot.size();
      for (int q = 0; q < M.n_pack; ++q) { pk_block.push_back(pb[q] + bo); pk_idx.push_back(pi[q]); }
      for (int q = 0; q < M.n_ap; ++q) {
        ap_block.push_back(ab[q] + bo);
        ap_idx.push_back(ai[q]);
        ap_off.push_back(ent_base + ao[q + 1]);
      }
      for (int x : as) {
        if (x >= M.n_pack) return fail(ORION_E_UNSUPPORTED, "a shard cannot join a group");
        ap_slot.push_back(slot_base + x);
      }
    }
    // sweeps: hyperplane t of every member, or the members' tiles after one another
    for (int dir = 0; dir < 2; ++dir) {
      const auto& off = M.sweep_off[dir];
      if (!off.empty()) {
        std::vector<Chunk> ch;
        if ((rc = download(c, ch, M.sweep_chunks[dir], (size_t)off.back()))) return rc;
        const int np = (int)off.size() - 1;
        if ((int)planes[dir].size() < np) planes[dir].resize(np);
        for (int t = 0; t < np; ++t)
          for (int q = off[t]; q < off[t + 1]; ++q) {
            Chunk x = ch[q];
            x.block += bo;
            planes[dir][t].push_back(x);
          }
      }
      std::vector<SweepTile> st;
      if ((rc = download(c, st, static_cast<const SweepTile*>(M.sweep_tiles[dir]), (size_t)M.n_sweep_tiles[dir])))
        return rc;
      const int sb = (int)stiles[dir].size();
      for (auto x : st) {
        x.block += bo;
        if (x.up_j >= 0) x.up_j += sb;
        if (x.up_k >= 0) x.up_k += sb;
        stiles[dir].push_back(x);
      }
    }
    max_planes = std::max(max_planes, M.max_planes);
  }
  // upload
  if ((rc = dev_upload(px, &L.pad_chunks, pad))) return rc;
  L.n_pad_chunks = (int)pad.size();
  if ((rc = dev_upload(px, &L.int_chunks, itr))) return rc;
  L.n_int_chunks = (int)itr.size();
  for (int d = 0; d < 3; ++d) {
    if ((rc = dev_upload(px, &L.tiles[d], tl[d]))) return rc;
    L.n_tiles[d] = (int)tl[d].size();
  }
  GroupRun& G = g->run;
  {
    std::vector<int> plist;
    L.phase_off.assign(1, 0);
    L.phase_maxpts.clear();
    for (auto& ph : phases) {
      int mx = 0;
      for (int r : ph) {
        plist.push_back(r);
        mx = std::max(mx, regs[r].npts);
      }
      L.phase_off.push_back((int)plist.size());
      L.phase_maxpts.push_back(mx);
    }
    if ((rc = dev_upload(px, &L.regions, regs)) || (rc = dev_upload(px, &L.phase_regions, plist))) return rc;
  }
  if ((rc = dev_upload(px, &L.pk_block, pk_block)) || (rc = dev_upload(px, &L.pk_idx, pk_idx))) return rc;
  L.n_pack = (int)pk_block.size();
  if ((rc = dev_alloc(px, &L.pack, (size_t)std::max(L.n_pack, 1) * 5))) return rc;
  if ((rc = dev_upload(px, &L.ap_block, ap_block)) || (rc = dev_upload(px, &L.ap_idx, ap_idx))) return rc;
  if ((rc = dev_upload(px, &L.ap_off, ap_off)) || (rc = dev_upload(px, &L.ap_slot, ap_slot))) return rc;
  L.n_ap = (int)ap_block.size();
  L.max_planes = max_planes;
  for (int dir = 0; dir < 2; ++dir) {
    std::vector<Chunk> ch;
    std::vector<int> off{0};
    for (auto& v : planes[dir]) {
      ch.insert(ch.end(), v.begin(), v.end());
      off.push_back((int)ch.size());
    }
    if ((rc = dev_upload(px, &L.sweep_chunks[dir], ch))) return rc;
    L.sweep_off[dir] = off;
    SweepTile* d = nullptr;
    if ((rc = dev_upload(px, &d, stiles[dir]))) return rc;
    L.sweep_tiles[dir] = d;
    L.n_sweep_tiles[dir] = (int)stiles[dir].size();
  }
  L.sweep_nt = kSweepThreads;
  {
    const int mx = std::max(L.n_sweep_tiles[0], L.n_sweep_tiles[1]);
    unsigned char* ctl = nullptr;
    if ((rc = dev_alloc(px, &ctl, offsetof(TileCtl, progress) + sizeof(unsigned int) * (size_t)std::max(mx, 1))))
      return rc;
    L.tile_ctl = ctl;
    L.tile_k = mem[0]->L.tile_k;
    int* sctl = nullptr;
    if ((rc = dev_alloc(px, &sctl, 4))) return rc;
    L.sweep_ctl = sctl;
  }
  if ((rc = dev_alloc(px, &L.partials, (size_t)std::max(L.n_int_chunks, 1)))) return rc;
  if ((rc = dev_alloc(px, &L.dt_part, (size_t)std::max(L.n_pad_chunks, 1)))) return rc;
  if ((rc = dev_upload(px, &G.members, gm))) return rc;
  G.nmembers = nm;
  g->block_off.assign(boff.begin(), boff.end() - 1);
  L.group = &G;
  return 0;
}

}  // namespace

extern "C" {

int orion_group_create(int n, const orion_case_t* cases, orion_group_t* out) {
  if (n < 1 || !cases || !out) return fail(ORION_E_INVALID, "bad arguments");
  *out = nullptr;
  for (int m = 0; m < n; ++m) {
    const orion_case_t c = cases[m];
    if (!c) return fail(ORION_E_INVALID, "null case");
    if (c->prec != cases[0]->prec) return fail(ORION_E_UNSUPPORTED, "the cases of a group share one precision");
    if (c->P.nvis != cases[0]->P.nvis) return fail(ORION_E_UNSUPPORTED, "the cases of a group are all viscous or all Euler");
    if (c->shard.nranks > 1) return fail(ORION_E_UNSUPPORTED, "a shard cannot join a group");
    if (c->pending_n > 0) return fail(ORION_E_INVALID, "a case has submitted steps that have not been polled");
    if (c->group) return fail(ORION_E_INVALID, "a case belongs to another group");
    for (int q = 0; q < m; ++q)
      if (cases[q] == c) return fail(ORION_E_INVALID, "a case is listed twice");
  }
  std::lock_guard<std::mutex> lk(g_struct_mu);
  auto g = std::make_unique<orion_group_s>();
  g->members.assign(cases, cases + n);
  auto px = std::make_unique<orion_case_s>();
  px->prec = cases[0]->prec;
  px->P = cases[0]->P;  // not read: every block carries its case's parameters
  px->device = cases[0]->device;
  CUDA_TRY(cudaSetDevice(px->device));
  CUDA_TRY(cudaStreamCreateWithFlags(&px->stream, cudaStreamNonBlocking));
  px->own_stream = true;
  bool tiles = true;
  for (auto c : g->members) {
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    tiles = tiles && c->L.tiles_on;
  }
  px->L.tiles_on = tiles;  // otherwise one launch per hyperplane
  g->proxy = px.get();
  int rc = px->prec == ORION_PREC_FP64 ? build_group<double>(g.get(), px.get()) : build_group<float>(g.get(), px.get());
  if (!rc) rc = ops_for(px->prec).set_attributes();
  if (!rc) {
    cudaError_t e = cudaStreamSynchronize(px->stream);
    if (e != cudaSuccess) rc = fail(ORION_E_CUDA, std::string("group set-up: ") + cudaGetErrorString(e));
  }
  if (rc) {
    destroy_case(px.release());
    return rc;
  }
  for (auto c : g->members) {
    g->saved_streams.push_back(c->stream);
    c->stream = px->stream;  // the members' copies, polls and per-stage calls follow the group's launches
    c->group = g.get();
  }
  px.release();
  *out = g.release();
  return 0;
}

int orion_group_destroy(orion_group_t g) {
  if (!g) return 0;
  std::lock_guard<std::mutex> lk(g_struct_mu);
  cudaStreamSynchronize(g->proxy->stream);
  for (size_t m = 0; m < g->members.size(); ++m) {
    g->members[m]->stream = g->saved_streams[m];
    g->members[m]->group = nullptr;
  }
  destroy_case(g->proxy);
  delete g;
  return 0;
}

int orion_group_submit(orion_group_t g, int nsteps) {
  if (!g || nsteps < 0) return fail(ORION_E_INVALID, "bad arguments");
  for (auto c : g->members) {
    if (c->pending_n + nsteps > kHistCap)
      return fail(ORION_E_INVALID, "more unpolled steps than the history ring holds (4096)");
    if (!c->hist_host && !(c->hist_host = acquire_hist_ring())) return fail(ORION_E_NOMEM, "pinned history ring");
    if (c->hist_count < 0) {
      int cnt = 0;
      CUDA_TRY(cudaStreamSynchronize(c->stream));
      CUDA_TRY(cudaMemcpy(&cnt, c->L.counter, sizeof(int), cudaMemcpyDeviceToHost));
      c->hist_count = cnt;
    }
  }
  if (nsteps == 0) return 0;
  int rc = launch_steps(g->proxy, nsteps);
  if (rc) return rc;
  for (auto c : g->members) {
    c->steps_done += nsteps;
    if ((rc = enqueue_hist_copy(c, nsteps))) return rc;
  }
  return 0;
}

int orion_group_sync(orion_group_t g) {
  if (!g) return fail(ORION_E_INVALID, "null group");
  CUDA_TRY(cudaStreamSynchronize(g->proxy->stream));
  return sweep_status(g->proxy);
}

int orion_group_step_launches(orion_group_t g, int* n) {
  if (!g || !n) return fail(ORION_E_INVALID, "null argument");
  int rc = ensure_graph(g->proxy);
  if (rc) return rc;
  *n = g->proxy->step_launches;
  return 0;
}

// ---------------------------------------------------------------------------
// Block sharding (exchange_plan.hpp): one case per shard, exchanges by buffer.
// ---------------------------------------------------------------------------
int orion_shard_blocks(orion_case_t c, int* nlocal, int* global_ids) {
  if (!c || !nlocal) return fail(ORION_E_INVALID, "null argument");
  *nlocal = c->nblocks;
  if (global_ids) std::copy(c->shard.global_ids.begin(), c->shard.global_ids.end(), global_ids);
  return 0;
}

static int shard_peer(orion_case_t c, int kind, int peer) {
  if (!c) return fail(ORION_E_INVALID, "null case");
  if (kind != ORION_XCHG_HALO && kind != ORION_XCHG_IFACE) return fail(ORION_E_INVALID, "bad exchange kind");
  if (peer < 0 || peer >= c->shard.nranks || peer == c->shard.rank) return fail(ORION_E_INVALID, "bad peer shard");
  return 0;
}

int orion_shard_counts(orion_case_t c, int kind, int peer, long long* nsend, long long* nrecv) {
  if (!nsend || !nrecv) return fail(ORION_E_INVALID, "null argument");
  int rc = shard_peer(c, kind, peer);
  if (rc) return rc;
  const auto& X = c->shard;
  if (kind == ORION_XCHG_HALO) {
    *nsend = X.n_halo_send[peer];
    *nrecv = X.n_halo_recv[peer];
  } else {
    *nsend = 5 * X.n_iface_send[peer];
    *nrecv = 5 * (long long)X.iface_recv_n[peer];
  }
  return 0;
}

int orion_shard_pack(orion_case_t c, int kind, int peer, double* buf) {
  int rc = shard_peer(c, kind, peer);
  if (rc) return rc;
  const auto& X = c->shard;
  const long long n = kind == ORION_XCHG_HALO ? X.n_halo_send[peer] : X.n_iface_send[peer];
  if (n == 0) return 0;
  if (!buf) return fail(ORION_E_INVALID, "null buffer");
  const long long work = kind == ORION_XCHG_HALO ? n : 5 * n;
  const int grid = (int)((work + kThreads - 1) / kThreads);
  if (kind == ORION_XCHG_HALO)
    k_shard_gather<<<grid, kThreads, 0, c->stream>>>(static_cast<const double*>(c->arena), X.halo_send[peer], buf, n);
  else
    k_shard_gather_slots<<<grid, kThreads, 0, c->stream>>>(c->L.pack, X.iface_send[peer], buf, n);
  CUDA_TRY(cudaGetLastError());
  return 0;
}

int orion_shard_unpack(orion_case_t c, int kind, int peer, const double* buf) {
  int rc = shard_peer(c, kind, peer);
  if (rc) return rc;
  const auto& X = c->shard;
  if (kind == ORION_XCHG_HALO) {
    const long long n = X.n_halo_recv[peer];
    if (n == 0) return 0;
    if (!buf) return fail(ORION_E_INVALID, "null buffer");
    k_shard_scatter<<<(int)((n + kThreads - 1) / kThreads), kThreads, 0, c->stream>>>(
        static_cast<double*>(c->arena), X.halo_recv[peer], buf, n);
    CUDA_TRY(cudaGetLastError());
  } else {
    const long long n = X.iface_recv_n[peer];
    if (n == 0) return 0;
    if (!buf) return fail(ORION_E_INVALID, "null buffer");
    CUDA_TRY(cudaMemcpyAsync(c->L.pack + (long long)X.iface_recv_base[peer] * 5, buf, sizeof(double) * 5 * n,
                             cudaMemcpyDeviceToDevice, c->stream));
  }
  return 0;
}

int orion_shard_average_begin(orion_case_t c) {
  return dispatch(c, [&](const StageOps& o) { return o.average_begin(c); });
}
int orion_shard_average_end(orion_case_t c) {
  return dispatch(c, [&](const StageOps& o) { return o.average_end(c); });
}

int orion_shard_residual(orion_case_t c, orion_shard_residual_t* out) {
  if (!c || !out) return fail(ORION_E_INVALID, "null argument");
  int rc = dispatch(c, [&](const StageOps& o) { return o.residual(c); });
  if (rc) return rc;
  CUDA_TRY(cudaStreamSynchronize(c->stream));
  ResPartial t{};
  unsigned long long bits = 0;
  CUDA_TRY(cudaMemcpy(&t, c->L.res_total, sizeof(t), cudaMemcpyDeviceToHost));
  CUDA_TRY(cudaMemcpy(&bits, c->L.dtmin, sizeof(bits), cudaMemcpyDeviceToHost));
  out->sum = t.sum;
  out->max = t.max;
  out->key = t.key;
  std::memcpy(&out->dtmin, &bits, sizeof(double));
  out->points = c->shard.total_interior_global;
  return 0;
}

int orion_shard_plan_counts(int nblocks, const orion_block_desc_t* blocks, const int* owner, int rank, int kind,
                            long long* nsend, long long* nrecv) {
  if (!owner || !nsend || !nrecv) return fail(ORION_E_INVALID, "null argument");
  if (kind != ORION_XCHG_HALO && kind != ORION_XCHG_IFACE) return fail(ORION_E_INVALID, "bad exchange kind");
  int rc = validate_blocks(nblocks, blocks);
  if (rc) return rc;
  std::vector<HostBlock> gb;
  if ((rc = host_blocks(nblocks, blocks, gb))) return rc;
  ExchangePlan plan;
  const std::string err = build_exchange_plan(gb, std::vector<int>(owner, owner + nblocks), rank, plan, NG);
  if (!err.empty()) return fail(ORION_E_INVALID, err);
  for (int r = 0; r < plan.nranks; ++r) {
    if (kind == ORION_XCHG_HALO) {
      nsend[r] = (long long)plan.halo_send[r].size();
      nrecv[r] = (long long)plan.halo_recv[r].size();
    } else {
      nsend[r] = 5 * (long long)plan.iface_send[r].size();
      nrecv[r] = 5 * (long long)plan.iface_recv_n[r];
    }
  }
  return 0;
}

}  // extern "C"
