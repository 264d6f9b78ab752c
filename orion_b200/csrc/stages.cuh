#include <mutex>
// Stage launchers, templated on storage S and compute T.  Included by exactly
// one translation unit per precision.
#pragma once
#include <cstdlib>

#include "case.hpp"
#include "kernels.cuh"
#include "sweep_tiles.cuh"

namespace orion {

// --------------------------------------------------------------------------
// stage launchers (templated on storage S and compute T)
// --------------------------------------------------------------------------
template <typename S, typename T>
struct Stages {
  static const BlockDev<S>* blocks(orion_case_t c) { return static_cast<const BlockDev<S>*>(c->d_blocks); }

  // Line kernels take up to kLineSmemBudget of dynamic shared memory; the
  // attribute is set once per process, before any stream capture.
  static int set_attributes() {
    static std::once_flag once;
    static int rc = 0;
    std::call_once(once, [] { rc = set_line_attributes(); });
    return rc;
  }

  // dynamic shared memory the tile sweeps may ask for (prefetch buffers and
  // the row-base cache of blocks of up to about 2,500 hyperplanes)
  static constexpr size_t kTileSmemMax = 160 * 1024;

  static int set_line_attributes() {
    const int b = (int)kLineSmemBudget;
    const int tb = (int)kTileSmemMax;
    CUDA_TRY(cudaFuncSetAttribute(k_sweep_tiles<S, T, SW_LUSGS_FWD, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, tb));
    CUDA_TRY(cudaFuncSetAttribute(k_sweep_tiles<S, T, SW_LUSGS_BWD, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, tb));
    CUDA_TRY(cudaFuncSetAttribute(k_sweep_tiles<S, T, SW_GS, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, tb));
    CUDA_TRY(cudaFuncSetAttribute(k_sweep_tiles<S, T, SW_GS, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, tb));
    CUDA_TRY(cudaFuncSetAttribute(k_viscous<0, S, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    CUDA_TRY(cudaFuncSetAttribute(k_viscous<1, S, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    CUDA_TRY(cudaFuncSetAttribute(k_viscous<2, S, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    CUDA_TRY(cudaFuncSetAttribute(k_inviscid<0, S, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    CUDA_TRY(cudaFuncSetAttribute(k_inviscid<1, S, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    CUDA_TRY(cudaFuncSetAttribute(k_inviscid<2, S, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, b));
    return 0;
  }

  static int exchange(orion_case_t c) {
    auto& L = c->L;
    if (L.group) {
      const GroupRun& GR = *L.group;
      if (GR.max_halo > 0) {
        // grid-stride per member: four CTAs per SM of a B200 (148 SMs) cover the longest list
        const int gx = std::min((GR.max_halo + kThreads - 1) / kThreads, 4 * 148);
        k_halo_copy_group<<<dim3(gx, GR.nmembers), kThreads, 0, c->stream>>>(GR.members);
      }
      return 0;
    }
    if (L.n_halo > 0)
      k_halo_copy<<<(L.n_halo + kThreads - 1) / kThreads, kThreads, 0, c->stream>>>(
          static_cast<double*>(c->arena), L.halo_src, L.halo_dst, L.n_halo);
    return 0;
  }

  static int bc(orion_case_t c) {
    auto& L = c->L;
    for (size_t p = 0; p + 1 < L.phase_off.size(); ++p) {
      const int nr = L.phase_off[p + 1] - L.phase_off[p];
      if (nr <= 0 || L.phase_maxpts[p] <= 0) continue;
      dim3 grid((L.phase_maxpts[p] + kThreads - 1) / kThreads, nr);
      k_bc_phase<S><<<grid, kThreads, 0, c->stream>>>(blocks(c), L.regions, L.phase_regions + L.phase_off[p]);
    }
    return 0;
  }

  static int state(orion_case_t c, bool with_dt, bool with_q) {
    auto& L = c->L;
    if (with_dt && with_q)
      k_state<S, true, true><<<L.n_pad_chunks, kThreads, 0, c->stream>>>(blocks(c), L.pad_chunks, L.dt_part);
    else if (with_dt)
      k_state<S, false, true><<<L.n_pad_chunks, kThreads, 0, c->stream>>>(blocks(c), L.pad_chunks, L.dt_part);
    else if (with_q)
      k_state<S, true, false><<<L.n_pad_chunks, kThreads, 0, c->stream>>>(blocks(c), L.pad_chunks, L.dt_part);
    else
      k_state<S, false, false><<<L.n_pad_chunks, kThreads, 0, c->stream>>>(blocks(c), L.pad_chunks, L.dt_part);
    if (with_dt) {
      if (L.group)
        k_dtmin_group<<<L.group->nmembers, 1024, 0, c->stream>>>(L.group->members, L.dt_part);
      else
        k_dtmin_final<<<1, 1024, 0, c->stream>>>(L.dt_part, L.n_pad_chunks, L.dtmin);
    }
    return 0;
  }

  static int timestep(orion_case_t c) {
    auto& L = c->L;
    k_timestep<S><<<L.n_int_chunks, kThreads, 0, c->stream>>>(blocks(c), L.int_chunks, L.dt_part);
    k_dtmin_final<<<1, 1024, 0, c->stream>>>(L.dt_part, L.n_int_chunks, L.dtmin);
    return 0;
  }

  template <int D>
  static void visc_dir(orion_case_t c) {
    auto& L = c->L;
    const size_t smem = (size_t)L.line_units[D] * 4 * sizeof(T);
    k_viscous<D, S, T><<<L.n_tiles[D], kThreads, smem, c->stream>>>(blocks(c), L.tiles[D]);
  }

  static int viscous(orion_case_t c) {
    if (c->P.nvis != 1) return 0;
    auto& L = c->L;
    k_node_derivs<S, T><<<L.n_int_chunks, kThreads, 0, c->stream>>>(blocks(c), L.int_chunks);
    visc_dir<0>(c);
    visc_dir<1>(c);
    visc_dir<2>(c);
    return 0;
  }

  template <int D>
  static void inv_dir(orion_case_t c) {
    auto& L = c->L;
    const size_t smem = (size_t)L.line_units[D] * 5 * sizeof(T);
    k_inviscid<D, S, T><<<L.n_tiles[D], kThreads, smem, c->stream>>>(blocks(c), L.tiles[D]);
    {
      // six outputs per line of the tile, whole warps: a CTA of 256 threads
      // would leave most of its registers idle (about 128 per thread)
      const int nt = std::min(kThreads, (6 * std::max(L.lanes[D], 1) + 31) / 32 * 32);
      k_inv_cascade<D, S, T><<<L.n_tiles[D], nt, 0, c->stream>>>(blocks(c), L.tiles[D]);
    }
  }

  static int inviscid(orion_case_t c) {
    inv_dir<0>(c);
    inv_dir<1>(c);
    inv_dir<2>(c);
    return 0;
  }

  static int average_begin(orion_case_t c) {
    auto& L = c->L;
    if (L.n_pack == 0) return 0;
    k_iface_pack<S><<<(L.n_pack + kThreads - 1) / kThreads, kThreads, 0, c->stream>>>(blocks(c), L.pk_block, L.pk_idx,
                                                                                       L.pack, L.n_pack);
    return 0;
  }

  static int average_end(orion_case_t c) {
    auto& L = c->L;
    if (L.n_ap == 0) return 0;
    k_iface_apply<S><<<(L.n_ap + kThreads - 1) / kThreads, kThreads, 0, c->stream>>>(
        blocks(c), L.ap_block, L.ap_idx, L.ap_off, L.ap_slot, L.pack, L.n_ap);
    return 0;
  }

  static int average(orion_case_t c) {
    average_begin(c);
    return average_end(c);
  }

  // One launch per hyperplane, each a programmatic dependent of the one before
  // (griddepcontrol in k_sweep_plane), so launch latency and the static loads
  // of a hyperplane overlap the previous one.
  template <int MODE, int NT>
  static int sweep_nt(orion_case_t c, int dir) {
    auto& L = c->L;
    const auto& off = L.sweep_off[dir];
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    for (int t = 0; t + 1 < (int)off.size(); ++t) {
      const int n = off[t + 1] - off[t];
      if (n <= 0) continue;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(n);
      cfg.blockDim = dim3(NT);
      cfg.stream = c->stream;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      CUDA_TRY(cudaLaunchKernelEx(&cfg, k_sweep_plane<S, T, MODE, NT>, blocks(c),
                                  (const Chunk*)(L.sweep_chunks[dir] + off[t])));
    }
    return 0;
  }

  template <int MODE>
  static int sweep(orion_case_t c, int dir) {
    return sweep_nt<MODE, kSweepThreads>(c, dir);
  }

  // Sweep scheduling.  Preferred: cluster sweeps (16- or 8-CTA clusters, as
  // many as are co-resident, mesh blocks grouped per cluster).  Otherwise the
  // persistent cooperative kernel, otherwise one launch per hyperplane.
  // ORION_SWEEP=planes|grid|cluster selects one explicitly.
  static size_t cluster_smem(orion_case_t c) {
    return sizeof(SweepBlock<S>) * c->nblocks + sizeof(SweepSlot) * 2 * (size_t)c->L.max_planes;
  }

  // The cluster kernel's function attributes are process-wide: they are set
  // once, to the largest shared memory any case may ask for, and never per
  // case (a case made on one host thread must not change an attribute that a
  // graph of another case, captured on another thread, was built against).
  static constexpr size_t kClusterSmemMax = 200 * 1024;

  template <int NT>
  static bool cluster_attributes() {
    static std::once_flag once;
    static bool ok = false;
    std::call_once(once, [] {
      auto kern = k_sweeps_cluster<S, T, NT>;
      ok = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kClusterSmemMax) ==
               cudaSuccess &&
           cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess;
      if (!ok) cudaGetLastError();
    });
    return ok;
  }

  // only_cs: 0 = largest co-resident cluster size (16, else 8), else just that size
  template <int NT>
  static int cluster_setup(orion_case_t c, int only_cs = 0) {
    auto kern = k_sweeps_cluster<S, T, NT>;
    const size_t smem = cluster_smem(c);
    if (smem > kClusterSmemMax || !cluster_attributes<NT>()) return 0;
    for (int cs : {16, 8}) {
      if (only_cs && cs != only_cs) continue;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(cs * 64);
      cfg.blockDim = dim3(NT);
      cfg.dynamicSmemBytes = smem;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = cs;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int ncl = 0;
      if (cudaOccupancyMaxActiveClusters(&ncl, kern, &cfg) != cudaSuccess || ncl < 1) {
        cudaGetLastError();
        continue;
      }
      int rc = build_cluster_lists(c, ncl);
      if (rc) return rc;
      c->L.cl_size = cs;
      return 0;
    }
    return 0;
  }

  // The cooperative grid form: one CTA pair per SM, all co-resident.
  static int grid_setup(orion_case_t c) {
    int dev = 0, coop = 0, nsm = 0, per_sm = 0;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweeps_persistent<S, T, kSweepThreads>,
                                                           kSweepThreads, 0));
    const int want = 2;  // two CTAs per SM
    if (!coop || per_sm < want) return 0;
    c->L.persist_grid = nsm * want;
    return 0;
  }

  // An explicit sweep form (ORION_SWEEP_TILES / _PLANES / _GRID / _CLUSTER with size cs).
  static int schedule(orion_case_t c, int form, int cs) {
    c->L.persist_grid = 0;
    c->L.cl_size = 0;
    c->L.tiles_on = form == ORION_SWEEP_TILES;
    if (form == ORION_SWEEP_PLANES || form == ORION_SWEEP_TILES) return 0;
    if (form == ORION_SWEEP_GRID) {
      int rc = grid_setup(c);
      if (rc) return rc;
      return c->L.persist_grid > 0 ? 0 : fail(ORION_E_UNSUPPORTED, "cooperative sweep grid not co-resident");
    }
    if (form == ORION_SWEEP_CLUSTER) {
      if (cs != 0 && cs != 8 && cs != 16) return fail(ORION_E_INVALID, "cluster size must be 8 or 16");
      int rc = cluster_setup<kSweepThreads>(c, cs);
      if (rc) return rc;
      return c->L.cl_size > 0 ? 0 : fail(ORION_E_UNSUPPORTED, "sweep clusters of that size are not co-resident");
    }
    return fail(ORION_E_INVALID, "unknown sweep form");
  }

  static int persistent_grid(orion_case_t c) {
    c->L.persist_grid = 0;
    c->L.cl_size = 0;
    c->L.tiles_on = false;
    // default: one programmatic-dependent launch per hyperplane (the fastest
    // form the autotuner measured on the configurations, both precisions)
    const char* env = getenv("ORION_SWEEP");
    const std::string mode = env ? std::string(env) : std::string("planes");
    const char* lim = getenv("ORION_SWEEP_SPIN_LIMIT");  // bound of the sweeps' device waits
    if (lim) c->L.spin_limit = atoll(lim);
    if (mode == "tiles") {
      c->L.tiles_on = true;
      return 0;
    }
    if (mode == "planes") return 0;
    if (mode == "cluster") {
      int rc = cluster_setup<kSweepThreads>(c);
      if (rc) return rc;
      if (c->L.cl_size > 0) return 0;
    }
    return grid_setup(c);
  }

  template <int NT>
  static int sweeps_cluster_nt(orion_case_t c) {
    auto& L = c->L;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(L.cl_count * L.cl_size);
    cfg.blockDim = dim3(NT);
    cfg.dynamicSmemBytes = cluster_smem(c);
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = L.cl_size;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CUDA_TRY(cudaLaunchKernelEx(&cfg, k_sweeps_cluster<S, T, NT>, blocks(c), c->nblocks, (const Chunk*)L.cl_chunks[0],
                                (const int*)L.cl_off[0], (const Chunk*)L.cl_chunks[1], (const int*)L.cl_off[1],
                                (const int*)L.cl_base, (const int*)L.cl_nplanes, c->P));
    return 0;
  }

  static int sweeps_persistent(orion_case_t c) {
    auto& L = c->L;
    SweepCtl* ctl = static_cast<SweepCtl*>(L.sweep_ctl);
    CUDA_TRY(cudaMemsetAsync(&ctl->counter, 0, sizeof(unsigned int), c->stream));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(L.persist_grid);
    cfg.blockDim = dim3(L.sweep_nt);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = c->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const long long spin_limit = L.spin_limit;
    CUDA_TRY(cudaLaunchKernelEx(&cfg, k_sweeps_persistent<S, T, kSweepThreads>, blocks(c),
                                (const Chunk*)L.sweep_chunks[0], (const int*)L.sweep_off_dev[0],
                                (const Chunk*)L.sweep_chunks[1], (const int*)L.sweep_off_dev[1], L.max_planes, c->P,
                                ctl, spin_limit));
    return 0;
  }

  // One pass of the tile wavefront: reset the tickets and progress words, then
  // one CTA per tile.
  template <int MODE, int DIR>
  static int tile_pass(orion_case_t c) {
    auto& L = c->L;
    const int d = DIR > 0 ? 0 : 1;
    const int n = L.n_sweep_tiles[d];
    if (n <= 0) return 0;
    CUDA_TRY(cudaMemsetAsync(L.tile_ctl, 0, offsetof(TileCtl, progress) + sizeof(unsigned int) * (size_t)n,
                             c->stream));
    SweepCtl* sc = static_cast<SweepCtl*>(L.sweep_ctl);
    const size_t smem = tile_smem_bytes<T, MODE>(L.max_planes);
    if (smem > kTileSmemMax) return fail(ORION_E_UNSUPPORTED, "block too long for the tile sweeps' row-base cache");
    k_sweep_tiles<S, T, MODE, DIR><<<n, 32 * TileShape<T>::TK + 32, smem, c->stream>>>(
        blocks(c), static_cast<const SweepTile*>(L.sweep_tiles[d]), n, static_cast<TileCtl*>(L.tile_ctl),
        &sc->error, L.spin_limit);
    return 0;
  }

  static int update(orion_case_t c, bool fuse_residual) {
    auto& L = c->L;
    if (L.tiles_on) {
      k_lusgs_prep<S, T, false><<<L.n_int_chunks, kThreads, 0, c->stream>>>(blocks(c), L.int_chunks);
    } else {
      k_lusgs_prep<S, T, true><<<L.n_int_chunks, kThreads, 0, c->stream>>>(blocks(c), L.int_chunks);
      k_sweep_pairs<S, T><<<L.n_int_chunks, kThreads, 0, c->stream>>>(blocks(c), L.int_chunks);
    }
    if (L.tiles_on) {
      int rc = tile_pass<SW_LUSGS_FWD, 1>(c);
      if (!rc) rc = tile_pass<SW_LUSGS_BWD, -1>(c);
      if (!rc) rc = tile_pass<SW_GS, 1>(c);
      if (!rc) rc = tile_pass<SW_GS, -1>(c);
      if (rc) return rc;
    } else if (L.cl_size > 0) {
      int rc = sweeps_cluster_nt<kSweepThreads>(c);
      if (rc) return rc;
    } else if (L.persist_grid > 0) {
      int rc = sweeps_persistent(c);
      if (rc) return rc;
    } else {
      int rc = sweep<SW_LUSGS_FWD>(c, 0);
      if (!rc) rc = sweep<SW_LUSGS_BWD>(c, 1);
      if (!rc) rc = sweep<SW_GS>(c, 0);
      if (!rc) rc = sweep<SW_GS>(c, 1);
      if (rc) return rc;
    }
    if (fuse_residual) {
      k_sweep_finish<S, true, kThreads><<<L.n_int_chunks, kThreads, 0, c->stream>>>(blocks(c), L.int_chunks,
                                                                                     L.partials);
      residual_final(c);
    } else {
      k_sweep_finish<S, false, kThreads><<<L.n_int_chunks, kThreads, 0, c->stream>>>(blocks(c), L.int_chunks,
                                                                                      L.partials);
    }
    return 0;
  }

  static int skew_static(orion_case_t c, int b) {
    k_skew_static<S><<<148 * 4, kThreads, 0, c->stream>>>(blocks(c), b);
    if constexpr (sizeof(S) == 4)
      k_metric_shadow<<<148 * 4, kThreads, 0, c->stream>>>(reinterpret_cast<const BlockDev<float>*>(blocks(c)), b);
    return 0;
  }

  static int prim_shadow(orion_case_t c, int b) {
    if constexpr (sizeof(S) == 4)
      k_prim_shadow<<<148 * 4, kThreads, 0, c->stream>>>(reinterpret_cast<const BlockDev<float>*>(blocks(c)), b);
    return 0;
  }

  static void residual_final(orion_case_t c) {
    auto& L = c->L;
    if (L.group) {
      k_res_final_group<S><<<L.group->nmembers, 1024, 0, c->stream>>>(L.group->members, L.partials, kHistCap);
      return;
    }
    k_res_final<S><<<1, 1024, 0, c->stream>>>(blocks(c), c->nblocks, L.partials, L.n_int_chunks, c->total_interior * 5,
                                              L.dtmin, L.hist, L.counter, kHistCap, L.res_total);
  }

  static int residual(orion_case_t c) {
    auto& L = c->L;
    k_update_res<S, false, true, kThreads><<<L.n_int_chunks, kThreads, 0, c->stream>>>(blocks(c), L.int_chunks,
                                                                                        L.partials);
    residual_final(c);
    return 0;
  }

  // One whole step in the order of OrionSolver::solve (OrionSolver.cpp:141-209).
  static int step(orion_case_t c, bool with_q) {
    exchange(c);
    bc(c);
    state(c, true, with_q);
    viscous(c);
    if (c->P.nvis == 1) average(c);
    inviscid(c);
    average(c);
    update(c, true);
    return 0;
  }

  static int init_flow(orion_case_t c, uint64_t seed, double amp) {
    auto& L = c->L;
    k_init_flow<S><<<L.n_pad_chunks, kThreads, 0, c->stream>>>(blocks(c), L.pad_chunks, L.pad_base, seed, amp);
    return 0;
  }
};

template <typename S, typename T>
StageOps make_ops() {
  using X = Stages<S, T>;
  StageOps o;
  o.set_attributes = &X::set_attributes;
  o.exchange = &X::exchange;
  o.bc = &X::bc;
  o.state = &X::state;
  o.timestep = &X::timestep;
  o.viscous = &X::viscous;
  o.average = &X::average;
  o.average_begin = &X::average_begin;
  o.average_end = &X::average_end;
  o.inviscid = &X::inviscid;
  o.update = &X::update;
  o.residual = &X::residual;
  o.step = &X::step;
  o.init_flow = &X::init_flow;
  o.skew_static = &X::skew_static;
  o.persistent_grid = &X::persistent_grid;
  o.schedule = &X::schedule;
  o.prim_shadow = &X::prim_shadow;
  return o;
}

}  // namespace orion
