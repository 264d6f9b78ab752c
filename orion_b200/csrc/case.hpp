// Host-side case object and shared runtime helpers of the C ABI.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <unordered_map>
#include <vector>

#include "device_types.cuh"
#include "orion_gpu.h"
#include "exchange_plan.hpp"
#include "topology.hpp"

namespace orion {

extern thread_local std::string g_last_error;

inline int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
int set_error(int code, const std::string& msg);

#define CUDA_TRY(expr)                                                                       \
  do {                                                                                       \
    cudaError_t _e = (expr);                                                                 \
    if (_e != cudaSuccess)                                                                   \
      return ::orion::fail(ORION_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
  } while (0)

constexpr int kThreads = 256;
constexpr int kChunk = 256;         // points per CTA (one per thread) for pointwise kernels
constexpr int kHistCap = 4096;      // residual history ring
// Points per sweep chunk (one per thread, one CTA per chunk).  128 measured
// fastest on the 64-block 385x257x129 case for both precisions (256: +1.1%,
// 64: +0.7% mixed): an average hyperplane there is below one wave of
// 256-thread CTAs, and smaller CTAs spread it over more SMs and leave room
// for the next hyperplane's CTAs to be resident early.
#ifndef ORION_SWEEP_THREADS
#define ORION_SWEEP_THREADS 128
#endif
constexpr int kSweepThreads = ORION_SWEEP_THREADS;
constexpr size_t kLineSmemBudget = 96 * 1024;

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// What a group of cases stepped together needs beyond the lists (orion_group_*).
struct GroupRun {
  GroupMember* members = nullptr;  // device array, one per case
  int nmembers = 0;
  int max_halo = 0;                // the longest member halo copy list
};

struct DeviceLists {
  const GroupRun* group = nullptr;  // set on a group's lists: the stages reduce per case
  Chunk* pad_chunks = nullptr;
  int n_pad_chunks = 0;
  Chunk* int_chunks = nullptr;
  int n_int_chunks = 0;
  LineTile* tiles[3] = {nullptr, nullptr, nullptr};
  int n_tiles[3] = {0, 0, 0};
  int lanes[3] = {1, 1, 1};
  int lanes_cap = 32;                            // line tiles: at most this many grid lines per CTA (set at creation)
  int lmax[3] = {0, 0, 0};
  int line_units[3] = {0, 0, 0};                 // line tiles' face slots (lanes x (longest line + 1)) of shared memory
  Chunk* sweep_chunks[2] = {nullptr, nullptr};  // forward / backward hyperplane launches
  std::vector<int> sweep_off[2];                 // host: chunk range of each launch
  int* sweep_off_dev[2] = {nullptr, nullptr};    // device copies of sweep_off
  void* sweep_ctl = nullptr;                     // SweepCtl of the persistent sweep kernel
  int persist_grid = 0;                          // CTAs of the persistent sweep kernel (0: per-plane launches)
  int sweep_nt = 256;                            // threads per sweep CTA = hyperplane chunk size
  // cluster sweeps: mesh blocks grouped per thread-block cluster
  int cl_size = 0;                               // CTAs per cluster (0: not used)
  int cl_count = 0;                              // clusters (= groups)
  Chunk* cl_chunks[2] = {nullptr, nullptr};      // forward / backward chunk lists of all groups
  int* cl_off[2] = {nullptr, nullptr};           // per-group hyperplane offsets, concatenated
  int* cl_base = nullptr;                        // start of each group's offsets
  int* cl_nplanes = nullptr;                     // hyperplanes of each group
  long long spin_limit = 1LL << 21;              // polls before a grid barrier gives up (about a second)
  // tile wavefront sweeps (sweep_tiles.cuh): per direction the tile list in
  // ticket order, and one control block (ticket + progress per tile) reset
  // before every pass
  bool tiles_on = false;
  void* sweep_tiles[2] = {nullptr, nullptr};     // SweepTile lists, forward / backward
  int n_sweep_tiles[2] = {0, 0};
  void* tile_ctl = nullptr;                      // TileCtl with max(n_sweep_tiles) progress words
  size_t tile_ctl_bytes = 0;
  int tile_k = 4;                                // k rows per tile (32 j rows)
  int max_planes = 0;
  long long* halo_src = nullptr;
  long long* halo_dst = nullptr;
  int n_halo = 0;
  RegionDev* regions = nullptr;
  int* phase_regions = nullptr;
  std::vector<int> phase_off;  // host: region list offsets per phase
  std::vector<int> phase_maxpts;
  int* pk_block = nullptr;
  long long* pk_idx = nullptr;
  double* pack = nullptr;
  int n_pack = 0;
  int* ap_block = nullptr;
  long long* ap_idx = nullptr;
  int* ap_off = nullptr;
  int* ap_slot = nullptr;
  int n_ap = 0;
  ResPartial* partials = nullptr;
  ResidualOut* hist = nullptr;
  int* counter = nullptr;
  unsigned long long* dtmin = nullptr;
  double* dt_part = nullptr;  // per-CTA minima of dt_phys
  long long* pad_base = nullptr;
  ResPartial* res_total = nullptr;  // the last residual's raw sum, max and key (shards reduce these)
};

// Block sharding: a case holding the blocks of one shard, and the device lists
// of its exchanges with every other shard (exchange_plan.hpp).
struct ShardLists {
  int rank = 0;
  int nranks = 1;
  std::vector<int> global_ids;          // global block id of each local block
  std::vector<long long> pad_base;      // global padded offset of each local block (initial noise)
  long long total_interior_global = 0;  // interior points of every shard
  std::vector<long long*> halo_send, halo_recv;  // per peer: arena offsets (FP64 elements)
  std::vector<long long> n_halo_send, n_halo_recv;
  std::vector<int*> iface_send;         // per peer: own slots
  std::vector<long long> n_iface_send;
  std::vector<int> iface_recv_base, iface_recv_n;
};

}  // namespace orion

// Pipelined host I/O (orion_io_*): staging copies of every block's prim and
// the copy streams and events that order them against the steps.
// One block's staging copy: n doubles from src to dst and, when shadow is
// set, the same values rounded to FP32 (the mixed path's prim shadow).
struct IoSpan {
  const double* src;
  double* dst;
  float* shadow;
  long long n;
};

// Two input and two output staging buffers, used in turn: the host copy of
// the next input lands in one while the other is installed, and the result of
// a step is staged in one while the host still reads the previous result
// from the other.
struct IoPipe {
  IoSpan* spans_in[2] = {nullptr, nullptr};   // device: staging k -> prim (+ shadow), one per block
  IoSpan* spans_out[2] = {nullptr, nullptr};  // device: prim -> staging k, one per block
  cudaStream_t in = nullptr, out = nullptr;
  double* stage_in[2] = {nullptr, nullptr};
  double* stage_out[2] = {nullptr, nullptr};
  std::vector<size_t> off;     // each block's prim in a staging buffer (doubles)
  long long max_n = 0;         // the longest span
  std::vector<uint8_t> put;    // blocks put since the last io step
  int put_buf = 0;             // the input buffer the next puts fill
  int out_buf = 0;             // the output buffer the next io step fills
  int get_buf = -1;            // the output buffer gets read (the last io step's)
  cudaEvent_t in_ready[2] = {nullptr, nullptr}, in_free[2] = {nullptr, nullptr};
  cudaEvent_t out_ready[2] = {nullptr, nullptr}, out_free[2] = {nullptr, nullptr};
  bool put_waits[2] = {false, false};   // a put into buffer k waits for in_free[k] (its last install)
  bool step_waits[2] = {false, false};  // staging into buffer k waits for out_free[k] (its last gets)
  bool got[2] = {false, false};         // gets were issued from buffer k since it was filled
};

struct orion_case_s {
  int nblocks = 0;
  int prec = ORION_PREC_FP64;
  orion::ParamsDev P{};
  std::vector<orion::HostBlock> hb;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int device = 0;
  void* arena = nullptr;
  size_t arena_bytes = 0;
  std::vector<void*> allocs;  // other device allocations
  std::vector<orion::BlockDev<double>> bd64;
  std::vector<orion::BlockDev<float>> bd32;
  void* d_blocks = nullptr;
  orion::DeviceLists L;
  orion::ShardLists shard;
  long long total_interior = 0;
  cudaGraphExec_t graph = nullptr;
  long long steps_done = 0;
  int step_launches = 0;
  // submitted steps whose history has not been polled (orion_step_submit / orion_case_poll)
  orion::ResidualOut* hist_host = nullptr;  // pinned mirror of the device history ring
  long long hist_count = -1;                // device history counter; -1 = not known on the host
  long long pending_first = 0;
  int pending_n = 0;
  struct orion_group_s* group = nullptr;  // the group the case steps in, if any
  // host copies of the work lists uploaded at set-up, by device address: a
  // group is built from them without reading the lists back
  std::unordered_map<const void*, std::vector<unsigned char>> list_mirror;
  IoPipe* io = nullptr;  // orion_io_*, made on first use
};

// A group of cases stepped together: one launch per stage over all of their
// blocks.  `proxy` is a case object whose lists, block descriptors and stream
// are the group's; the stage launchers run it as they run a case.
struct orion_group_s {
  std::vector<orion_case_t> members;
  std::vector<cudaStream_t> saved_streams;  // the members' own streams, given back on destroy
  orion_case_s* proxy = nullptr;
  orion::GroupRun run;
  std::vector<int> block_off;  // each member's first block in the group's descriptors
};

namespace orion {

// Launchers of one precision (plain FP64 or mixed), compiled in their own
// translation unit with that precision's floating-point flags.
struct StageOps {
  int (*set_attributes)();
  int (*exchange)(orion_case_t);
  int (*bc)(orion_case_t);
  int (*state)(orion_case_t, bool with_dt, bool with_q);
  int (*timestep)(orion_case_t);
  int (*viscous)(orion_case_t);
  int (*average)(orion_case_t);
  int (*average_begin)(orion_case_t);  // pack own interface slots
  int (*average_end)(orion_case_t);    // average every receiving point
  int (*inviscid)(orion_case_t);
  int (*update)(orion_case_t, bool fuse_residual);
  int (*residual)(orion_case_t);
  int (*step)(orion_case_t, bool with_q);
  int (*init_flow)(orion_case_t, uint64_t seed, double amp);
  int (*skew_static)(orion_case_t, int block);
  int (*persistent_grid)(orion_case_t);
  int (*schedule)(orion_case_t, int form, int cluster_size);
  int (*prim_shadow)(orion_case_t, int block);
};

// Groups the mesh blocks into `nclusters` clusters (largest first onto the
// least-loaded cluster) and uploads each group's hyperplane chunk lists.
int build_cluster_lists(orion_case_t c, int nclusters);

const StageOps& plain_ops();
const StageOps& mixed_ops();

}  // namespace orion
