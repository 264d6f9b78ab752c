/*
 * orion_gpu.h - C ABI of the B200 (sm_100a) implementation of ORION's per-step
 * solver path.  Plain pointers and sizes only; no C++ or CUDA types cross it.
 *
 * Every function returns 0 on success and a negative ORION_E* code on error;
 * orion_last_error() returns the message of the last failing call on the
 * calling thread.  No exception crosses this boundary (the reference turns
 * exceptions into std::exit(-1), src/solver/InviscidFluxComputer.cpp:534-540;
 * here they become error codes).
 *
 * Data layout at the boundary is the reference's own: every per-block field is
 * a padded array (idim+6) x (jdim+6) x (kdim+6) [x ncomp], i fastest, component
 * slowest, exactly as OrionArray<double> stores it (src/core/OrionArray.hpp:240-261,
 * src/preprocess/FlowField.cpp:73-85), so host<->device transfers are plain copies.
 * Ghost layers: 3 (src/preprocess/FlowField.cpp:9-16).
 */
#ifndef ORION_GPU_H
#define ORION_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORION_GPU_ABI_VERSION 1

/* error codes */
#define ORION_OK 0
#define ORION_E_INVALID (-1)   /* bad argument */
#define ORION_E_CUDA (-2)      /* CUDA runtime error */
#define ORION_E_NOMEM (-3)     /* device allocation failed */
#define ORION_E_UNSUPPORTED (-4)
#define ORION_E_NUMERIC (-5)   /* non-finite residual */
#define ORION_E_TIMEOUT (-6)   /* a bounded device wait gave up */

/* precision of a case */
#define ORION_PREC_FP64 0      /* plain form: every stage in FP64 */
#define ORION_PREC_MIXED 1     /* FP32 flux/viscous/LU-SGS increments; FP64 metrics, Q update, norms */

/* Forms of the LU-SGS / GS hyperplane sweeps (all give the reference's
 * Gauss-Seidel order; they differ in how hyperplanes are separated). */
#define ORION_SWEEP_PLANES 0   /* one launch per hyperplane */
#define ORION_SWEEP_GRID 1     /* one cooperative launch, bounded grid barrier per hyperplane */
#define ORION_SWEEP_CLUSTER 2  /* thread-block clusters (8 or 16 CTAs), cluster barrier per hyperplane */
#define ORION_SWEEP_TILES 3    /* one launch per pass: 32x4-line tiles, each waiting only on its upstream
                                  neighbour tiles' progress (bounded waits); the default */

/* BC types (src/bc/PhysicalBC.cpp:576-613) */
#define ORION_BC_INTERFACE (-1)
#define ORION_BC_WALL 2
#define ORION_BC_SYMMETRY 3
#define ORION_BC_FARFIELD 4
#define ORION_BC_FREESTREAM 5
#define ORION_BC_EXTRAPOLATION 6

/* fields of a block (names of src/preprocess/FlowField.hpp:19-71) */
#define ORION_FIELD_PRIM 0     /* 6 comps: rho,u,v,w,p,T */
#define ORION_FIELD_Q 1        /* 5 comps: conservative variables */
#define ORION_FIELD_DQ 2       /* 5 comps: residual / increment */
#define ORION_FIELD_METRICS 3  /* 9 comps: xi_x..zeta_z (times Jacobian) */
#define ORION_FIELD_VOL 4      /* 1 comp */
#define ORION_FIELD_DT 5       /* 1 comp: dt_phys / vol */
#define ORION_FIELD_C 6        /* 1 comp: speed of sound */
#define ORION_FIELD_MU 7       /* 1 comp: laminar viscosity */

/* Flow parameters read by the hot path (subset of core::Params,
 * src/core/Params.hpp:9-120, after init_inflow, src/preprocess/Inflow.cpp:300-459). */
typedef struct {
  double gamma;    /* inflow.gama */
  double moo;      /* inflow.moo */
  double reynolds; /* inflow.reynolds */
  double prl;      /* inflow.prl */
  double cfl;      /* step.cfl */
  double twall;    /* inflow.twall (<= 1e-6: adiabatic wall) */
  double tref;     /* inflow.tref */
  double visc;     /* inflow.visc = 110.4 / tref (Sutherland constant) */
  double roo, uoo, voo, woo, poo, too; /* non-dimensional freestream */
  int nvis;        /* flowtype.nvis: 1 = Navier-Stokes */
  int method;      /* control.method: 1 = finite difference */
  int ntmst;       /* step.ntmst */
  int csrv;        /* technic.csrv (an int in the reference) */
} orion_params_t;

/* One BC window (src/bc/BCData.hpp:8-54), 1-based inclusive point ranges. */
typedef struct {
  int s_st[3], s_ed[3];
  int bctype;
  int t_st[3], t_ed[3]; /* interfaces only */
  int nbt;              /* interfaces only: target block, 1-based */
  int ibcwin;           /* interfaces only: target region, 1-based */
} orion_region_t;

typedef struct {
  int idim, jdim, kdim;           /* interior grid points */
  int nregions;
  const orion_region_t* regions;  /* in file order */
} orion_block_desc_t;

/* Residual statistics of one step (ResidualStats, src/solver/ResidualMonitor.hpp:8-12)
 * plus the local physical time step (TimeIntegrator, params.step.phydtime). */
typedef struct {
  double rms;
  double max;
  int max_loc[5];   /* block (0-based), i, j, k (1-based interior), var (1-based) */
  int pad;
  double phydtime;
} orion_residual_t;

typedef struct orion_case_s* orion_case_t;
typedef struct orion_group_s* orion_group_t;

/* A step schedule: sweep form, cluster size (CLUSTER form: 8 or 16; 0 = the
 * largest co-resident) and the grid lines per CTA of the viscous and inviscid
 * line kernels (1-32).  ms_per_step is filled by orion_case_autotune. */
typedef struct {
  int sweep_form;
  int cluster_size;
  int lanes;
  float ms_per_step;
} orion_schedule_t;

const char* orion_last_error(void);
int orion_abi_version(void);

/* Device and case lifetime --------------------------------------------------
 * Replaces the CUDA backend hook the reference's build expects
 * (src/CMakeLists.txt:50-58 names backend/cuda/BackendCUDA.cu; the CPU hook is
 * backend_cpu_init(), src/backend/cpu/BackendCPU.cpp:3-6). */
int orion_gpu_init(int device);

/* Creates a device-resident case: allocates every block's fields in one arena
 * and builds the halo-copy, BC-phase and interface-averaging work lists from
 * the region lists (the maps of src/bc/BCPreprocess.cpp:16-192). */
int orion_case_create(int nblocks, const orion_block_desc_t* blocks, const orion_params_t* params,
                      int precision, orion_case_t* out);
int orion_case_destroy(orion_case_t c);
/* Replaces the case's parameters (the reference passes core::Params to every
 * stage call, InviscidFluxComputer.hpp:17-18 and the others); takes effect
 * from the next launch, the captured step graph is rebuilt. */
int orion_case_set_params(orion_case_t c, const orion_params_t* params);
/* Optional: run on a caller-provided cudaStream_t (passed as void*); NULL = the case's own stream. */
int orion_case_set_stream(orion_case_t c, void* stream);
int orion_case_sync(orion_case_t c);
/* The cudaStream_t (as void*) the case enqueues on, for timing with events. */
int orion_case_stream(orion_case_t c, void** stream);
/* Kernel launches one captured step issues (after the first orion_step). */
int orion_case_step_launches(orion_case_t c, int* n);
/* How the implicit sweeps are scheduled: out[0] = mode (0 one launch per
 * hyperplane, 1 persistent cooperative grid, 2 thread-block clusters, 3 tile
 * wavefront), out[1] = CTAs (grid), clusters or forward tiles, out[2] = CTAs per cluster, out[3] = threads
 * per CTA, out[4] = hyperplanes of the longest sweep.  Waits for set-up only. */
int orion_case_sweep_schedule(orion_case_t c, int out[5]);
/* Device bytes held by the case (the HBM footprint used for admission). */
int orion_case_footprint(orion_case_t c, size_t* bytes);
size_t orion_footprint_estimate(int nblocks, const orion_block_desc_t* blocks, int precision);

/* Host <-> device copies of one block field (reference layout, FP64). */
int orion_case_upload(orion_case_t c, int block, int field, const double* host);
int orion_case_download(orion_case_t c, int block, int field, double* host);

/* Set-up on the device: freestream + seeded noise on rho and u + EOS
 * temperature (initialize_flow / update_temperature,
 * src/preprocess/InitialCondition.cpp:7-147).  Noise: splitmix64(seed), draws
 * 2n+1 and 2n+2 scale rho and u at padded point n (blocks in order, k,j,i). */
int orion_case_init_flow(orion_case_t c, uint64_t seed, double amp);

/* Grid metrics and Jacobian of one block computed on the device into the
 * case's METRICS and VOL fields (compute_grid_metrics + check_grid_metrics,
 * src/mesh/MetricComputer.cpp:103-500): x,y,z are the block's host
 * coordinates, idim*jdim*kdim, i fastest (Plot3D order).  Bit-identical to
 * orion_grid_metrics_host; gcl=1 selects the Visbal conservative form.  Waits. */
int orion_case_grid_metrics(orion_case_t c, int block, const double* x, const double* y, const double* z, int gcl);

/* Solution output of one block (the fields PostProcess::write_solution
 * writes, src/postprocess/PostProcess.cpp:116-243): host receives 7 arrays of
 * idim*jdim*kdim floats, i fastest: density, pressure, temperature, Mach
 * (sqrt(|u|^2 / (gamma p / rho)) in FP64, 0 where gamma p / rho <= 1e-30),
 * u, v, w.  Packed on the device, then copied; waits. */
int orion_case_pack_output(orion_case_t c, int block, float* host);

/* Grid metrics and Jacobian of one block on the host (compute_grid_metrics +
 * check_grid_metrics, src/mesh/MetricComputer.cpp:103-500): x,y,z are
 * idim*jdim*kdim, i fastest; metrics (9 comps) and vol are written in the
 * padded layout, ghosts zero.  gcl=1 selects the Visbal conservative form. */
int orion_grid_metrics_host(int idim, int jdim, int kdim, const double* x, const double* y,
                            const double* z, int gcl, double* metrics, double* vol);

/* Per-stage entry points, one per reference static method -------------------
 * Each enqueues its kernels on the case stream and returns without waiting. */
int orion_exchange_bc(orion_case_t c);                 /* HaloExchanger::exchange_bc, HaloExchanger.hpp:20-21 */
int orion_apply_physical_bc(orion_case_t c);           /* bc::apply_physical_bc, PhysicalBC.hpp:17-19 */
int orion_update_flow_states(orion_case_t c);          /* StateUpdater::update_flow_states, StateUpdater.hpp:14-15 */
int orion_calculate_time_step(orion_case_t c);         /* TimeIntegrator::calculate_time_step, TimeIntegrator.hpp:10-11 */
int orion_compute_viscous_rhs(orion_case_t c);         /* FluxComputer::compute_viscous_rhs, FluxComputer.hpp:15-16 */
int orion_average_interface_residuals(orion_case_t c); /* HaloExchanger::average_interface_residuals, HaloExchanger.hpp:25 */
int orion_compute_inviscid_rhs(orion_case_t c);        /* InviscidFluxComputer::compute_inviscid_rhs, InviscidFluxComputer.hpp:17-18 */
int orion_update_solution(orion_case_t c);             /* StateUpdater::update_solution, StateUpdater.hpp:21-23 */
int orion_residual_compute(orion_case_t c, orion_residual_t* out); /* ResidualMonitor::compute, ResidualMonitor.hpp:20-21 (waits) */
int orion_phydtime(orion_case_t c, double* out);       /* params.step.phydtime after the last time step (waits) */

/* Whole steps in the order of OrionSolver::solve (src/core/OrionSolver.cpp:141-209,
 * without its debug block).  The step is captured once as a CUDA graph and
 * replayed; residual statistics of every step go to a device history that is
 * copied to `hist` (nsteps entries) when hist is not NULL.  Waits. */
int orion_step(orion_case_t c, int nsteps, orion_residual_t* hist);
/* Same, but enqueue only (no wait, no history copy); for overlapping cases. */
int orion_step_async(orion_case_t c, int nsteps);
/* Copies the residual of the most recent step (waits). */
int orion_last_residual(orion_case_t c, orion_residual_t* out);

/* Applies a schedule (deterministic: use it to fix a tuned choice).  Results
 * do not depend on the lanes; on the plain path they do not depend on the
 * sweep form either (the same operations in the same order). */
int orion_case_set_schedule(orion_case_t c, const orion_schedule_t* s);
int orion_case_get_schedule(orion_case_t c, orion_schedule_t* s);
/* Autotuner: times candidate schedules on this case (line lanes 8/16/32 with
 * the current sweep form, then every sweep form the device supports with the
 * best lanes), steps_per_trial timed steps each after one warm-up step, and
 * applies the fastest.  The state (prim, the step counter) is saved before and
 * restored after every trial, so tuning leaves the solution where it was; the
 * next whole step recomputes every derived field.  Fills trials[0..*ntrials)
 * (cap entries at most) and *best.  Waits; no steps may be pending. */
int orion_case_autotune(orion_case_t c, int steps_per_trial, orion_schedule_t* trials, int cap, int* ntrials,
                        orion_schedule_t* best);

/* Non-blocking stepping for request loops that keep many cases in flight.
 * orion_step_submit enqueues nsteps whole steps on the case's stream and an
 * asynchronous copy of their residual history (the per-step
 * ResidualMonitor::compute result, ResidualMonitor.hpp:20-21) into a pinned
 * ring the case owns, and returns at once.  At most 4096 steps may be
 * submitted and not yet polled.  The first call on a case waits once to read
 * the device's step counter.
 * orion_case_poll returns 0 while submitted steps are still running, and 1
 * when the case's stream is idle, after copying up to cap of the finished
 * steps' history entries, oldest first, to out (*n of them; the rest stay for
 * the next poll).  It never waits. */
int orion_step_submit(orion_case_t c, int nsteps);
int orion_case_poll(orion_case_t c, orion_residual_t* out, int cap, int* n);

/* Pipelined host I/O of the primitive state ------------------------------
 * The reference's driver loop reads and writes host arrays around every step
 * (OrionSolver.cpp:139-209 over the host FlowFieldSet, FlowField.hpp:73-87);
 * orion_case_upload / orion_case_download are that, one blocking copy at a
 * time.  These calls stream states through a case with the copies overlapping
 * the steps, for a sequence of independent inputs (each io step's input comes
 * from the host, its result goes back to the host):
 *   orion_io_put   enqueues the copy of one block's prim (6 x npad doubles,
 *                  the upload layout) from PINNED host memory into the case's
 *                  input staging, on the case's input copy stream;
 *   orion_io_step  on the case's stream: installs the blocks put since the
 *                  last io step into prim, runs nsteps whole steps with their
 *                  residual history copied as orion_step_submit does (poll it
 *                  with orion_case_poll), then copies prim to the output
 *                  staging; returns at once;
 *   orion_io_get   enqueues the copy of one block's prim as the last io step
 *                  left it into PINNED host memory, on the output copy stream;
 *   orion_io_wait  waits for every copy and step enqueued.
 * Input and output staging are double-buffered: the puts for the next io step
 * fill one input buffer while the current one is installed, and an io step
 * stages its result in one output buffer while the gets of the previous step
 * still read the other.  The device orders them: a put reuses a buffer once
 * the io step two back has installed it, and an io step overwrites an output
 * buffer only after the gets issued from it have read it.  Results are
 * bit-identical to upload, step, download.  Host buffers stay untouched by the
 * caller until orion_io_wait (pageable memory works but does not overlap).
 * Not for shards or grouped cases. */
int orion_io_put(orion_case_t c, int block, const double* host);
int orion_io_step(orion_case_t c, int nsteps);
int orion_io_get(orion_case_t c, int block, double* host);
int orion_io_wait(orion_case_t c);

/* Groups of cases: many cases, one launch per stage ------------------------
 * No single counterpart in the reference, which steps the blocks of one case
 * one after another in every stage (StateUpdater.cpp:544-580,
 * InviscidFluxComputer.cpp:524-541, FluxComputer.cpp:724-732).  A group steps
 * several device-resident cases together: every stage is one launch over the
 * blocks of all members (the sweeps: one launch per hyperplane, or per pass
 * in the tile form when every member uses it), each block with its own
 * case's parameters; the residual and time-step reductions run per member,
 * into the member's own history.  A member's results are bit-identical to
 * stepping it alone.  The members share one precision and are all viscous or
 * all Euler; they have no unpolled submitted steps; a case joins at most one
 * group.  While in a group a case enqueues on the group's stream, so
 * orion_case_poll and the per-case calls follow the group's launches; destroy
 * the group before destroying or re-grouping its cases.
 * orion_group_submit enqueues nsteps group steps (one CUDA graph per step)
 * and each member's history copy, and returns at once; poll each member with
 * orion_case_poll.  orion_group_sync waits for the group's stream. */
int orion_group_create(int n, const orion_case_t* cases, orion_group_t* out);
int orion_group_submit(orion_group_t g, int nsteps);
int orion_group_sync(orion_group_t g);
int orion_group_step_launches(orion_group_t g, int* n);
int orion_group_destroy(orion_group_t g);

/* Allocation-free residual norm of one block ------------------------------
 * No counterpart in the reference.  For callers that cannot call cudaMalloc
 * where they need the residual (a solver that reserves its whole device budget
 * up front, a loop inside another framework's memory pool, a step that must not
 * let an allocation synchronize the device): computes the statistics of
 * orion_residual_compute for ONE block (rms, max and its location; phydtime
 * is written as 0, since in the case-based path it is the time-step stage's
 * dt minimum, which this call does not run) from device pointers the caller
 * owns (dq: 5 comps, vol, dt: padded layout, FP64) and writes them to the host
 * struct `out`, waiting for `stream` (a cudaStream_t as void*, NULL = default).
 * Its scratch is a fixed array in the library's device memory, so blocks are
 * limited to ORION_NOALLOC_MAX_POINTS interior points (larger ones get
 * ORION_E_INVALID).  Every call looks up that array's address in the current
 * context; the first call on a device may load the library's device code, so
 * make it before any stream capture on that device.  The call synchronizes
 * `stream`, so it never runs on a capturing stream: it returns ORION_E_INVALID
 * there.  All calls on a device share the array: calls that overlap on the GPU
 * (different streams, or threads without ordering) race and must not be
 * issued. */
#define ORION_NOALLOC_MAX_POINTS 8388608
int orion_residual_block_noalloc(const double* dq, const double* vol, const double* dt, int idim, int jdim,
                                 int kdim, void* stream, orion_residual_t* out);

/* Block sharding ----------------------------------------------------------
 * Replaces the MPI call sites of the step (one process per GPU, blocks spread
 * over the processes, ORION's src/solver/HaloExchanger.cpp:70-179 and :186-398
 * and the reductions of src/solver/ResidualMonitor.cpp:11-137).
 * orion_case_create_shard takes the GLOBAL block list, identical on every
 * shard, and owner[b], the shard (0 .. nshards-1) of global block b; the case
 * holds the blocks owner[b] == rank, ascending (local block i is global block
 * global_ids[i], orion_shard_blocks).  Every shard owns at least one block.
 * A shard steps through the per-stage entry points in OrionSolver::solve's
 * order, with the two exchanges between shards done by the caller:
 *   orion_exchange_bc (pairs inside the shard), then for every peer
 *     orion_shard_pack(HALO) -> send, receive -> orion_shard_unpack(HALO);
 *   orion_shard_average_begin, for every peer orion_shard_pack(IFACE) -> send,
 *     receive -> orion_shard_unpack(IFACE), then orion_shard_average_end
 *     (in place of orion_average_interface_residuals);
 *   orion_shard_residual, then sum `sum`, take the max of `max` (the smallest
 *     key among equal maxima) and the min of `dtmin` over the shards:
 *     rms = sqrt(sum / (5 points)); key / 5 is the global interior point
 *     (blocks in global order, then k, j, i) and key % 5 the component.
 * Buffers are FP64 device memory of orion_shard_counts' sizes (doubles); pack
 * and unpack are enqueued on the case's stream.  The lists of a pair of shards
 * agree element for element: each shard derives them from the global list.
 * The graph-captured step, orion_average_interface_residuals and
 * orion_residual_compute return ORION_E_INVALID on a shard of several. */
#define ORION_XCHG_HALO 0   /* exchange_bc: primitive elements */
#define ORION_XCHG_IFACE 1  /* average_interface_residuals: packed dq/vol, 5 per point */
typedef struct {
  double sum;       /* sum of squared residuals of the shard's points */
  double max;       /* largest residual of the shard */
  long long key;    /* 5 * global interior point + component of the max */
  double dtmin;     /* min(1000, min dt*vol) of the shard (phydtime) */
  long long points; /* interior points of ALL shards */
} orion_shard_residual_t;
int orion_case_create_shard(int nblocks, const orion_block_desc_t* blocks, const int* owner, int rank,
                            const orion_params_t* params, int precision, orion_case_t* out);
int orion_shard_blocks(orion_case_t c, int* nlocal, int* global_ids);
int orion_shard_counts(orion_case_t c, int kind, int peer, long long* nsend, long long* nrecv);
int orion_shard_pack(orion_case_t c, int kind, int peer, double* buf);
int orion_shard_unpack(orion_case_t c, int kind, int peer, const double* buf);
int orion_shard_average_begin(orion_case_t c);
int orion_shard_average_end(orion_case_t c);
int orion_shard_residual(orion_case_t c, orion_shard_residual_t* out); /* waits */
/* Host only (no device use): the doubles shard `rank` sends to and receives
 * from every shard, nsend[s] / nrecv[s] for s in 0 .. max(owner). */
int orion_shard_plan_counts(int nblocks, const orion_block_desc_t* blocks, const int* owner, int rank, int kind,
                            long long* nsend, long long* nrecv);

#ifdef __cplusplus
}
#endif

#endif /* ORION_GPU_H */
