#!/usr/bin/env python
"""Benchmark of the B200 per-step solver path (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config C] [--impl ours|reference]

Workload (default --config 3): bump channel 385x257x129 points (13.3M) in 64
seeded uneven blocks, Mach 0.8, Re 1e5, synthetic initial state (freestream +
1% seeded noise).  A step is one full solver time step of the whole case.
`value` is the mixed-precision batched path (FP32 flux / viscous / LU-SGS
increments, FP64 metrics, Q update and norms); the plain FP64 path is timed
beside it, and the relative L2 error of the mixed state against the plain
state is taken after L2_STEPS steps from the same initial state, and at
several horizons of the workload and of configuration 0 (L2_HORIZONS).  Every GPU runs its own replica (weak scaling, no
collective on the data path); times are CUDA events, max over ranks.

--impl reference times the reference's own CPU implementation (compiled from
its sources into oracle/_ref) on a bounded sample of the same workload: some
of its blocks, each run as a standalone case by one reference process, all
processes concurrently on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
# 32 hardware work queues for the serving run's many streams (read when the
# CUDA context is made, so set before torch touches the GPU)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

METRIC = "cell-updates/s/GPU plain vs mixed-batched at ≤1e-6 L2 err; p50/p99 solve ms"
UNIT = "cell-updates/s"
FALLBACK_HBM_GBS = 6650.0

# Algorithmic bytes per grid point of each stage (each stage reads its inputs
# and writes its outputs once): (plain FP64, mixed).
STAGE_BYTES = {
    "state": (144, 112), "timestep": (136, 124), "viscous": (200, 152), "inviscid": (192, 152),
    "update_solution": (1184, 892), "residual": (56, 32),
}
STEP_BYTES = (1912, 1444)

# DRAM bytes per grid point that ncu measured for the update stage's kernels
# (mixed path, C1 = 1,254,792 points: k_lusgs_prep 176.3 MB + k_sweep_pairs
# 218.5 MB + the 704 k_sweep_plane launches of one step 1,220.6 MB +
# k_sweep_finish 118.8 MB; ncu flushes caches per launch, so this is an upper
# bound); scaled to the bench workload by its point count.
UPDATE_DRAM_BYTES_PER_POINT_MIXED = 1734.2e6 / 1254792

# The mixed state is compared with the plain FP64 state from the same initial
# state at several horizons: on the bench workload (transonic, 64 blocks, whose
# flow the reference's own scheme does not converge) and on configuration 0
# (one block, converging).
L2_STEPS = 10
L2_HORIZONS = {"workload": (10, 30, 50), "c0_97x49x33": (10, 50, 100, 200), "c2_289x161x65_27blk": (10, 50, 100)}
# the reference-CPU leg of the line: timed steps after warm-up steps per process
CPU_STEPS, CPU_WARMUP = 5, 2


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, TypeError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


# ---------------------------------------------------------------------------
# clocks sampler
# ---------------------------------------------------------------------------
class Clocks:
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:  # no nvidia-smi: the line says "unsampled"
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 7:
                continue
            try:
                sm.append(float(p[0]))
                smax = float(p[1])
            except ValueError:
                continue
            for n, v in zip(names, p[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# reference CPU measurement (oracle/_ref harness)
# ---------------------------------------------------------------------------
def standalone_block_case(case, b):
    """One block of `case` as its own case: interface faces closed with
    zero-gradient extrapolation (type 6), physical BCs kept."""
    from orion_b200 import cases as C
    blk = case.blocks[b]
    nb = C.Block(blk.idim, blk.jdim, blk.kdim, blk.x, blk.y, blk.z, [])
    for r in blk.regions:
        if r.bctype < 0:
            nb.regions.append(C.Region(r.s_st, r.s_ed, C.BC_EXTRAPOLATION))
        else:
            nb.regions.append(C.Region(r.s_st, r.s_ed, r.bctype))
    return C.Case(f"{case.name}_blk{b}", [nb], case.params, case.noise_seed, case.noise_amp, 1)


def reference_sample(case, steps: int, warmup: int, procs: int):
    harness = os.path.join(ROOT, "oracle", "_ref", "orion_ref_harness")
    if not os.path.exists(harness):
        return None, "reference build oracle/_ref missing"
    nblk = len(case.blocks)
    procs = max(1, min(procs, nblk))
    picks = [int(round(i * (nblk - 1) / max(procs - 1, 1))) for i in range(procs)] if procs > 1 else [0]
    tmp = tempfile.mkdtemp(prefix="orion_refbench_")
    runs = []
    for n, b in enumerate(picks):
        sub = standalone_block_case(case, b)
        d = os.path.join(tmp, f"c{n}")
        sub.write_reference_inputs(d)
        os.makedirs(d + "/out", exist_ok=True)
        runs.append((d, sub.npoints))
    ps = [subprocess.Popen([harness, d, str(steps), d + "/out", "--time-only", "--warmup", str(warmup)],
                           stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True) for d, _ in runs]
    secs, pts = [], 0
    for p, (_, npts) in zip(ps, runs):
        out, _ = p.communicate()
        rec = json.loads(out.strip().splitlines()[-1])
        secs.append(rec["seconds"])
        pts += npts
    value = pts * steps / max(secs)
    sample = (f"{procs} of the {nblk} blocks of {case.name}, each a standalone reference case "
              f"(interfaces closed by zero-gradient BCs), {steps} timed steps after {warmup} warm-up, "
              f"{procs} concurrent single-rank processes; {pts} points")
    return {"value": value, "unit": UNIT, "cores": procs, "kind": "reference", "sample": sample}, None


# ---------------------------------------------------------------------------
def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=24,
                    help="requests of the bounded serving run (0: skip it)")
    ap.add_argument("--serve-max-steps", type=int, default=300)
    ap.add_argument("--serve-drop", type=float, default=0.1,
                    help="residual drop at which a served request retires (the bounded stream)")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    from orion_b200 import cases
    case = cases.config(args.config)

    if args.impl == "reference":
        if rank != 0:
            return
        ncpu = os.cpu_count() or 1
        rec, err = reference_sample(case, args.steps, args.warmup, min(ncpu, len(case.blocks)))
        if rec is None:
            print(json.dumps({"impl": "reference", "unavailable": err}))
            return
        line = {"impl": "reference", "metric": METRIC, "value": rec["value"], "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": case.name, "points": case.npoints, "blocks": len(case.blocks)},
                "cpu_baseline": rec,
                "e2e": {"value": rec["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    from orion_b200 import _lib, replicas, solver
    group = replicas.from_env()
    K, W = args.steps, args.warmup
    npts = case.npoints
    barrier, max_over_ranks = group.barrier, group.max_over_ranks

    def timed_steps(fs, nsteps):
        s = torch.cuda.ExternalStream(fs.stream_ptr())
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        e0.record(s)
        fs.step_async(nsteps)
        e1.record(s)
        e1.synchronize()
        barrier()
        return max_over_ranks(e0.elapsed_time(e1))

    clocks = Clocks(local)
    results = {}
    states = {}
    def interior(fs):
        return [fs.download(b, "prim")[:5, 3:-3, 3:-3, 3:-3] for b in range(len(fs.case.blocks))]

    def rel_l2(a, b):
        num = sum(float(np.sum((x - y) ** 2)) for x, y in zip(a, b))
        return (num / sum(float(np.sum(y ** 2)) for y in b)) ** 0.5

    horizon_states = {}
    for name, prec in (("mixed", _lib.PREC_MIXED), ("plain", _lib.PREC_FP64)):
        fs = solver.FlowFieldSet(case, precision=prec, device=local)
        done = 0
        for hz in L2_HORIZONS["workload"]:
            fs.step(hz - done)
            done = hz
            horizon_states[(name, "workload", hz)] = interior(fs)
            if hz == L2_STEPS:
                states[name] = horizon_states[(name, "workload", hz)]
        tune = fs.autotune(steps_per_trial=3)  # schedule chosen by timing on this case; solution unchanged
        fs.step(W)
        if name == "mixed":
            clocks.start()
        ms = timed_steps(fs, K)
        results[name] = {"ms": ms, "launches": fs.step_launches(), "fs": fs, "sweeps": fs.sweep_schedule(),
                         "tune": tune}
        if name == "plain":
            clk = clocks.stop()
    # L2 error of the mixed state against the plain FP64 state after L2_STEPS
    # steps, and at the horizons of the workload and of configuration 0
    l2 = rel_l2(states["mixed"], states["plain"])
    l2_horizons = {"workload": {str(hz): rel_l2(horizon_states[("mixed", "workload", hz)],
                                                horizon_states[("plain", "workload", hz)])
                                for hz in L2_HORIZONS["workload"]}}
    for cfg, key in ((0, "c0_97x49x33"), (2, "c2_289x161x65_27blk")):
        cc = cases.config(cfg)
        cc_states = {}
        for name, prec in (("mixed", _lib.PREC_MIXED), ("plain", _lib.PREC_FP64)):
            f0 = solver.FlowFieldSet(cc, precision=prec, device=local)
            done = 0
            for hz in L2_HORIZONS[key]:
                f0.step(hz - done)
                done = hz
                cc_states[(name, hz)] = interior(f0)
            f0.close()
        l2_horizons[key] = {str(hz): rel_l2(cc_states[("mixed", hz)], cc_states[("plain", hz)])
                            for hz in L2_HORIZONS[key]}
    per_rank_pts = npts * K
    mixed_ms, plain_ms = results["mixed"]["ms"], results["plain"]["ms"]
    value = group.aggregate_rate(per_rank_pts, mixed_ms / 1e3)
    plain_value = group.aggregate_rate(per_rank_pts, plain_ms / 1e3)

    # per-stage timing of one step on the mixed case -> dominant stage roofline
    fsm = results["mixed"]["fs"]
    s = torch.cuda.ExternalStream(fsm.stream_ptr())
    stage_ops = [
        ("exchange_bc", lambda: solver.HaloExchanger().exchange_bc(None, fsm)),
        ("apply_physical_bc", lambda: solver.apply_physical_bc(None, fsm)),
        ("state", lambda: solver.StateUpdater.update_flow_states(fsm)),
        ("timestep", lambda: _lib.check(_lib.load().orion_calculate_time_step(fsm.handle))),
        ("viscous", lambda: solver.FluxComputer.compute_viscous_rhs(fsm)),
        ("average", lambda: solver.HaloExchanger().average_interface_residuals(None, fsm)),
        ("inviscid", lambda: solver.InviscidFluxComputer.compute_inviscid_rhs(fsm)),
        ("average2", lambda: solver.HaloExchanger().average_interface_residuals(None, fsm)),
        ("update_solution", lambda: solver.StateUpdater.update_solution(fsm)),
        ("residual", lambda: solver.ResidualMonitor.compute(fsm)),
    ]
    stage_ms = {}
    for rep in range(3):
        for nm, fn in stage_ops:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(s)
            fn()
            e1.record(s)
            e1.synchronize()
            if rep > 0:
                stage_ms.setdefault(nm, []).append(e0.elapsed_time(e1))
    stage_ms = {k: float(np.mean(v)) for k, v in stage_ms.items()}
    peak, peak_kind = hbm_peak()
    dom = max((k for k in stage_ms if k in STAGE_BYTES), key=lambda k: stage_ms[k])
    bpp = STAGE_BYTES[dom][1]
    achieved = bpp * npts / (stage_ms[dom] / 1e3) / 1e9
    traffic = None
    if dom == "update_solution":
        traffic = UPDATE_DRAM_BYTES_PER_POINT_MIXED * npts
        dom = "update_solution (k_lusgs_prep, k_sweep_pairs, k_sweep_plane x 4 passes, k_sweep_finish)"
    roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "peak_kind": f"{peak_kind} hbm_gbs",
                "bytes_per_point": bpp, "points_per_launch": npts,
                "traffic_source": "ncu dram__bytes_read+write of the stage's kernels on C1, scaled by points"}
    step_gbs = STEP_BYTES[1] * (value / world) / 1e9
    step_roofline = {"mixed_achieved_gbs": step_gbs, "mixed_frac": step_gbs / peak,
                     "plain_achieved_gbs": STEP_BYTES[0] * (plain_value / world) / 1e9,
                     "plain_frac": STEP_BYTES[0] * (plain_value / world) / 1e9 / peak}

    # end to end through the C ABI with host buffers.  Pipelined (orion_io_*,
    # the headline): every step copies a state (prim of every block) in from
    # pinned host memory and its result and residual back out to pinned host
    # memory, on copy streams that overlap the neighbouring steps; the inputs
    # are a stream of states (here the same buffers every step).  Blocking
    # (orion_case_upload, orion_step, orion_case_download): the same copies,
    # one after another, each step's input the previous step's output.
    fse = results["mixed"]["fs"]
    host_prim = [torch.from_numpy(fse.download(b, "prim").reshape(-1)).pin_memory() for b in range(len(case.blocks))]
    host_out = [torch.empty_like(t).pin_memory() for t in host_prim]
    lib = _lib.load()
    h2d = sum(int(t.numel()) * 8 for t in host_prim)
    d2h = h2d + 48
    import ctypes as C
    res = _lib.Residual()
    ne = max(2, K)  # the whole job: the first input's copy and the last result's copy included

    def io_round():
        for b, t in enumerate(host_prim):
            fse.io_put(b, t)
        fse.io_step(1)
        for b, t in enumerate(host_out):
            fse.io_get(b, t)

    io_round()  # staging buffers and copy streams made on first use
    fse.io_wait()
    fse.poll()
    barrier()
    t0 = time.perf_counter()
    for _ in range(ne):
        io_round()
    fse.io_wait()
    io_hist = fse.poll()
    assert io_hist is not None and len(io_hist) == ne
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = group.aggregate_rate(npts * ne, e2e_s)

    barrier()
    t0 = time.perf_counter()
    for _ in range(ne):
        for b, t in enumerate(host_prim):
            _lib.check(lib.orion_case_upload(fse.handle, b, _lib.FIELD_PRIM, C.c_void_p(t.data_ptr())))
        _lib.check(lib.orion_step(fse.handle, 1, C.byref(res)))
        for b, t in enumerate(host_prim):
            _lib.check(lib.orion_case_download(fse.handle, b, _lib.FIELD_PRIM, C.c_void_p(t.data_ptr())))
    torch.cuda.synchronize()
    e2e_blocking = group.aggregate_rate(npts * ne, max_over_ranks(time.perf_counter() - t0))

    # bounded serving run: seeded request stream (Poisson arrivals, mixed sizes and
    # flow conditions), continuous batching on the mixed path against the same
    # requests served one at a time on the plain FP64 path
    ws_gb = fsm.footprint() / 1e9
    serving_out = None
    if args.serve_requests > 0:
        from orion_b200 import serving
        for r in results.values():
            r["fs"].close()
        reqs = serving.c4_requests(args.serve_requests, seed=4, mean_ms=50.0, max_steps=args.serve_max_steps,
                                   drop=args.serve_drop)
        srv = serving.Server(_lib.PREC_MIXED, device=local, quantum=20)  # every resident case on its own stream
        mixed_s = serving.summarize(srv.run(reqs))
        mixed_s["peak_resident_cases"] = srv.peak_resident
        mixed_s["mode"] = "streams: every resident case on its own stream (the default)"
        srv_group = serving.Server(_lib.PREC_MIXED, device=local, quantum=20, batched=True)
        group_s = serving.summarize(srv_group.run(reqs))
        group_s["peak_resident_cases"] = srv_group.peak_resident
        group_s["mode"] = "group: one launch per stage over all resident cases"
        seq = serving.Server(_lib.PREC_FP64, device=local, quantum=20, max_active=1, batched=False)
        plain_s = serving.summarize(seq.run(reqs))
        peak, _kind = hbm_peak()
        for sm, nb in ((mixed_s, STEP_BYTES[1]), (group_s, STEP_BYTES[1]), (plain_s, STEP_BYTES[0])):
            sm["hbm_gbs"] = sm["cell_updates_per_s"] * nb / 1e9
            sm["hbm_frac"] = sm["hbm_gbs"] / peak
        serving_out = {"requests": args.serve_requests, "max_steps": args.serve_max_steps, "drop": args.serve_drop,
                       "mean_interarrival_ms": 50.0,
                       "mixed_continuous": mixed_s, "mixed_continuous_group": group_s,
                       "plain_one_at_a_time": plain_s,
                       "throughput_ratio": mixed_s["cell_updates_per_s"] / plain_s["cell_updates_per_s"],
                       "vs_single_case_mixed": mixed_s["cell_updates_per_s"] / (value / world)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ncpu = os.cpu_count() or 1
        cpu, err = reference_sample(case, CPU_STEPS, CPU_WARMUP, min(ncpu, len(case.blocks)))
        if cpu is None:
            cpu = {"value": None, "unit": UNIT, "cores": 0, "kind": "reference", "sample": err}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": mixed_ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64 (mixed)", "data": "synthetic",
            "config": {"workload": case.name + " mixed-batched", "points": npts, "blocks": len(case.blocks),
                       "mach": case.params.moo, "reynolds": case.params.reynolds,
                       "l2_flush": "none needed: working set %.1f GB per GPU > 126 MB L2" %
                                   ws_gb},
            "plain_fp64": {"value": plain_value, "unit": UNIT, "ms_per_step": plain_ms / K, "dtype": "f64"},
            "mixed_over_plain": plain_ms / mixed_ms,
            "sweep_schedule": {"mixed": results["mixed"]["sweeps"], "plain": results["plain"]["sweeps"]},
            "autotune": {"mixed": results["mixed"]["tune"], "plain": results["plain"]["tune"]},
            "mixed_vs_plain_rel_l2": l2, "mixed_vs_plain_l2_after_steps": L2_STEPS,
            "mixed_vs_plain_rel_l2_horizons": l2_horizons,
            "roofline": roofline, "step_roofline": step_roofline,
            "stage_ms": stage_ms,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": ne, "mode": "pipelined: orion_io_put / orion_io_step / orion_io_get, copies overlap steps",
                    "blocking_value": e2e_blocking},
            "serving": serving_out,
            "gpu_launches": results["mixed"]["launches"] * K,
            "clocks": clk,
        }
        print(json.dumps(line))
    for r in results.values():
        r["fs"].close()
    group.close()


if __name__ == "__main__":
    main()
