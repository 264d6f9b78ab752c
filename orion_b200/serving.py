"""Request loop: many device-resident cases in flight at once (continuous batching).

Requests (bump cases of different grid sizes and flow conditions) arrive over
time.  The loop admits a queued request as soon as a slot and enough HBM are
free (admission by the case's device footprint, orion_footprint_estimate),
builds its case (grid, metrics, initial state) on an admission thread while
the GPU keeps running the admitted cases, and steps every admitted case on its
own CUDA stream in quanta of graph-captured steps (orion_step_submit), so the
work of all resident cases overlaps on the device.  With batched=True every
resident case is stepped in one group instead, one launch per stage over the
blocks of all of them (orion_group_*), rebuilt between quanta when cases join
or retire.  Streams are the default: on the C4 request mix they served about
1.4x the group's throughput, because one case's line kernels overlap other
cases' sweep chains, while a group's stages run one after another and its
sweep chain is as long as its largest member's.  A case retires at the end
of the first quantum in which its residual has dropped to `drop` times its
first-step residual (rms, ResidualMonitor::compute), or after max_steps, or
as diverged when its residual stops being finite or grows past diverge_growth
(1e3) times the first step's; its memory is freed in stream order and the
next request takes its place.

Every case keeps its own work lists and reductions and runs the same
deterministic kernels whatever else is resident (alone, on its own stream, or
in a group), and the quanta are the same, so a request's result does not
depend on the mix it ran in.  A case steps whole quanta: max_steps should be a
multiple of the quantum.

    python -m orion_b200.serving --requests 256 --mean-ms 50 --max-steps 2000
"""
from __future__ import annotations

import os

# Every resident case runs on its own stream.  CUDA maps streams onto a few
# hardware work queues (8 by default), which serialises independent cases;
# 32 queues (the maximum) let them overlap.  Read when the CUDA context is
# made, so it only takes effect if this module is imported first.
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

import argparse
import concurrent.futures as cf
import json
import math
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Callable, Dict, List, Optional

import numpy as np

from . import _lib, cases

DIMS = (33, 49, 65, 97, 129)


@dataclass
class Request:
    """A bump case to solve, built on admission (its arrays are not held while queued)."""
    rid: int
    arrival_s: float
    dims: tuple
    nblocks: int
    height: float
    moo: float
    reynolds: float
    noise_seed: int
    max_steps: int = 2000
    drop: float = 1e-6

    def split(self) -> tuple:
        """1-D split along the longest axis (2-D and 3-D splits of the reference's
        interface scheme do not converge: corner ghosts are never exchanged)."""
        ax = int(np.argmax(self.dims))
        parts = max(1, min(self.nblocks, (self.dims[ax] - 1) // (cases.MIN_BLOCK_DIM - 1)))
        sp = [1, 1, 1]
        sp[ax] = parts
        return tuple(sp)

    def build_case(self) -> cases.Case:
        return cases.bump_case(f"req{self.rid}", *self.dims, height=self.height, split=self.split(),
                               moo=self.moo, reynolds=self.reynolds, nsteps=self.max_steps,
                               noise_seed=self.noise_seed)

    @property
    def npoints(self) -> int:
        return int(np.prod(self.dims))


def c4_requests(n: int = 256, seed: int = 4, mean_ms: float = 50.0, max_steps: int = 2000, drop: float = 1e-6,
                dims=DIMS) -> List[Request]:
    """Seeded request stream: Poisson arrivals (mean inter-arrival mean_ms), per-axis
    points from `dims`, 1-8 blocks, bump height U[0.02,0.08], Mach U[0.2,0.85],
    Re log-uniform in [1e3,1e5]."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += float(rng.exponential(mean_ms / 1e3))
        d = tuple(int(x) for x in rng.choice(dims, 3))
        out.append(Request(rid=i, arrival_s=t, dims=d, nblocks=int(rng.integers(1, 9)),
                           height=float(rng.uniform(0.02, 0.08)), moo=float(rng.uniform(0.2, 0.85)),
                           reynolds=float(10.0 ** rng.uniform(3.0, 5.0)), noise_seed=seed * 100003 + i,
                           max_steps=max_steps, drop=drop))
    return out


@dataclass
class Result:
    rid: int
    npoints: int
    nblocks: int
    status: str            # converged | max_steps | diverged | rejected
    steps: int             # steps executed
    steps_to_drop: int     # first step meeting the criterion (0: never)
    arrival_s: float
    admit_s: float
    done_s: float
    rms_first: float
    rms_last: float
    state: Optional[List[np.ndarray]] = None  # interior prim per block (keep_state)

    @property
    def latency_s(self) -> float:
        return self.done_s - self.arrival_s


@dataclass
class _Slot:
    req: Request
    fs: object
    footprint: int
    admit_s: float
    hist: List[np.ndarray] = field(default_factory=list)
    steps: int = 0


class Server:
    """The request loop.  precision: _lib.PREC_MIXED (default) or PREC_FP64."""

    def __init__(self, precision: int = _lib.PREC_MIXED, device: int = 0, hbm_budget: Optional[int] = None,
                 max_active: int = 256, quantum: int = 20, keep_state: bool = False, builders: int = 4,
                 diverge_growth: float = 1e3, clock: Callable[[], float] = time.perf_counter,
                 batched: bool = False):
        self.batched = batched
        self.precision = precision
        self.device = device
        self.max_active = max_active
        self.quantum = quantum
        self.keep_state = keep_state
        self.builders = max(1, builders)
        self.diverge_growth = diverge_growth
        self.clock = clock
        if hbm_budget is None:
            import torch

            free, _total = torch.cuda.mem_get_info(device)
            hbm_budget = int(free * 0.85)
        self.hbm_budget = int(hbm_budget)
        self.peak_resident = 0
        self.peak_bytes = 0

    # -- pieces that tests replace -------------------------------------------------
    def footprint(self, req: Request) -> int:
        return _footprint_dims(req, self.precision)

    def make_case(self, req: Request):
        from . import solver

        return solver.FlowFieldSet(req.build_case(), precision=self.precision, device=self.device)

    def make_group(self, members: List[object]):
        from . import solver

        return solver.CaseGroup(members)

    # -- the loop ----------------------------------------------------------------------
    def run(self, requests: List[Request]) -> List[Result]:
        if self.batched:
            return self._run_batched(requests)
        return self._run_streams(requests)

    def _run_batched(self, requests: List[Request]) -> List[Result]:
        """Every resident case in one group: one launch per stage for all of
        them, `quantum` steps per round.  Between rounds the finished cases
        retire, the cases built meanwhile join, and the group is rebuilt when
        its membership changed."""
        pending = deque(sorted(requests, key=lambda r: r.arrival_s))
        queue: deque = deque()
        active: Dict[int, _Slot] = {}
        results: List[Result] = []
        used = 0
        building: List[tuple] = []  # (future, request, footprint), oldest first
        ready: List[tuple] = []     # built cases waiting for the next round
        group = None
        running = False
        hs: Dict[int, np.ndarray] = {}
        pool = cf.ThreadPoolExecutor(max_workers=self.builders)
        t0 = self.clock()
        try:
            while pending or queue or active or building or ready:
                now = self.clock() - t0
                while pending and pending[0].arrival_s <= now:
                    queue.append(pending.popleft())
                while queue and len(building) < self.builders and \
                        len(active) + len(building) + len(ready) < self.max_active:
                    req = queue[0]
                    fp = self.footprint(req)
                    if fp > self.hbm_budget:
                        queue.popleft()
                        results.append(Result(req.rid, req.npoints, req.nblocks, "rejected", 0, 0, req.arrival_s,
                                              now, now, math.nan, math.nan))
                        continue
                    if used + fp > self.hbm_budget:
                        break
                    queue.popleft()
                    used += fp
                    building.append((pool.submit(self.make_case, req), req, fp))
                while building and building[0][0].done():  # in admission order
                    fut, req, fp = building.pop(0)
                    ready.append((fut.result(), req, fp))
                if running:
                    for rid, slot in active.items():  # the group's stream: all finish together
                        if rid not in hs:
                            h = slot.fs.poll()
                            if h is None:
                                break
                            hs[rid] = h
                    if len(hs) < len(active):
                        time.sleep(2e-4)
                        continue
                    running = False
                    retired = []
                    for rid, h in hs.items():
                        slot = active[rid]
                        slot.hist.append(h)
                        slot.steps += len(h)
                        res = self._retire_check(slot, self.clock() - t0)
                        if res is not None:
                            retired.append((rid, res))
                    if retired or ready:
                        if group is not None:
                            group.close()
                            group = None
                        for rid, res in retired:
                            slot = active.pop(rid)
                            if self.keep_state:
                                res.state = [slot.fs.download(b, "prim")[:5, 3:-3, 3:-3, 3:-3].copy()
                                             for b in range(len(slot.fs.case.blocks))]
                            slot.fs.close()
                            used -= slot.footprint
                            results.append(res)
                if not running:
                    if ready:
                        if group is not None:
                            group.close()
                            group = None
                        for fs, req, fp in ready:
                            active[req.rid] = _Slot(req, fs, fp, self.clock() - t0)
                        ready = []
                        self.peak_resident = max(self.peak_resident, len(active))
                        self.peak_bytes = max(self.peak_bytes, used)
                    if active:
                        if group is None:
                            group = self.make_group([slot.fs for slot in active.values()])
                        group.submit(self.quantum)
                        running = True
                        hs = {}  # this round's histories, per member
                    else:
                        time.sleep(2e-4)
        finally:
            pool.shutdown(wait=True)
            if group is not None:
                group.close()
            for slot in active.values():
                slot.fs.close()
            for fs, _req, _fp in ready:
                fs.close()
        return sorted(results, key=lambda r: r.rid)

    def _run_streams(self, requests: List[Request]) -> List[Result]:
        pending = deque(sorted(requests, key=lambda r: r.arrival_s))
        queue: deque = deque()
        active: Dict[int, _Slot] = {}
        results: List[Result] = []
        used = 0
        building: List[tuple] = []  # (future, request, footprint), oldest first
        pool = cf.ThreadPoolExecutor(max_workers=self.builders)
        t0 = self.clock()
        try:
            while pending or queue or active or building:
                now = self.clock() - t0
                while pending and pending[0].arrival_s <= now:
                    queue.append(pending.popleft())
                # admission: first come first served, up to `builders` cases being built
                while queue and len(building) < self.builders and len(active) + len(building) < self.max_active:
                    req = queue[0]
                    fp = self.footprint(req)
                    if fp > self.hbm_budget:
                        queue.popleft()
                        results.append(Result(req.rid, req.npoints, req.nblocks, "rejected", 0, 0, req.arrival_s,
                                              now, now, math.nan, math.nan))
                        continue
                    if used + fp > self.hbm_budget:
                        break
                    queue.popleft()
                    used += fp
                    building.append((pool.submit(self.make_case, req), req, fp))
                while building and building[0][0].done():  # in admission order
                    fut, req, fp = building.pop(0)
                    fs = fut.result()
                    slot = _Slot(req, fs, fp, self.clock() - t0)
                    fs.submit(min(self.quantum, req.max_steps))
                    active[req.rid] = slot
                    self.peak_resident = max(self.peak_resident, len(active))
                    self.peak_bytes = max(self.peak_bytes, used)
                progressed = False
                for rid in list(active):
                    slot = active[rid]
                    h = slot.fs.poll()
                    if h is None:
                        continue
                    progressed = True
                    slot.hist.append(h)
                    slot.steps += len(h)
                    res = self._retire_check(slot, self.clock() - t0)
                    if res is None:
                        slot.fs.submit(min(self.quantum, slot.req.max_steps - slot.steps))
                        continue
                    if self.keep_state:
                        res.state = [slot.fs.download(b, "prim")[:5, 3:-3, 3:-3, 3:-3].copy()
                                     for b in range(len(slot.fs.case.blocks))]
                    slot.fs.close()
                    used -= slot.footprint
                    del active[rid]
                    results.append(res)
                if not progressed:
                    time.sleep(2e-4)
        finally:
            pool.shutdown(wait=True)
            for slot in active.values():
                slot.fs.close()
        return sorted(results, key=lambda r: r.rid)

    def _retire_check(self, slot: _Slot, now: float) -> Optional[Result]:
        hist = np.concatenate(slot.hist, axis=0)
        rms = hist[:, 0]
        rms1 = rms[0]
        req = slot.req
        status = None
        hit = np.nonzero(rms <= req.drop * rms1)[0]
        if not np.all(np.isfinite(rms)) or np.any(rms > self.diverge_growth * rms1):
            status = "diverged"
        elif hit.size:
            status = "converged"
        elif slot.steps >= req.max_steps:
            status = "max_steps"
        if status is None:
            return None
        return Result(req.rid, req.npoints, req.nblocks, status, slot.steps, int(hit[0]) + 1 if hit.size else 0,
                      req.arrival_s, slot.admit_s, now, float(rms1), float(rms[-1]))


def _footprint_dims(req: Request, precision: int) -> int:
    """Device bytes of the request's case from its block dims alone (no grid arrays)."""
    import ctypes as C

    pts = [cases.even_splits(n, p) for n, p in zip(req.dims, req.split())]
    ext = [[b - a + 1 for a, b in zip(sp[:-1], sp[1:])] for sp in pts]  # shared planes
    descs = []
    for kd in ext[2]:
        for jd in ext[1]:
            for idm in ext[0]:
                d = _lib.BlockDesc()
                d.idim, d.jdim, d.kdim = idm, jd, kd
                d.nregions = 0
                d.regions = None
                descs.append(d)
    arr = (_lib.BlockDesc * len(descs))(*descs)
    return int(_lib.load().orion_footprint_estimate(len(descs), arr, precision))


def summarize(results: List[Result]) -> dict:
    done = [r for r in results if r.status != "rejected"]
    lat = np.array([r.latency_s for r in done]) * 1e3
    work = sum(r.npoints * r.steps for r in done)
    t_end = max((r.done_s for r in done), default=0.0)
    t_start = min((r.arrival_s for r in done), default=0.0)
    span = max(t_end - t_start, 1e-9)
    counts = {}
    for r in results:
        counts[r.status] = counts.get(r.status, 0) + 1
    return {
        "requests": len(results),
        "status": counts,
        "p50_ms": float(np.percentile(lat, 50)) if lat.size else None,
        "p99_ms": float(np.percentile(lat, 99)) if lat.size else None,
        "mean_ms": float(lat.mean()) if lat.size else None,
        "cell_updates": int(work),
        "makespan_s": span,
        "cell_updates_per_s": work / span,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=256)
    ap.add_argument("--mean-ms", type=float, default=50.0)
    ap.add_argument("--max-steps", type=int, default=2000)
    ap.add_argument("--drop", type=float, default=1e-6)
    ap.add_argument("--seed", type=int, default=4)
    ap.add_argument("--quantum", type=int, default=20)
    ap.add_argument("--max-active", type=int, default=256)
    ap.add_argument("--baseline", action="store_true", help="also serve one at a time on the plain FP64 path")
    ap.add_argument("--group", action="store_true", help="step every resident case in one group (orion_group_*)")
    a = ap.parse_args()
    reqs = c4_requests(a.requests, a.seed, a.mean_ms, a.max_steps, a.drop)
    out = {"config": vars(a)}
    srv = Server(_lib.PREC_MIXED, quantum=a.quantum, max_active=a.max_active, batched=a.group)
    out["mixed_continuous"] = summarize(srv.run(reqs))
    out["mixed_continuous"]["peak_resident_cases"] = srv.peak_resident
    if a.baseline:
        seq = Server(_lib.PREC_FP64, quantum=a.quantum, max_active=1)
        out["plain_one_at_a_time"] = summarize(seq.run(reqs))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
