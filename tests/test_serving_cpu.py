"""Host logic of the request loop (orion_b200.serving) with fake device cases.

The fake case runs `submit`ted steps instantly and reports a residual history
rms_k = r0 * decay**(k-1) (NaN from step `nan_at` on).  Checks: admission
never exceeds the HBM budget, requests are admitted first come first served,
a case retires at the end of the quantum in which its residual dropped to
`drop` x its first-step residual, at max_steps, or as diverged when it stops
being finite or grows past 1e3 x the first step's, and a request larger than
the whole budget is rejected.
"""
import math

import numpy as np
import pytest

from orion_b200 import serving

BATCHED = pytest.mark.parametrize("batched", [True, False], ids=["group", "streams"])


class FakeCase:
    def __init__(self, req, log, busy_polls=0):
        self.req = req
        self.log = log
        self.k = 0
        self.pending = 0
        self.closed = False
        self.busy_polls = busy_polls  # polls that find submitted steps still running
        self.busy = 0

    def submit(self, n):
        self.pending += n
        self.busy = self.busy_polls

    def poll(self, cap=4096):
        if not self.pending:
            return None
        if self.busy > 0:
            self.busy -= 1
            return None
        rows = []
        for _ in range(self.pending):
            self.k += 1
            r = self.req.decay ** (self.k - 1) if self.k < self.req.nan_at else math.nan
            rows.append([r, r, 0, 1, 1, 1, 1, 0.0])
        self.pending = 0
        return np.array(rows)

    def close(self):
        self.closed = True
        self.log.append(("close", self.req.rid))


class FakeGroup:
    """Steps its members together (orion_group_* on the device)."""

    def __init__(self, members, log):
        self.members = members
        self.log = log
        self.closed = False
        log.append(("group", tuple(m.req.rid for m in members)))

    def submit(self, n):
        assert not self.closed
        for m in self.members:
            assert not m.closed
            m.submit(n)

    def close(self):
        self.closed = True
        self.log.append(("ungroup", tuple(m.req.rid for m in self.members)))


class FakeServer(serving.Server):
    def __init__(self, sizes, **kw):
        self.sizes = sizes
        self.log = []
        self.group_log = []
        self.resident = 0
        self.max_resident_bytes = 0
        kw.setdefault("builders", 1)  # one builder: the admission log is in admission order
        self.busy_polls = kw.pop("busy_polls", 0)
        super().__init__(hbm_budget=kw.pop("hbm_budget"), clock=self._clock, **kw)
        self.t = 0.0

    def _clock(self):
        self.t = getattr(self, "t", 0.0) + 0.001  # 1 ms per look at the clock
        return self.t

    def footprint(self, req):
        return self.sizes[req.rid]

    def make_case(self, req):
        self.log.append(("admit", req.rid))
        return FakeCase(req, self.log, self.busy_polls)

    def make_group(self, members):
        return FakeGroup(members, self.group_log)


def _req(rid, arrival, decay=0.5, nan_at=10 ** 9, max_steps=100):
    r = serving.Request(rid=rid, arrival_s=arrival, dims=(33, 33, 33), nblocks=1, height=0.05, moo=0.5,
                        reynolds=1e3, noise_seed=rid, max_steps=max_steps, drop=1e-3)
    r.decay, r.nan_at = decay, nan_at
    return r


@BATCHED
def test_retirement_rules_and_quanta(batched):
    reqs = [_req(0, 0.0, decay=0.5),                 # 0.5**10 < 1e-3 at step 11
            _req(1, 0.0, decay=0.99, max_steps=30),  # never drops: stops at max_steps
            _req(2, 0.0, decay=0.9, nan_at=7),       # NaN at step 7
            _req(3, 0.0, decay=1.5)]                 # grows past 1e3 x the first step at step 19
    srv = FakeServer({0: 10, 1: 10, 2: 10, 3: 10}, hbm_budget=100, quantum=5, batched=batched)
    res = {r.rid: r for r in srv.run(reqs)}
    assert res[0].status == "converged" and res[0].steps_to_drop == 11 and res[0].steps == 15
    assert res[1].status == "max_steps" and res[1].steps == 30
    assert res[2].status == "diverged" and res[2].steps == 10
    assert res[3].status == "diverged" and res[3].steps == 20
    assert all(r.latency_s > 0 for r in res.values())


@BATCHED
def test_admission_respects_hbm_budget_and_arrival_order(batched):
    sizes = {0: 60, 1: 50, 2: 30, 3: 40}
    reqs = [_req(i, 0.001 * i, decay=0.5) for i in range(4)]
    srv = FakeServer(sizes, hbm_budget=100, quantum=4, batched=batched)
    res = srv.run(reqs)
    assert [r.status for r in res] == ["converged"] * 4
    admits = [rid for ev, rid in srv.log if ev == "admit"]
    assert admits == [0, 1, 2, 3]  # first come, first served
    # replay the log: resident bytes never above the budget
    used, peak = 0, 0
    for ev, rid in srv.log:
        used += sizes[rid] if ev == "admit" else -sizes[rid]
        peak = max(peak, used)
    assert peak <= 100
    assert srv.peak_bytes <= 100


@BATCHED
def test_parallel_builders_keep_the_budget(batched):
    sizes = {i: 20 + 10 * (i % 4) for i in range(12)}
    reqs = [_req(i, 0.0005 * i, decay=0.6) for i in range(12)]
    srv = FakeServer(sizes, hbm_budget=90, quantum=3, builders=3, batched=batched)
    res = srv.run(reqs)
    assert [r.status for r in res] == ["converged"] * 12
    assert srv.peak_bytes <= 90
    assert srv.peak_resident >= 2


@BATCHED
def test_request_larger_than_budget_is_rejected(batched):
    srv = FakeServer({0: 500, 1: 10}, hbm_budget=100, quantum=4, batched=batched)
    res = {r.rid: r for r in srv.run([_req(0, 0.0), _req(1, 0.0)])}
    assert res[0].status == "rejected"
    assert res[1].status == "converged"


def test_c4_request_stream_is_seeded_and_within_ranges():
    a = serving.c4_requests(64, seed=4)
    b = serving.c4_requests(64, seed=4)
    assert [(r.dims, r.arrival_s, r.moo) for r in a] == [(r.dims, r.arrival_s, r.moo) for r in b]
    gaps = np.diff([0.0] + [r.arrival_s for r in a])
    assert 0.02 < gaps.mean() < 0.1  # mean inter-arrival 50 ms
    for r in a:
        assert set(r.dims) <= set(serving.DIMS)
        assert 1 <= r.nblocks <= 8 and 0.2 <= r.moo <= 0.85 and 1e3 <= r.reynolds <= 1e5
        assert 0.02 <= r.height <= 0.08
        split = r.split()
        assert sorted(split)[:2] == [1, 1]  # one split axis at most
        assert serving._footprint_dims(r, 1) > 0


def test_batched_rounds_group_every_resident_case_and_close_before_retiring():
    """Cases that arrive while a group steps join at the next round; a group is
    closed before any of its cases is closed, and no case is in two groups."""
    reqs = [_req(0, 0.0, decay=0.8), _req(1, 0.0, decay=0.99, max_steps=400), _req(2, 0.02, decay=0.9)]
    srv = FakeServer({0: 10, 1: 10, 2: 10}, hbm_budget=100, quantum=5, batched=True, builders=3, busy_polls=30)
    res = {r.rid: r for r in srv.run(reqs)}
    assert res[0].status == "converged" and res[0].steps == 35  # 0.8**31 < 1e-3 at step 32
    assert res[1].status == "max_steps" and res[1].steps == 400
    groups = [m for ev, m in srv.group_log if ev == "group"]
    assert groups and all(len(set(g)) == len(g) for g in groups)
    assert any(len(g) >= 2 for g in groups)
    open_groups = 0
    for ev, _m in srv.group_log:
        open_groups += 1 if ev == "group" else -1
        assert 0 <= open_groups <= 1
    assert open_groups == 0
