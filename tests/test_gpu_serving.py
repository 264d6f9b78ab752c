"""The request loop on the GPU: a request's result is the same alone and in a mix.

Four small requests of different sizes and flow conditions are served once
each on their own and once together (all resident at the same time): in one
group stepped with one launch per stage over all their blocks, or each on
its own stream with their steps overlapping on the device.  Tolerance: identical status and step
counts, and the final interior primitive state equal to 1e-12 relative (the
kernels are deterministic, so in practice bit for bit).
"""
import numpy as np
import pytest

from orion_b200 import _lib, serving

pytestmark = pytest.mark.gpu


def _requests():
    spec = [((33, 33, 33), 1, 0.5, 1e3), ((49, 33, 25), 2, 0.7, 1e4), ((65, 25, 25), 3, 0.3, 3e3),
            ((25, 49, 33), 1, 0.8, 1e5)]
    return [serving.Request(rid=i, arrival_s=0.0, dims=d, nblocks=nb, height=0.05, moo=m, reynolds=re,
                            noise_seed=100 + i, max_steps=60, drop=1e-2) for i, (d, nb, m, re) in enumerate(spec)]


@pytest.mark.parametrize("batched", [True, False], ids=["group", "streams"])
def test_results_are_the_same_alone_and_in_the_mix(batched):
    reqs = _requests()
    alone = {}
    for r in reqs:
        srv = serving.Server(_lib.PREC_MIXED, quantum=10, keep_state=True, batched=False)
        alone[r.rid] = srv.run([r])[0]
    srv = serving.Server(_lib.PREC_MIXED, quantum=10, keep_state=True, batched=batched)
    mixed = {r.rid: r for r in srv.run(reqs)}
    assert srv.peak_resident >= 2  # the requests really were resident together
    for rid, a in alone.items():
        m = mixed[rid]
        assert (a.status, a.steps, a.steps_to_drop) == (m.status, m.steps, m.steps_to_drop)
        assert a.status in ("converged", "max_steps")
        for sa, sm in zip(a.state, m.state):
            assert np.max(np.abs(sa - sm)) <= 1e-12 * np.max(np.abs(sa))


def test_summary_reports_latency_percentiles_and_throughput():
    srv = serving.Server(_lib.PREC_MIXED, quantum=10)
    res = srv.run(_requests())
    s = serving.summarize(res)
    assert s["requests"] == 4 and s["p50_ms"] > 0 and s["p99_ms"] >= s["p50_ms"]
    assert s["cell_updates_per_s"] > 0
