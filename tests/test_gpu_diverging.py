"""Requests of the serving stream that diverge diverge in the reference too.

tests/golden/c4_diverging.npz holds the reference's residual history over 200
steps of two requests of the seeded stream serving.c4_requests(24, seed=4):
request 1 (65x33x97 in 7 blocks, Mach 0.79, Re 9,001) and request 18
(129x49x49 in 3 blocks, Mach 0.79, Re 42,177), made by
tests/golden/gen_golden.py from the reference's own build.  Their residual
grows past 1e3 times the first step's in the reference, so the request loop's
"diverged" retirement of these flows is the reference's scheme at their
conditions, not this path's.  The plain path reproduces the first 20 steps to
1e-10 and diverges as well.
"""
import json
import os

import numpy as np
import pytest

from orion_b200 import _lib, serving, solver

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c4_diverging.npz")


def _fixture():
    g = np.load(GOLDEN)
    return g["hist"], json.loads(str(g["recipe"][0]))


def test_reference_history_of_the_diverging_requests_grows():
    hist, spec = _fixture()
    for h in hist:
        rms = h[:, 0]
        assert np.nanmax(rms) > 1e3 * rms[0] or not np.all(np.isfinite(rms))


@pytest.mark.gpu
def test_plain_path_follows_the_reference_and_diverges_too():
    hist, spec = _fixture()
    reqs = serving.c4_requests(spec["requests"], seed=spec["seed"], mean_ms=50.0, max_steps=spec["steps"])
    for rid, ref in zip(spec["rids"], hist):
        fs = solver.FlowFieldSet(reqs[rid].build_case(), precision=_lib.PREC_FP64)
        h = fs.step(spec["steps"])
        fs.close()
        rel = np.abs(h[:20, 0] - ref[:20, 0]) / np.abs(ref[:20, 0])
        assert np.all(rel <= 1e-10), f"request {rid}: rel {rel.max():.3e}"
        rms = h[:, 0]
        assert np.nanmax(rms) > 1e3 * rms[0] or not np.all(np.isfinite(rms))
