"""Step schedules and the autotuner.

Every schedule (sweep form: tile wavefront, per-hyperplane launches,
cooperative grid, clusters of 8 or 16 CTAs; 8/16/32 grid lines per CTA in the
line kernels)
keeps the reference's Gauss-Seidel order and the per-point arithmetic, so on
the plain FP64 path the results are bit-identical whatever the schedule; on
the mixed path they agree within the mixed tolerance (1e-6 relative L2).
Autotuning times the candidates and leaves the solution where it was.
"""
import numpy as np
import pytest

from orion_b200 import _lib, cases, solver

pytestmark = pytest.mark.gpu

SCHEDULES = [("planes", 0, 32), ("tiles", 0, 16), ("grid", 0, 8), ("cluster", 16, 16), ("cluster", 8, 32)]


def _case():
    return cases.small_case("tune", dims=(41, 27, 25), split=(3, 2, 2), noise_seed=9, uneven_seed=4, moo=0.8,
                            reynolds=1.0e5, height=0.08)


def _state(fs):
    return [fs.download(b, "prim") for b in range(len(fs.case.blocks))]


def test_plain_results_do_not_depend_on_the_schedule():
    case = _case()
    ref = None
    for sweep, cs, lanes in SCHEDULES:
        fs = solver.FlowFieldSet(case, precision=_lib.PREC_FP64)
        fs.set_schedule(sweep, cs, lanes)
        assert fs.get_schedule() == {"sweep": sweep, "cluster_size": cs if sweep == "cluster" else 0, "lanes": lanes}
        h = fs.step(4)
        st = _state(fs)
        fs.close()
        if ref is None:
            ref = (h, st)
            continue
        assert np.array_equal(h, ref[0])
        assert all(np.array_equal(a, b) for a, b in zip(st, ref[1]))


def test_mixed_results_agree_across_schedules():
    case = _case()
    states = []
    for sweep, cs, lanes in SCHEDULES:
        fs = solver.FlowFieldSet(case, precision=_lib.PREC_MIXED)
        fs.set_schedule(sweep, cs, lanes)
        fs.step(4)
        states.append(_state(fs))
        fs.close()
    for st in states[1:]:
        num = sum(float(np.sum((a[:5, 3:-3, 3:-3, 3:-3] - b[:5, 3:-3, 3:-3, 3:-3]) ** 2)) for a, b in zip(st, states[0]))
        den = sum(float(np.sum(b[:5, 3:-3, 3:-3, 3:-3] ** 2)) for b in states[0])
        assert (num / den) ** 0.5 <= 1e-6


def test_autotune_keeps_the_solution_and_picks_a_timed_schedule():
    case = _case()
    a = solver.FlowFieldSet(case, precision=_lib.PREC_FP64)
    b = solver.FlowFieldSet(case, precision=_lib.PREC_FP64)
    ha1, hb1 = a.step(3), b.step(3)
    rep = a.autotune(steps_per_trial=2)
    assert len(rep["trials"]) >= 4
    assert rep["best"]["ms_per_step"] == min(t["ms_per_step"] for t in rep["trials"])
    assert a.get_schedule() == {k: rep["best"][k] for k in ("sweep", "cluster_size", "lanes")}
    ha2, hb2 = a.step(3), b.step(3)  # continues exactly as the untuned case
    assert np.array_equal(np.vstack([ha1, ha2]), np.vstack([hb1, hb2]))
    assert all(np.array_equal(x, y) for x, y in zip(_state(a), _state(b)))
    a.close()
    b.close()
