"""The mixed-precision path against the plain FP64 path (the FP64 oracle).

The mixed path keeps prim, metrics, vol, the Q update and the residual norm in
FP64 and runs fluxes, viscous terms, time step and LU-SGS/GS increments in
FP32.  Tolerance: relative L2 of the interior primitive state <= 1e-6.

* On a converging single-block case the error stays below the tolerance for
  the whole run (it does not accumulate: the increments vanish as the case
  converges).
* On multi-block 2x2x2 splits the reference's own scheme stops converging
  after about 15 steps (corner ghosts where four blocks meet are never
  exchanged), so the comparison there is taken inside the first 10 steps.
"""
import numpy as np
import pytest

from orion_b200 import _lib, cases, solver

pytestmark = pytest.mark.gpu

TOL_L2 = 1e-6


def _rel_l2(case, fm, fp):
    num = den = 0.0
    for b in range(len(case.blocks)):
        m = fm.download(b, "prim")[:5, 3:-3, 3:-3, 3:-3]
        p = fp.download(b, "prim")[:5, 3:-3, 3:-3, 3:-3]
        num += float(np.sum((m - p) ** 2))
        den += float(np.sum(p ** 2))
    return (num / den) ** 0.5


def _pair(case):
    metrics = [solver.grid_metrics(b, case.params.gcl) for b in case.blocks]
    return (solver.FlowFieldSet(case, precision=_lib.PREC_MIXED, metrics=metrics),
            solver.FlowFieldSet(case, precision=_lib.PREC_FP64, metrics=metrics))


def test_mixed_tracks_fp64_on_converging_case():
    case = cases.small_case("mixed1", dims=(49, 33, 25), noise_seed=11)
    fm, fp = _pair(case)
    for nsteps in (10, 90):
        hm, hp = fm.step(nsteps), fp.step(nsteps)
        assert _rel_l2(case, fm, fp) <= TOL_L2
        assert np.all(np.abs(hm[:, 0] - hp[:, 0]) <= 1e-3 * hp[:, 0])
    assert hp[-1, 0] < hp[0, 0]  # the case converges
    fm.close()
    fp.close()


def test_mixed_tracks_fp64_on_uneven_multiblock_case():
    case = cases.small_case("mixed8", dims=(41, 27, 25), split=(3, 2, 2), noise_seed=9, uneven_seed=4,
                            moo=0.8, reynolds=1.0e5, height=0.08)
    fm, fp = _pair(case)
    fm.step(10)
    fp.step(10)
    assert _rel_l2(case, fm, fp) <= TOL_L2
    fm.close()
    fp.close()


@pytest.mark.parametrize("name,flow", [
    ("mixedbc", dict(twall=300.0, attack=3.0, physical={"imin": cases.BC_FREESTREAM, "imax": cases.BC_EXTRAPOLATION,
                                                         "kmax": cases.BC_EXTRAPOLATION})),
    ("mixedeuler", dict(nvis=0, method=0)),
])
def test_mixed_tracks_fp64_with_other_bcs_and_euler(name, flow):
    """Freestream / extrapolation faces, isothermal walls and attack; and the
    Euler path (slip walls, no viscous stage)."""
    case = cases.small_case(name, dims=(33, 25, 23), split=(2, 1, 1), noise_seed=12, **flow)
    fm, fp = _pair(case)
    fm.step(10)
    fp.step(10)
    assert _rel_l2(case, fm, fp) <= TOL_L2
    fm.close()
    fp.close()


def test_mixed_path_stores_increments_in_fp32():
    case = cases.small_case("mixedfp", dims=(25, 17, 13))
    fm, fp = _pair(case)
    assert fm.footprint() < fp.footprint()
    assert fm.download(0, "dq").dtype == np.float64  # downloads widen to the reference's type
    fm.close()
    fp.close()
