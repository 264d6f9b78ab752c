"""Failure detection on the GPU without a fault: the bounded barrier wait.

The cooperative-grid form of the LU-SGS/GS sweeps separates hyperplanes with a
software grid barrier whose wait is bounded (ORION_SWEEP_SPIN_LIMIT polls,
read when a case is made).  With a limit of one poll the first CTA to arrive
gives up at once: the kernel records the error and every CTA returns, the host
reports ORION_E_TIMEOUT, and the context stays usable for the next case.
"""
import os

import numpy as np
import pytest

from orion_b200 import _lib, cases, solver
from orion_b200._lib import OrionError

pytestmark = pytest.mark.gpu


def test_grid_barrier_timeout_is_reported_and_the_context_survives():
    case = cases.small_case("timeout", dims=(33, 25, 23), noise_seed=5)
    os.environ["ORION_SWEEP_SPIN_LIMIT"] = "1"
    try:
        fs = solver.FlowFieldSet(case, precision=_lib.PREC_FP64)
    finally:
        del os.environ["ORION_SWEEP_SPIN_LIMIT"]
    fs.set_schedule("grid", 0, 32)
    with pytest.raises(OrionError) as err:
        fs.step(1)
    assert "-6" in str(err.value) and "gave up waiting" in str(err.value)
    fs.close()
    # a new case on the same context runs and matches a fresh reference run
    a = solver.FlowFieldSet(case, precision=_lib.PREC_FP64)
    b = solver.FlowFieldSet(case, precision=_lib.PREC_FP64)
    a.set_schedule("grid", 0, 32)
    assert np.array_equal(a.step(3), b.step(3))
    a.close()
    b.close()


def test_tile_wavefront_wait_timeout_is_reported_and_the_context_survives():
    """The tile wavefront's waits on its upstream tiles are bounded too: with a
    limit of one poll a tile that finds its upstream tile behind gives up, the
    error word stops every other waiting tile, and the host reports
    ORION_E_TIMEOUT.  The case is made of blocks wide enough in j and k to hold
    several tiles each, so that tiles do wait on one another."""
    case = cases.small_case("timeout_tiles", dims=(33, 70, 25), split=(1, 1, 1), noise_seed=5)
    os.environ["ORION_SWEEP_SPIN_LIMIT"] = "1"
    try:
        fs = solver.FlowFieldSet(case, precision=_lib.PREC_FP64)
    finally:
        del os.environ["ORION_SWEEP_SPIN_LIMIT"]
    fs.set_schedule("tiles", 0, 32)
    with pytest.raises(OrionError) as err:
        fs.step(1)
    assert "-6" in str(err.value)
    fs.close()
    a = solver.FlowFieldSet(case, precision=_lib.PREC_FP64)
    b = solver.FlowFieldSet(case, precision=_lib.PREC_FP64)
    b.set_schedule("planes", 0, 32)
    assert np.array_equal(a.step(3), b.step(3))
    a.close()
    b.close()
