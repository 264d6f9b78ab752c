"""Grid metrics on the device (orion_case_grid_metrics) against the host
restatement (orion_grid_metrics_host), which the CPU tests pin to the
reference's compute_grid_metrics: bit-identical, both the cross-product form
and the Visbal conservative form (gcl=1), on uneven and minimum-size blocks."""
import numpy as np
import pytest

from orion_b200 import _lib, cases, solver

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("gcl", [0, 1])
@pytest.mark.parametrize("dims,split", [((41, 27, 25), (3, 2, 2)), ((12, 12, 12), (1, 1, 1)),
                                        ((97, 49, 33), (1, 1, 1))])
def test_device_metrics_equal_host_metrics(gcl, dims, split):
    case = cases.bump_case("m", *dims, split=split, uneven_seed=5 if split != (1, 1, 1) else None, height=0.08)
    case.params.gcl = gcl
    fs = solver.FlowFieldSet(case, init=False)  # metrics computed on the device
    for b, blk in enumerate(case.blocks):
        met, vol = solver.grid_metrics(blk, gcl)
        assert np.array_equal(fs.download(b, "metrics"), met)
        assert np.array_equal(fs.download(b, "vol"), vol)
    fs.close()


def test_device_metrics_give_the_same_run_as_host_metrics():
    case = cases.small_case("mrun", dims=(33, 25, 23), split=(2, 1, 1), noise_seed=3)
    host = [solver.grid_metrics(b, case.params.gcl) for b in case.blocks]
    a = solver.FlowFieldSet(case, precision=_lib.PREC_FP64)
    b = solver.FlowFieldSet(case, precision=_lib.PREC_FP64, metrics=host)
    assert np.array_equal(a.step(5), b.step(5))
    a.close()
    b.close()
