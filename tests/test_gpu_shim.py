"""The reference's own driver on the B200 path, through the C++ drop-in layer.

oracle/_ref/orion_shim_harness is the oracle driver (the reference's set-up
code and the step loop of OrionSolver::solve) compiled against the
reference's headers and linked with orion_b200/shim/orion_backend_cuda.cpp in
place of src/solver/*.cpp and src/bc/PhysicalBC.cpp.  Run on the same case
files as the reference build, its residual history and final state must match
the reference within 1e-10 relative (plain FP64), in both residency modes.
"""
import os

import numpy as np
import pytest

import refio
from orion_b200 import cases
from parity import rel_err

pytestmark = pytest.mark.gpu
needs = pytest.mark.skipif(not (refio.reference_available() and refio.shim_available()),
                           reason="oracle/_ref harnesses not built")

TOL_RUN = 1e-10
CASES = {
    "multi8": dict(name="multi8", dims=(33, 25, 23), split=(2, 2, 2), noise_seed=8),
    "uneven_transonic": dict(name="uneven", dims=(41, 27, 25), split=(3, 2, 2), noise_seed=9, uneven_seed=4,
                             moo=0.8, reynolds=1.0e5, height=0.08),
    "bc_mix": dict(name="bcmix", dims=(33, 25, 23), split=(2, 1, 1), noise_seed=10, twall=300.0, attack=3.0,
                   physical={"imin": cases.BC_FREESTREAM, "imax": cases.BC_EXTRAPOLATION,
                             "kmax": cases.BC_EXTRAPOLATION}),
    "euler": dict(name="euler", dims=(33, 25, 23), split=(1, 2, 1), noise_seed=11, nvis=0, method=0),
}
NSTEPS = 5


def _runs(key, tmp_path, extra):
    case = cases.small_case(nsteps=NSTEPS, **CASES[key])
    cdir = str(tmp_path / "case")
    case.write_reference_inputs(cdir)
    refio.run_reference(cdir, NSTEPS, str(tmp_path / "ref"))
    out = refio.run_shim(cdir, NSTEPS, str(tmp_path / "shim"), extra)
    assert "CUDA backend initialized" in out
    return [(refio.read_hist(str(tmp_path / d / "hist.bin")), refio.read_state(str(tmp_path / d / "final.bin")))
            for d in ("ref", "shim")]


@needs
@pytest.mark.parametrize("key,mode", [("multi8", "coherent"), ("multi8", "resident"),
                                      ("uneven_transonic", "coherent"), ("bc_mix", "coherent"),
                                      ("euler", "resident")])
def test_reference_driver_on_device_matches_reference(key, mode, tmp_path):
    (href, sref), (hgpu, sgpu) = _runs(key, tmp_path, ["--resident"] if mode == "resident" else [])
    assert np.all(np.abs(hgpu[:, :2] - href[:, :2]) <= TOL_RUN * np.abs(href[:, :2]))
    assert np.array_equal(hgpu[:, 2:7], href[:, 2:7])
    assert np.all(np.abs(hgpu[:, 7] - href[:, 7]) <= TOL_RUN * np.abs(href[:, 7]))
    for f in ("prim", "q", "dq", "dt", "c", "mu"):
        err = max(rel_err(g[f], r[f]) for g, r in zip(sgpu["blocks"], sref["blocks"]))
        assert err <= TOL_RUN, (f, err)


@needs
def test_reference_driver_on_mixed_path_within_tolerance(tmp_path):
    (_, sref), (_, sgpu) = _runs("uneven_transonic", tmp_path, ["--resident", "--mixed"])
    num = sum(float(np.sum((g["prim"][:5] - r["prim"][:5])[:, 3:-3, 3:-3, 3:-3] ** 2))
              for g, r in zip(sgpu["blocks"], sref["blocks"]))
    den = sum(float(np.sum(r["prim"][:5, 3:-3, 3:-3, 3:-3] ** 2)) for r in sref["blocks"])
    assert (num / den) ** 0.5 <= 1e-6
