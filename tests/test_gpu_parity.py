"""GPU parity of the plain FP64 path against the reference.

* stage by stage: every per-stage entry point starts from the reference's
  snapshot before that stage and must reproduce the reference's snapshot after
  it (bit-identical except the far-field BC, whose std::pow may differ from the
  device pow by an ulp: tolerance 1e-13 relative there);
* whole runs: residual history and final state against the committed golden
  fixtures and, when oracle/_ref is present, against live reference runs of
  multi-block cases and of cases with freestream, extrapolation and
  isothermal-wall BCs and an Euler case, within 1e-10 relative.
"""
import json
import os

import numpy as np
import pytest

import refio
from orion_b200 import cases, solver
from parity import ROOT, STAGES, interior, rel_err, run_reference_case

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not refio.reference_available(), reason="oracle/_ref not built")

TOL_RUN = 1e-10


def _stage_ops(fs):
    return [
        ("exchange", lambda: solver.HaloExchanger().exchange_bc(None, fs), ["prim"], 0.0),
        ("bc", lambda: solver.apply_physical_bc(None, fs), ["prim"], 1e-13),
        ("state", lambda: solver.StateUpdater.update_flow_states(fs), ["prim", "c", "mu", "q", "dq"], 0.0),
        ("dt", lambda: solver.TimeIntegrator.calculate_time_step(fs), ["dt"], 0.0),
        ("visc", lambda: solver.FluxComputer.compute_viscous_rhs(fs), ["dq"], 0.0),
        ("avg1", lambda: solver.HaloExchanger().average_interface_residuals(None, fs), ["dq"], 0.0),
        ("inv", lambda: solver.InviscidFluxComputer.compute_inviscid_rhs(fs), ["dq"], 0.0),
        ("avg2", lambda: solver.HaloExchanger().average_interface_residuals(None, fs), ["dq"], 0.0),
        ("update", lambda: solver.StateUpdater.update_solution(fs), ["prim", "dq"], 0.0),
    ]


STAGE_CASES = {
    "single": dict(name="single", dims=(25, 17, 13), split=(1, 1, 1), noise_seed=7),
    "multi8": dict(name="multi8", dims=(33, 25, 23), split=(2, 2, 2), noise_seed=8),
    "uneven_transonic": dict(name="uneven", dims=(41, 27, 25), split=(3, 2, 2), noise_seed=9, uneven_seed=4,
                             moo=0.8, reynolds=1.0e5, height=0.08),
    # freestream and extrapolation faces, isothermal walls, flow at 3 degrees of attack
    "bc_mix": dict(name="bcmix", dims=(33, 25, 23), split=(2, 1, 1), noise_seed=10, twall=300.0, attack=3.0,
                   physical={"imin": cases.BC_FREESTREAM, "imax": cases.BC_EXTRAPOLATION,
                             "kmax": cases.BC_EXTRAPOLATION}),
    # Euler: slip walls, no viscous stage; method 0 (no wall-normal averaging)
    "inviscid_m0": dict(name="inviscid", dims=(33, 25, 23), split=(1, 2, 1), noise_seed=11, nvis=0, method=0),
}


@needs_ref
@pytest.mark.parametrize("key", list(STAGE_CASES))
def test_stage_parity(key, tmp_path):
    case = cases.small_case(nsteps=2, **STAGE_CASES[key])
    _, odir = run_reference_case(case, 2, snap_step=1, workdir=str(tmp_path))
    # without viscosity the reference runs neither the viscous stage nor its averaging
    skip = set() if case.params.nvis == 1 else {"visc", "avg1"}
    snaps = {s: refio.read_state(os.path.join(odir, f"snap_1_{s}.bin")) for s in STAGES if s not in skip}
    hist = refio.read_hist(os.path.join(odir, "hist.bin"))
    pre = snaps["pre"]
    fs = solver.FlowFieldSet(case, init=False, metrics=[(b["metrics"], b["vol"]) for b in pre["blocks"]])
    prev = "pre"
    for name, fn, fields, tol in _stage_ops(fs):
        if name in skip:
            continue
        fs.upload_state(snaps[prev])
        fn()
        fs.sync()
        for f in fields:
            for n, blk in enumerate(snaps[name]["blocks"]):
                g, r = fs.download(n, f), blk[f]
                if f == "dt":
                    g, r = interior(g), interior(r)
                e = rel_err(g, r)
                assert e <= tol, f"stage {name} field {f} block {n}: rel err {e:.3e}"
        if name == "dt":
            assert solver.TimeIntegrator.calculate_time_step(fs) == snaps["dt"]["phydtime"]
        prev = name
    fs.upload_state(snaps["update"])
    r = solver.ResidualMonitor.compute(fs)
    assert abs(r.rms_residual - hist[1, 0]) <= 1e-13 * hist[1, 0]
    assert r.max_residual == hist[1, 1]
    assert list(r.max_loc) == [int(v) for v in hist[1, 2:7]]
    fs.close()


@pytest.mark.parametrize("key", ["small_1blk", "small_8blk", "small_uneven", "small_bcmix", "small_euler"])
def test_whole_run_matches_golden(key):
    g = np.load(os.path.join(ROOT, "tests", "golden", key + ".npz"))
    case = cases.small_case(**json.loads(str(g["recipe"][0])))
    fs = solver.FlowFieldSet(case)
    hist = fs.step(case.nsteps)
    ref = g["hist"]
    for col in (0, 1, 7):
        e = np.max(np.abs(hist[:, col] - ref[:, col]) / np.abs(ref[:, col]))
        assert e <= TOL_RUN, (key, col, e)
    assert np.array_equal(hist[:, 2:7], ref[:, 2:7])
    sub = int(g["sub"][0])
    prim = np.concatenate([fs.download(b, "prim")[:5, 3:-3, 3:-3, 3:-3].reshape(5, -1)
                           for b in range(len(case.blocks))], axis=1)[:, ::sub]
    assert rel_err(prim, g["prim"]) <= TOL_RUN
    fs.close()


@needs_ref
@pytest.mark.parametrize("key", ["bc_mix", "inviscid_m0"])
def test_whole_run_matches_reference_other_bcs(key, tmp_path):
    """Five steps of the cases with the other BC types and flow options, against live reference runs."""
    case = cases.small_case(nsteps=5, **STAGE_CASES[key])
    _, odir = run_reference_case(case, 5, workdir=str(tmp_path))
    ref_hist = refio.read_hist(os.path.join(odir, "hist.bin"))
    ref = refio.read_state(os.path.join(odir, "final.bin"))
    fs = solver.FlowFieldSet(case)
    hist = fs.step(5)
    for col in (0, 1, 7):
        assert np.max(np.abs(hist[:, col] - ref_hist[:, col]) / np.abs(ref_hist[:, col])) <= TOL_RUN, col
    assert np.array_equal(hist[:, 2:7], ref_hist[:, 2:7])
    for n, blk in enumerate(ref["blocks"]):
        assert rel_err(interior(fs.download(n, "prim")[:5]), interior(blk["prim"][:5])) <= TOL_RUN
    fs.close()


@needs_ref
def test_config1_multiblock_run_matches_reference(tmp_path):
    """The 8-block 193x97x65 configuration, first 5 steps, against a live reference run."""
    case = cases.config(1, nsteps=5)
    _, odir = run_reference_case(case, 5, workdir=str(tmp_path))
    ref_hist = refio.read_hist(os.path.join(odir, "hist.bin"))
    ref = refio.read_state(os.path.join(odir, "final.bin"))
    fs = solver.FlowFieldSet(case)
    hist = fs.step(5)
    assert np.max(np.abs(hist[:, 0] - ref_hist[:, 0]) / ref_hist[:, 0]) <= TOL_RUN
    assert np.max(np.abs(hist[:, 1] - ref_hist[:, 1]) / ref_hist[:, 1]) <= TOL_RUN
    for n, blk in enumerate(ref["blocks"]):
        assert rel_err(interior(fs.download(n, "prim")[:5]), interior(blk["prim"][:5])) <= TOL_RUN
        q = fs.conservative(n)
        assert rel_err(interior(q), interior(solver.conservative_from_prim(blk["prim"], 1.4))) <= TOL_RUN
    fs.close()


def test_device_init_matches_host_restatement():
    case = cases.small_case("init", dims=(21, 17, 15), split=(1, 1, 1), noise_seed=99)
    fs = solver.FlowFieldSet(case)
    prim = solver.initial_prim(case)
    assert np.array_equal(fs.download(0, "prim"), prim[0])
    fs.close()


def test_graph_replay_is_deterministic():
    case = cases.small_case("det", dims=(25, 17, 13), split=(2, 1, 1), noise_seed=5)
    runs = []
    for _ in range(2):
        fs = solver.FlowFieldSet(case)
        hist = fs.step(4)
        runs.append((hist, [fs.download(b, "prim") for b in range(len(case.blocks))]))
        fs.close()
    assert np.array_equal(runs[0][0], runs[1][0])
    for a, b in zip(runs[0][1], runs[1][1]):
        assert np.array_equal(a, b)


def test_per_stage_sequence_equals_graph_step():
    """The reference-named per-stage entry points, called in the driver's order,
    give the same state as the captured step."""
    case = cases.small_case("seq", dims=(25, 17, 13), split=(2, 1, 1), noise_seed=6)
    a = solver.FlowFieldSet(case)
    ha = a.step(2)
    b = solver.FlowFieldSet(case)
    hx = solver.HaloExchanger()
    for _ in range(2):
        hx.exchange_bc(None, b)
        solver.apply_physical_bc(None, b)
        solver.StateUpdater.update_flow_states(b)
        solver.TimeIntegrator.calculate_time_step(b)
        solver.FluxComputer.compute_viscous_rhs(b)
        hx.average_interface_residuals(None, b)
        solver.InviscidFluxComputer.compute_inviscid_rhs(b)
        hx.average_interface_residuals(None, b)
        solver.StateUpdater.update_solution(b)
        r = solver.ResidualMonitor.compute(b)
    assert r.rms_residual == ha[-1, 0] and r.max_residual == ha[-1, 1]
    for n in range(len(case.blocks)):
        assert np.array_equal(a.download(n, "prim"), b.download(n, "prim"))
    a.close()
    b.close()
