"""Groups of cases: many cases stepped together, one launch per stage.

Cases of different sizes, splits (even and uneven) and flow conditions are
stepped alone and then together in one group (orion_group_*).  Every stage of
the group is one launch over the blocks of all members (the sweeps one launch
per hyperplane, or per pass in the tile form), each block reading its own
case's parameters; the residual and time-step reductions run per member in
the member's own order.  So each member's residual history and state must be
bit-identical to its run alone, in both precisions and both sweep forms.
"""
import numpy as np
import pytest

from orion_b200 import _lib, cases, solver

pytestmark = pytest.mark.gpu

SPECS = [
    dict(name="g0", dims=(33, 25, 23), split=(2, 1, 1), noise_seed=31, moo=0.5, reynolds=1e3),
    dict(name="g1", dims=(41, 27, 25), split=(3, 2, 2), noise_seed=32, uneven_seed=4, moo=0.8, reynolds=1e5,
         height=0.08),
    dict(name="g2", dims=(25, 33, 17), split=(1, 2, 1), noise_seed=33, moo=0.3, reynolds=3e3, attack=2.0),
]


def _state(fs):
    return [fs.download(b, "prim") for b in range(len(fs.case.blocks))]


@pytest.mark.parametrize("precision", [_lib.PREC_FP64, _lib.PREC_MIXED], ids=["plain", "mixed"])
@pytest.mark.parametrize("sweep", ["planes", "tiles"])
def test_members_step_exactly_as_alone(precision, sweep):
    nsteps = 6
    alone = []
    for sp in SPECS:
        fs = solver.FlowFieldSet(cases.small_case(**sp), precision=precision)
        fs.set_schedule(sweep, 0, 16)
        h = fs.step(nsteps)
        alone.append((h, _state(fs)))
        fs.close()
    members = []
    for sp in SPECS:
        fs = solver.FlowFieldSet(cases.small_case(**sp), precision=precision)
        fs.set_schedule(sweep, 0, 16)
        members.append(fs)
    g = solver.CaseGroup(members)
    hists = g.step(nsteps)
    g.close()
    for (h_a, st_a), h_g, fs in zip(alone, hists, members):
        assert np.array_equal(h_a, h_g)
        for a, b in zip(st_a, _state(fs)):
            assert np.array_equal(a, b)
        fs.close()


def test_one_launch_per_stage_for_all_members():
    """The group's step issues about as many launches as one member's (the
    stage launches do not multiply with the member count)."""
    members = [solver.FlowFieldSet(cases.small_case(**sp), precision=_lib.PREC_MIXED) for sp in SPECS]
    for fs in members:
        fs.set_schedule("tiles", 0, 16)
    one = members[1].step_launches()
    g = solver.CaseGroup(members)
    n = g.step_launches()
    g.close()
    for fs in members:
        fs.close()
    assert n <= one + 4, (n, one)


def test_submit_and_poll_continue_after_the_group():
    """Members keep their step counters and histories: steps in a group, then
    alone, give the same history as the same number of steps alone."""
    sp = SPECS[0]
    ref = solver.FlowFieldSet(cases.small_case(**sp), precision=_lib.PREC_FP64)
    h_ref = ref.step(8)
    ref.close()
    a = solver.FlowFieldSet(cases.small_case(**sp), precision=_lib.PREC_FP64)
    b = solver.FlowFieldSet(cases.small_case(**SPECS[2]), precision=_lib.PREC_FP64)
    g = solver.CaseGroup([a, b])
    g.submit(5)
    g.sync()
    h1 = a.poll()
    b.poll()
    g.close()
    h2 = a.step(3)
    assert np.array_equal(np.vstack([h1, h2]), h_ref)
    a.close()
    b.close()


@pytest.mark.parametrize("precision", [_lib.PREC_FP64, _lib.PREC_MIXED], ids=["plain", "mixed"])
def test_new_parameters_reach_a_grouped_member(precision):
    """orion_case_set_params on a member of a group: its next steps use the new
    gamma, viscosity switch and CFL (the block descriptors the group's sweeps
    read are refreshed), exactly as when the case steps alone."""
    import dataclasses

    def changed(p):
        return dataclasses.replace(p, gamma=1.3, cfl=0.5 * p.cfl)

    ref = []
    for sp in SPECS:
        fs = solver.FlowFieldSet(cases.small_case(**sp), precision=precision)
        h1 = fs.step(3)
        if sp["name"] == "g1":
            fs.set_params(changed(fs.params))
        h2 = fs.step(3)
        ref.append((np.concatenate([h1, h2]), _state(fs)))
        fs.close()
    members = [solver.FlowFieldSet(cases.small_case(**sp), precision=precision) for sp in SPECS]
    g = solver.CaseGroup(members)
    h1 = g.step(3)
    members[1].set_params(changed(members[1].params))
    h2 = g.step(3)
    g.close()
    for (h_a, st_a), a1, a2, fs in zip(ref, h1, h2, members):
        assert np.array_equal(h_a, np.concatenate([a1, a2]))
        for a, b in zip(st_a, _state(fs)):
            assert np.array_equal(a, b)
        fs.close()
