"""Pipelined host I/O (orion_io_put / orion_io_step / orion_io_get /
orion_io_wait): a stream of independent states through one case, with the
copies on their own streams overlapping the steps.  Each io step's result and
residual history must be bit-identical to the blocking upload, step, download
of the same input (the reference's host-array driver loop,
src/core/OrionSolver.cpp:139-209), in both precisions, with the puts of the
next input issued before the previous results are read back."""
import numpy as np
import pytest
import torch

from orion_b200 import _lib, cases, solver
from orion_b200._lib import OrionError

pytestmark = pytest.mark.gpu

SPEC = dict(name="io", dims=(41, 27, 25), split=(3, 2, 2), noise_seed=41, uneven_seed=4, moo=0.8, reynolds=1e5,
            height=0.08)


def _states(precision, n):
    """n distinct valid states: the case after 1, 2, ... n steps."""
    fs = solver.FlowFieldSet(cases.small_case(**SPEC), precision=precision)
    out = []
    for _ in range(n):
        fs.step(1)
        out.append([fs.download(b, "prim").copy() for b in range(len(fs.case.blocks))])
    fs.close()
    return out


@pytest.mark.parametrize("precision", [_lib.PREC_FP64, _lib.PREC_MIXED], ids=["plain", "mixed"])
def test_pipelined_io_matches_blocking_copies(precision):
    nin, nsteps = 4, 2
    states = _states(precision, nin)
    # blocking: upload, step, download, one input after another
    fs = solver.FlowFieldSet(cases.small_case(**SPEC), precision=precision)
    want, want_h = [], []
    for st in states:
        for b, a in enumerate(st):
            fs.upload(b, "prim", a)
        want_h.append(fs.step(nsteps))
        want.append([fs.download(b, "prim") for b in range(len(st))])
    fs.close()
    # pipelined: every put and get enqueued before any wait, pinned buffers
    fs = solver.FlowFieldSet(cases.small_case(**SPEC), precision=precision)
    ins = [[torch.from_numpy(a.reshape(-1)).pin_memory() for a in st] for st in states]
    outs = [[torch.empty_like(t).pin_memory() for t in st] for st in ins]
    for k in range(nin):
        for b, t in enumerate(ins[k]):
            fs.io_put(b, t)
        fs.io_step(nsteps)
        for b, t in enumerate(outs[k]):
            fs.io_get(b, t)
    fs.io_wait()
    hist = fs.poll()
    fs.close()
    assert np.array_equal(hist, np.concatenate(want_h))
    for k in range(nin):
        for b in range(len(states[k])):
            assert np.array_equal(outs[k][b].numpy(), want[k][b].reshape(-1)), f"input {k} block {b}"


def test_io_needs_a_step_before_a_get_and_refuses_grouped_cases():
    fs = solver.FlowFieldSet(cases.small_case(**SPEC), precision=_lib.PREC_MIXED)
    buf = np.zeros(6 * int(np.prod(fs.case.blocks[0].padded)))
    with pytest.raises(OrionError):
        fs.io_get(0, buf)
    other = solver.FlowFieldSet(cases.small_case(**SPEC), precision=_lib.PREC_MIXED)
    g = solver.CaseGroup([other])
    with pytest.raises(OrionError):
        other.io_put(0, buf)
    g.close()
    other.close()
    fs.close()


def test_partial_puts_install_only_the_blocks_put():
    """Blocks put in scattered runs (0, 2-3, 5 of 12) are installed; the others keep
    the state the previous io step left, as with blocking uploads of those blocks."""
    precision = _lib.PREC_MIXED
    states = _states(precision, 2)
    put_blocks = [0, 2, 3, 5]
    fs = solver.FlowFieldSet(cases.small_case(**SPEC), precision=precision)
    for b, a in enumerate(states[0]):
        fs.upload(b, "prim", a)
    fs.step(1)
    for b in put_blocks:
        fs.upload(b, "prim", states[1][b])
    want_h = fs.step(2)
    want = [fs.download(b, "prim") for b in range(len(states[0]))]
    fs.close()
    fs = solver.FlowFieldSet(cases.small_case(**SPEC), precision=precision)
    ins0 = [torch.from_numpy(a.reshape(-1)).pin_memory() for a in states[0]]
    ins1 = {b: torch.from_numpy(states[1][b].reshape(-1)).pin_memory() for b in put_blocks}
    outs = [torch.empty_like(t).pin_memory() for t in ins0]
    for b, t in enumerate(ins0):
        fs.io_put(b, t)
    fs.io_step(1)
    for b in put_blocks:
        fs.io_put(b, ins1[b])
    fs.io_step(2)
    for b, t in enumerate(outs):
        fs.io_get(b, t)
    fs.io_wait()
    hist = fs.poll()
    fs.close()
    assert np.array_equal(hist[1:], want_h)
    for b in range(len(states[0])):
        assert np.array_equal(outs[b].numpy(), want[b].reshape(-1)), f"block {b}"
