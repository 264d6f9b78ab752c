"""Block-sharded stepping on one GPU: every shard a device case of its own
blocks, the exchanges between shards done with each shard's gather/scatter
kernels over device buffers (LocalTransport), against the same case stepped
as one through the same per-stage entry points.  The state must be
bit-identical on every block (ghosts included), the residual maximum, its
location and phydtime identical, the rms equal up to the order of the
shards' sums.  No kernel waits on another shard: the host orders every
exchange.
"""
import numpy as np
import pytest

from orion_b200 import _lib, cases, shard, solver

pytestmark = pytest.mark.gpu


def _single(case, precision, steps):
    """The whole case through the same per-stage entry points a shard uses."""
    fs = solver.FlowFieldSet(case, precision=precision)
    halo = solver.HaloExchanger()
    hist = []
    for _ in range(steps):
        halo.exchange_bc(None, fs)
        solver.apply_physical_bc(None, fs)
        solver.StateUpdater.update_flow_states(fs)
        solver.TimeIntegrator.calculate_time_step(fs)
        solver.FluxComputer.compute_viscous_rhs(fs)
        if case.params.nvis == 1:
            halo.average_interface_residuals(None, fs)
        solver.InviscidFluxComputer.compute_inviscid_rhs(fs)
        halo.average_interface_residuals(None, fs)
        solver.StateUpdater.update_solution(fs)
        hist.append(solver.ResidualMonitor.compute(fs))
    prim = [fs.download(b, "prim") for b in range(len(case.blocks))]
    fs.close()
    return hist, prim


def _sharded(case, owner, precision, steps):
    shards = [shard.Shard(case, owner, r, precision=precision) for r in range(max(owner) + 1)]
    group = shard.ShardGroup(shards, shard.LocalTransport())
    stats = group.run(steps)
    prim = [None] * len(case.blocks)
    for s in shards:
        for g in s.global_ids:
            prim[g] = s.download(g, "prim")
    for s in shards:
        s.close()
    return stats, prim


def _check(hist, prim1, stats, prim):
    assert len(stats) == len(hist)
    for h, st in zip(hist, stats):
        assert st.max_residual == h.max_residual
        assert tuple(st.max_loc) == tuple(h.max_loc)
        assert st.phydtime == h.phydtime
        assert abs(st.rms_residual - h.rms_residual) <= 1e-12 * h.rms_residual
    for b, (a, c) in enumerate(zip(prim1, prim)):
        assert np.array_equal(a, c), f"block {b}"


@pytest.mark.parametrize("precision", [_lib.PREC_FP64, _lib.PREC_MIXED])
def test_shards_equal_single_case(precision):
    case = cases.small_case("sh", dims=(61, 45, 37), split=(3, 2, 2), uneven_seed=5, noise_seed=3)
    hist, prim1 = _single(case, precision, 3)
    nb = len(case.blocks)
    for owner in (shard.partition(case, 2), [b % 3 for b in range(nb)], [0] * (nb - 1) + [1]):
        stats, prim = _sharded(case, owner, precision, 3)
        _check(hist, prim1, stats, prim)


def test_four_shards_equal_single_case_full_size():
    case = cases.config(3)  # 385x257x129 in 64 uneven blocks
    hist, prim1 = _single(case, _lib.PREC_FP64, 2)
    stats, prim = _sharded(case, shard.partition(case, 4), _lib.PREC_FP64, 2)
    _check(hist, prim1, stats, prim)


def test_shard_refuses_whole_case_calls():
    case = cases.small_case("rf", dims=(41, 33, 25), split=(2, 1, 1))
    s = shard.Shard(case, [0, 1], 0)
    lib = _lib.load()
    with pytest.raises(_lib.OrionError):
        _lib.check(lib.orion_step_async(s.handle, 1))
    with pytest.raises(_lib.OrionError):
        _lib.check(lib.orion_average_interface_residuals(s.handle))
    r = _lib.Residual()
    with pytest.raises(_lib.OrionError):
        _lib.check(lib.orion_residual_compute(s.handle, r))
    assert s.global_ids == [0]
    send, recv = s.counts(shard.HALO, 1)
    assert send > 0 and recv > 0
    s.close()


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _dist_rank(rank, world, port, q):
    """One shard per process on the same GPU, exchanges staged through host
    memory over gloo: no kernel of one process waits for another's."""
    import datetime
    import os
    import sys

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import torch.distributed as dist

    from orion_b200 import _lib as L
    from orion_b200 import cases as cs
    from orion_b200 import shard as sh

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    case = cs.small_case("sh", dims=(61, 45, 37), split=(3, 2, 2), uneven_seed=5, noise_seed=3)
    s = sh.Shard(case, sh.partition(case, world), rank, precision=L.PREC_FP64)
    stats = sh.ShardGroup([s], sh.DistTransport(host_staging=True)).run(3)
    prim = {g: s.download(g, "prim") for g in s.global_ids}
    s.close()
    q.put((rank, [(t.rms_residual, t.max_residual, tuple(t.max_loc), t.phydtime) for t in stats], prim))
    dist.barrier()
    dist.destroy_process_group()


def test_one_shard_per_process_host_staged_equals_single_case():
    import torch.multiprocessing as mp

    case = cases.small_case("sh", dims=(61, 45, 37), split=(3, 2, 2), uneven_seed=5, noise_seed=3)
    hist, prim1 = _single(case, _lib.PREC_FP64, 3)
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dist_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    prim = [None] * len(case.blocks)
    for rank, stats, blocks in out:
        for (rms, mx, loc, dt), h in zip(stats, hist):
            assert mx == h.max_residual and loc == tuple(h.max_loc) and dt == h.phydtime
            assert abs(rms - h.rms_residual) <= 1e-12 * h.rms_residual
        for g, a in blocks.items():
            prim[g] = a
    for b, (a, c) in enumerate(zip(prim1, prim)):
        assert c is not None and np.array_equal(a, c), f"block {b}"
