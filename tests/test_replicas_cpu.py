"""Multi-process host logic of the N-GPU bench on CPU (gloo, world size 2).

Each GPU runs its own replica of the case; the job time is the slowest rank's
time and the whole-job throughput is world x units per rank / that time.
"""
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    from orion_b200 import replicas

    r = replicas.from_env(backend="gloo", timeout_s=60)
    r.barrier()
    slowest = r.max_over_ranks(1.0 + rank)  # rank 1 is the slow replica
    q.put((rank, slowest, r.aggregate_rate(100.0, slowest), r.world))
    r.close()


def test_max_over_ranks_and_aggregate_rate_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, rate, w in out:
        assert w == world
        assert slowest == 2.0  # every rank sees the slowest replica's time
        assert rate == world * 100.0 / 2.0


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    from orion_b200 import replicas

    env = {k: os.environ.pop(k) for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK") if k in os.environ}
    try:
        r = replicas.from_env()
        assert r.world == 1 and r.dist is None
        assert r.max_over_ranks(3.5) == 3.5
        assert r.aggregate_rate(10.0, 2.0) == 5.0
    finally:
        os.environ.update(env)


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
