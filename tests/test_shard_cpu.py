"""Block sharding, host side (no GPU).

* The exchange plan (orion_b200/csrc/exchange_plan.hpp) compiled on the host:
  for several owner maps per case (fixed layouts, then seeded random splits
  and maps), exchange_bc and the interface averaging done shard by shard with
  explicit pack -> wire -> unpack equal, bit for bit on every block, the same
  exchanges done with the single-case lists (tests/shard/plan_check.cpp).
* The library's host-only plan counts agree between the two ends of every
  pair when each rank computes its own (gloo, world size 2).
* The residual reduction over ranks (gloo) equals the single-case reduction
  of the same partials: maximum with the smallest key among ties, key decoded
  to the global block and point.
* partition: contiguous runs, every shard non-empty, points balanced.
* DistTransport over gloo (world size 3, host buffers, stand-in shards):
  every rank's sends arrive at the right peer, complete and in order, for
  both exchanges and with the buffers reused.
"""
import os
import socket
import subprocess
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from orion_b200 import _lib, cases, shard

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def plan_check(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("plan") / "plan_check")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "orion_b200", "csrc"), "-I",
                    os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "shard", "plan_check.cpp"),
                    "-o", exe], check=True)
    return exe


def _describe(case, maps):
    out = [str(len(case.blocks))]
    for b in case.blocks:
        out.append(f"{b.idim} {b.jdim} {b.kdim} {len(b.regions)}")
        for g in b.regions:
            out.append(" ".join(str(v) for v in (*g.s_st, *g.s_ed, *g.t_st, *g.t_ed, g.bctype, g.nbt, g.ibcwin)))
    out.append(str(len(maps)))
    for m in maps:
        out.append(" ".join(str(v) for v in m))
    return "\n".join(out) + "\n"


def _maps(case, rng):
    nb = len(case.blocks)
    maps = [shard.partition(case, n) for n in (2, 3, min(4, nb)) if n <= nb]
    maps.append([b % 2 for b in range(nb)])                 # alternating blocks
    maps.append([int(v) for v in rng.integers(0, 3, nb)])    # random, possibly with holes
    maps.append([0] * (nb - 1) + [1])                        # one block alone
    # owner ids must cover 0..max: renumber the random map densely
    m = maps[-2]
    ids = {v: i for i, v in enumerate(sorted(set(m)))}
    maps[-2] = [ids[v] for v in m]
    return [m for m in maps if max(m) >= 1]


@pytest.mark.parametrize("name,dims,split,uneven", [
    ("even_2x2x1", (41, 33, 25), (2, 2, 1), None),
    ("even_2x2x2", (41, 33, 29), (2, 2, 2), None),
    ("uneven_3x2x2", (61, 45, 37), (3, 2, 2), 5),
    ("line_4x1x1", (97, 25, 17), (4, 1, 1), None),
])
def test_sharded_exchanges_equal_single_case(plan_check, name, dims, split, uneven):
    case = cases.small_case(name, dims=dims, split=split, uneven_seed=uneven)
    maps = _maps(case, np.random.default_rng(11))
    r = subprocess.run([plan_check], input=_describe(case, maps), capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = [ln for ln in r.stdout.splitlines() if "identical" in ln]
    assert len(lines) == len(maps)


def test_partition_contiguous_balanced():
    case = cases.config(2)  # 27 uneven blocks
    for n in (1, 2, 3, 4, 8, 27):
        o = shard.partition(case, n)
        assert o == sorted(o) and set(o) == set(range(n))
        pts = np.zeros(n)
        for b, s in zip(case.blocks, o):
            pts[s] += b.npoints
        if n <= 4:
            assert pts.max() / pts.mean() < 1.25
    with pytest.raises(_lib.OrionError):
        shard.partition(case, 28)


def test_single_shard_plan_sends_nothing():
    case = cases.small_case("one", dims=(41, 33, 25), split=(2, 2, 1))
    for kind in (shard.HALO, shard.IFACE):
        s, r = shard.plan_counts(case, [0] * len(case.blocks), 0, kind)
        assert s.tolist() == [0] and r.tolist() == [0]


def test_plan_rejects_bad_owner_lists():
    case = cases.small_case("bad", dims=(41, 33, 25), split=(2, 1, 1))
    with pytest.raises(_lib.OrionError):
        shard.plan_counts(case, [0, -1], 0, shard.HALO)
    with pytest.raises(_lib.OrionError):
        shard.plan_counts(case, [0, 1], 2, shard.HALO)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    from orion_b200 import cases as cs
    from orion_b200 import shard as sh

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    case = cs.small_case("g", dims=(61, 45, 37), split=(3, 2, 2), uneven_seed=5)
    owner = sh.partition(case, world)
    counts = {}
    for kind in (sh.HALO, sh.IFACE):
        s, r = sh.plan_counts(case, owner, rank, kind)
        t = torch.tensor(np.stack([s, r]), dtype=torch.int64)
        out = [torch.empty_like(t) for _ in range(world)]
        dist.all_gather(out, t)
        counts[kind] = [o.numpy().tolist() for o in out]
    # synthetic partials: rank 1 holds the largest residual, tied with rank 0 at a larger key
    parts = [(1.5, 0.25, 5 * 10 + 2, 0.02), (2.5, 0.25, 5 * 7 + 4, 0.01)]
    gathered = sh.gather_partials(parts[rank], dist)
    stats = sh.reduce_partials(gathered, case)
    q.put((rank, counts, gathered, stats))
    dist.barrier()
    dist.destroy_process_group()


def test_plan_counts_and_residual_reduction_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted((q.get(timeout=180) for _ in range(world)), key=lambda v: v[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, counts, gathered, stats in out:
        for kind, per_rank in counts.items():
            for a in range(world):
                for b in range(world):
                    # a sends to b exactly what b expects from a
                    assert per_rank[a][0][b] == per_rank[b][1][a]
            assert sum(per_rank[0][0]) > 0  # the split crosses the shards
        assert len(gathered) == world
        case = cases.small_case("g", dims=(61, 45, 37), split=(3, 2, 2), uneven_seed=5)
        npts = sum(b.npoints for b in case.blocks)
        assert stats.rms_residual == pytest.approx(np.sqrt(4.0 / (5 * npts)), rel=1e-15)
        assert stats.max_residual == 0.25
        b0 = case.blocks[0]
        assert stats.max_loc == (0, 7 % b0.idim + 1, (7 // b0.idim) % b0.jdim + 1, 7 // (b0.idim * b0.jdim) + 1, 5)
        assert stats.phydtime == 0.01


class _HostShard:
    """Stands in for a Shard on the host: exchange sizes from a formula, pack
    writes values naming sender, receiver, kind and position, unpack keeps
    what arrived."""

    def __init__(self, rank, nshards):
        self.rank, self.nshards, self.device = rank, nshards, 0
        self.got = {}

    @staticmethod
    def size(src, dst, kind):
        return 3 + 2 * src + dst + 4 * kind

    def counts(self, kind, peer):
        return self.size(self.rank, peer, kind), self.size(peer, self.rank, kind)

    @staticmethod
    def values(src, dst, kind):
        n = _HostShard.size(src, dst, kind)
        return 1000.0 * src + 100.0 * dst + 10.0 * kind + np.arange(n)

    def pack(self, kind, peer, ptr):
        import ctypes
        v = self.values(self.rank, peer, kind)
        ctypes.memmove(ptr, v.ctypes.data, v.nbytes)

    def unpack(self, kind, peer, ptr):
        import ctypes
        n = self.size(peer, self.rank, kind)
        a = np.empty(n)
        ctypes.memmove(a.ctypes.data, ptr, a.nbytes)
        self.got[(kind, peer)] = a

    def sync(self):
        pass


def _transport_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime

    import torch.distributed as dist

    from orion_b200 import shard as sh
    from test_shard_cpu import _HostShard

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    s = _HostShard(rank, world)
    t = sh.DistTransport(buffer_device="cpu")
    for _ in range(2):  # buffers are reused across exchanges
        t.exchange([s], sh.HALO)
        t.exchange([s], sh.IFACE)
    q.put((rank, {k: v.tolist() for k, v in s.got.items()}))
    dist.barrier()
    dist.destroy_process_group()


def test_dist_transport_pairs_every_send_with_its_receive_gloo():
    world = 3
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_transport_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, got in out.items():
        assert len(got) == 2 * (world - 1)
        for (kind, peer), vals in got.items():
            assert vals == _HostShard.values(peer, rank, kind).tolist()


def _dead_peer_main(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime
    import time

    import torch.distributed as dist

    from orion_b200 import shard as sh
    from test_shard_cpu import _HostShard

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=5))
    dist.barrier()
    if rank == 1:  # this rank leaves between steps, before the next exchange
        q.put((1, "left"))
        q.close()
        q.join_thread()
        os._exit(0)
    t0 = time.time()
    try:
        sh.DistTransport(buffer_device="cpu").exchange([_HostShard(0, world)], sh.HALO)
        msg = "no error"
    except Exception as e:  # the survivor learns of it on the host
        msg = f"raised {type(e).__name__} after {time.time() - t0:.1f} s"
    q.put((0, msg))
    q.close()
    q.join_thread()
    os._exit(0)


def test_exchange_with_a_departed_rank_fails_on_the_host_gloo():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_dead_peer_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
    assert out[1] == "left"
    assert out[0].startswith("raised"), out[0]
    assert float(out[0].split()[-2]) < 60.0


def test_sharded_exchanges_equal_single_case_random_layouts(plan_check):
    """Seeded random splits (even and uneven, up to 3 x 3 x 2 blocks) and owner
    maps (up to 4 shards): the sharded exchanges equal the single-case ones."""
    rng = np.random.default_rng(2024)
    for trial in range(6):
        split = tuple(int(v) for v in (rng.integers(1, 4), rng.integers(1, 4), rng.integers(1, 3)))
        if split == (1, 1, 1):
            split = (2, 1, 1)
        dims = tuple(int(13 * s + rng.integers(0, 9)) for s in split)
        uneven = int(rng.integers(0, 100)) if trial % 2 else None
        try:
            case = cases.small_case(f"r{trial}", dims=dims, split=split, uneven_seed=uneven)
        except ValueError:  # an uneven cut below the minimum block extent
            case = cases.small_case(f"r{trial}", dims=dims, split=split)
        nb = len(case.blocks)
        maps = []
        for _ in range(3):
            k = int(rng.integers(2, min(4, nb) + 1))
            m = [int(v) for v in rng.integers(0, k, nb)]
            ids = {v: i for i, v in enumerate(sorted(set(m)))}
            m = [ids[v] for v in m]
            if max(m) >= 1:
                maps.append(m)
        if not maps:
            continue
        r = subprocess.run([plan_check], input=_describe(case, maps), capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, (split, dims, r.stdout + r.stderr)
        assert sum("identical" in ln for ln in r.stdout.splitlines()) == len(maps)
