"""Block-sharded stepping: the blocks of one case spread over shards, one GPU
per shard, in place of the reference's MPI decomposition.

The reference runs one MPI rank per block group and exchanges, every step,
the interface halo (src/solver/HaloExchanger.cpp:70-179), the interface
residual averages (HaloExchanger.cpp:186-398, twice) and the residual
reductions (src/solver/ResidualMonitor.cpp:11-137).  Here each shard is a
device case of its own blocks (orion_case_create_shard); the two exchanges
travel as packed FP64 buffers that the shard's own kernels gather and scatter
(orion_shard_pack / orion_shard_unpack), and the residual is reduced from each
shard's raw sum, maximum and key, so the result is the whole case's:
the state is bit-identical to the single-case step, the maximum and its
location identical, the rms equal up to the order of one sum.

* partition(case, n): owner of every block, contiguous runs of blocks with
  balanced point counts.
* Shard: one shard's device case.
* LocalTransport: every shard in this process (one GPU); a peer's buffer is
  handed over in device memory.
* DistTransport: one shard per process over torch.distributed point-to-point
  (NCCL between GPUs; the shard's buffers are CUDA tensors).
* ShardGroup(shards, transport).step(): one step in OrionSolver::solve's order.

    python -m orion_b200.shard --config 3 --shards 4 --precision mixed

times a configuration as shards on one GPU against the same case as one.
"""
from __future__ import annotations

import ctypes as C
import math
from typing import Dict, List, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import OrionError, check
from .cases import Case
from .solver import ResidualStats, _block_descs, _params_struct

HALO, IFACE = _lib.XCHG_HALO, _lib.XCHG_IFACE


def partition(case: Case, nshards: int) -> List[int]:
    """Owner of every block: contiguous runs in block order.  A shard is closed
    when the next block's midpoint passes its equal share of the points, or
    when the blocks left are just enough for the shards left."""
    nb = len(case.blocks)
    if not 1 <= nshards <= nb:
        raise OrionError(f"cannot spread {nb} blocks over {nshards} shards")
    pts = [b.npoints for b in case.blocks]
    total = float(sum(pts))
    owner: List[int] = []
    s, cum, count = 0, 0.0, 0
    for b in range(nb):
        if s < nshards - 1 and count > 0 and (cum + pts[b] / 2 > total * (s + 1) / nshards
                                              or nb - b == nshards - 1 - s):
            s, count = s + 1, 0
        owner.append(s)
        count += 1
        cum += pts[b]
    return owner


def plan_counts(case: Case, owner: Sequence[int], rank: int, kind: int) -> Tuple[np.ndarray, np.ndarray]:
    """Doubles shard `rank` sends to / receives from every shard (host only)."""
    descs, _keep = _block_descs(case)
    n = max(owner) + 1
    own = (C.c_int * len(owner))(*owner)
    snd, rcv = (C.c_longlong * n)(), (C.c_longlong * n)()
    check(_lib.load().orion_shard_plan_counts(len(case.blocks), descs, own, rank, kind, snd, rcv))
    return np.array(snd[:], dtype=np.int64), np.array(rcv[:], dtype=np.int64)


def reduce_partials(parts: Sequence[Tuple[float, float, int, float]], case: Case) -> ResidualStats:
    """Residual statistics of the whole case from every shard's (sum, max, key,
    dtmin): the maximum with the smallest key among equal maxima, as the
    single-case reduction combines its partials; the key decoded to the global
    (block, i, j, k, component), 1-based except the block."""
    total = sum(p[0] for p in parts)
    mx, key = -1.0, (1 << 63) - 1
    for p in parts:
        if p[1] > mx or (p[1] == mx and p[2] < key):
            mx, key = p[1], int(p[2])
    dtmin = min(p[3] for p in parts)
    npts = sum(b.npoints for b in case.blocks)
    pt, comp = divmod(key, 5)
    base = 0
    loc = (0, 0, 0, 0, 0)
    for g, b in enumerate(case.blocks):
        if base <= pt < base + b.npoints:
            n = pt - base
            loc = (g, n % b.idim + 1, (n // b.idim) % b.jdim + 1, n // (b.idim * b.jdim) + 1, comp + 1)
            break
        base += b.npoints
    rms = math.sqrt(total / (5.0 * npts)) if npts else 0.0
    return ResidualStats(rms_residual=rms, max_residual=mx, max_loc=loc, phydtime=dtmin)


class Shard:
    """The blocks owner[b] == rank of `case` as one device case.  Metrics come
    from the coordinates on the device and the initial state from the case's
    seeded noise, keyed by global point, so every shard starts where the whole
    case starts."""

    def __init__(self, case: Case, owner: Sequence[int], rank: int, precision: int = _lib.PREC_FP64,
                 device: int = 0, init: bool = True):
        lib = _lib.load()
        check(lib.orion_gpu_init(device))
        if len(owner) != len(case.blocks):
            raise OrionError("owner list length differs from the block count")
        self.case, self.owner, self.rank, self.precision = case, list(owner), rank, precision
        self.nshards = max(owner) + 1
        self.device = device
        descs, self._keep = _block_descs(case)
        own = (C.c_int * len(owner))(*owner)
        h = C.c_void_p()
        check(lib.orion_case_create_shard(len(case.blocks), descs, own, rank, C.byref(_params_struct(case.params)),
                                          precision, C.byref(h)))
        self._h = h
        n = C.c_int()
        ids = (C.c_int * len(case.blocks))()
        check(lib.orion_shard_blocks(h, C.byref(n), ids))
        self.global_ids = list(ids[:n.value])
        self._local = {g: i for i, g in enumerate(self.global_ids)}
        for i, g in enumerate(self.global_ids):
            b = case.blocks[g]
            x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (b.x, b.y, b.z))
            check(lib.orion_case_grid_metrics(h, i, x.ctypes.data, y.ctypes.data, z.ctypes.data, case.params.gcl))
        if init:
            check(lib.orion_case_init_flow(h, case.noise_seed, case.noise_amp))
        self.sync()

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().orion_case_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        check(_lib.load().orion_case_sync(self._h))

    def counts(self, kind: int, peer: int) -> Tuple[int, int]:
        s, r = C.c_longlong(), C.c_longlong()
        check(_lib.load().orion_shard_counts(self._h, kind, peer, C.byref(s), C.byref(r)))
        return int(s.value), int(r.value)

    def pack(self, kind: int, peer: int, dev_ptr: int):
        check(_lib.load().orion_shard_pack(self._h, kind, peer, C.c_void_p(dev_ptr)))

    def unpack(self, kind: int, peer: int, dev_ptr: int):
        check(_lib.load().orion_shard_unpack(self._h, kind, peer, C.c_void_p(dev_ptr)))

    def residual(self) -> Tuple[float, float, int, float]:
        r = _lib.ShardResidual()
        check(_lib.load().orion_shard_residual(self._h, C.byref(r)))
        return float(r.sum), float(r.max), int(r.key), float(r.dtmin)

    def owns(self, block: int) -> bool:
        return block in self._local

    def download(self, block: int, field: str) -> np.ndarray:
        """A field of GLOBAL block `block` (owned by this shard), padded layout."""
        if block not in self._local:
            raise OrionError(f"block {block} is not in shard {self.rank}")
        fid = _lib.FIELD_NAMES[field]
        nx, ny, nz = self.case.blocks[block].padded
        nc = _lib.FIELD_NCOMP[fid]
        a = np.empty((nc, nz, ny, nx) if nc > 1 else (nz, ny, nx))
        check(_lib.load().orion_case_download(self._h, self._local[block], fid, a.ctypes.data))
        return a


def _device_buffer(n: int, device):
    """FP64 buffer of n values on CUDA device `device` (an int), or on the
    device torch names by a string ("cpu" for gloo)."""
    import torch
    dev = f"cuda:{device}" if isinstance(device, int) else device
    return torch.empty(max(n, 1), dtype=torch.float64, device=dev)


class LocalTransport:
    """Every shard in this process, on one GPU: the sender's pack buffer is the
    receiver's unpack buffer.  The sender's stream is drained before the
    receiver reads, and every shard's stream after the exchange, so a buffer
    is never rewritten while a reader is pending."""

    def __init__(self):
        self._bufs: Dict[Tuple[int, int, int], object] = {}

    def exchange(self, shards: Sequence[Shard], kind: int):
        for s in shards:
            for p in shards:
                if p.rank == s.rank:
                    continue
                nsend, nrecv_at_p = s.counts(kind, p.rank)[0], p.counts(kind, s.rank)[1]
                if nsend != nrecv_at_p:
                    raise OrionError(f"shards {s.rank}->{p.rank} disagree on the exchange size")
                if nsend == 0:
                    continue
                buf = self._bufs.get((kind, s.rank, p.rank))
                if buf is None:
                    buf = self._bufs[(kind, s.rank, p.rank)] = _device_buffer(nsend, s.device)
                s.pack(kind, p.rank, buf.data_ptr())
                s.sync()
                p.unpack(kind, s.rank, buf.data_ptr())
        for s in shards:
            s.sync()

    def reduce(self, shards: Sequence[Shard], parts) -> List[Tuple[float, float, int, float]]:
        return list(parts)


class DistTransport:
    """One shard per process over torch.distributed point-to-point: every rank
    posts its sends and receives to every peer together (batch_isend_irecv),
    so the order of ranks cannot deadlock.  The packs finish before the
    transfer starts and the transfer before the unpacks.

    * Default: the buffers live on the shard's GPU and the group moves them
      (NCCL between GPUs).
    * host_staging=True: the shard packs into and unpacks from its GPU
      buffers, and host copies of them cross the group (gloo over TCP, for
      machines without a GPU-to-GPU path).
    * buffer_device="cpu": the buffers themselves are host memory; only for
      shards whose pack/unpack work on host memory."""

    def __init__(self, group=None, buffer_device=None, host_staging: bool = False):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.buffer_device = buffer_device
        self.host_staging = host_staging
        self._bufs: Dict[Tuple[int, int, str], object] = {}

    def _buf(self, kind: int, peer: int, side: str, n: int, device):
        key = (kind, peer, side, str(device))
        b = self._bufs.get(key)
        if b is None or b.numel() < n:
            b = self._bufs[key] = _device_buffer(n, device)
        return b

    def exchange(self, shards: Sequence[Shard], kind: int):
        import torch
        (s,) = shards
        dev = self.buffer_device or s.device
        ops, sends, recvs = [], [], []
        for peer in range(s.nshards):
            if peer == s.rank:
                continue
            nsend, nrecv = s.counts(kind, peer)
            if nsend:
                b = self._buf(kind, peer, "send", nsend, dev)
                s.pack(kind, peer, b.data_ptr())
                sends.append((peer, b[:nsend]))
            if nrecv:
                recvs.append((peer, self._buf(kind, peer, "recv", nrecv, dev)[:nrecv]))
        s.sync()  # packs done before anything reads the buffers
        for peer, b in sends:
            w = self._buf(kind, peer, "send-host", b.numel(), "cpu")[:b.numel()] if self.host_staging else b
            if self.host_staging:
                w.copy_(b)
            ops.append(self.dist.P2POp(self.dist.isend, w, peer, self.group))
        wires = []
        for peer, b in recvs:
            w = self._buf(kind, peer, "recv-host", b.numel(), "cpu")[:b.numel()] if self.host_staging else b
            wires.append(w)
            ops.append(self.dist.P2POp(self.dist.irecv, w, peer, self.group))
        if ops:
            for req in self.dist.batch_isend_irecv(ops):
                req.wait()
        if self.host_staging:
            for (peer, b), w in zip(recvs, wires):
                b.copy_(w)
        if self.buffer_device is None:
            torch.cuda.synchronize(s.device)  # received data in place before the case's stream reads it
        for peer, b in recvs:
            s.unpack(kind, peer, b.data_ptr())

    def reduce(self, shards: Sequence[Shard], parts) -> List[Tuple[float, float, int, float]]:
        dev = "cpu" if (self.host_staging or self.buffer_device) else f"cuda:{shards[0].device}"
        return gather_partials(parts[0], self.dist, self.group, device=dev)


def gather_partials(part: Tuple[float, float, int, float], dist, group=None, device: str = "cpu"):
    """Every rank's (sum, max, key, dtmin), on every rank (the key is exact in
    FP64 below 2**53)."""
    import torch
    t = torch.tensor([part[0], part[1], float(part[2]), part[3]], dtype=torch.float64, device=device)
    out = [torch.empty_like(t) for _ in range(dist.get_world_size(group))]
    dist.all_gather(out, t, group=group)
    return [(float(v[0]), float(v[1]), int(v[2]), float(v[3])) for v in (o.cpu() for o in out)]


class ShardGroup:
    """Steps the shards of this process; with a DistTransport, every process
    steps its own shard and the group is the whole case."""

    def __init__(self, shards: Sequence[Shard], transport):
        self.shards = list(shards)
        self.transport = transport
        self.case = self.shards[0].case

    def _each(self, fn: str):
        lib = _lib.load()
        for s in self.shards:
            check(getattr(lib, fn)(s.handle))

    def average(self):
        self._each("orion_shard_average_begin")
        self.transport.exchange(self.shards, IFACE)
        self._each("orion_shard_average_end")

    def step(self) -> ResidualStats:
        """One step in the order of OrionSolver::solve (src/core/OrionSolver.cpp:141-209)."""
        self._each("orion_exchange_bc")
        self.transport.exchange(self.shards, HALO)
        self._each("orion_apply_physical_bc")
        self._each("orion_update_flow_states")
        self._each("orion_calculate_time_step")
        self._each("orion_compute_viscous_rhs")
        if self.case.params.nvis == 1:
            self.average()
        self._each("orion_compute_inviscid_rhs")
        self.average()
        self._each("orion_update_solution")
        parts = [s.residual() for s in self.shards]
        return reduce_partials(self.transport.reduce(self.shards, parts), self.case)

    def run(self, nsteps: int) -> List[ResidualStats]:
        return [self.step() for _ in range(nsteps)]


def _per_stage_step(fs, nvis: int):
    from . import solver
    halo = solver.HaloExchanger()
    halo.exchange_bc(None, fs)
    solver.apply_physical_bc(None, fs)
    solver.StateUpdater.update_flow_states(fs)
    solver.TimeIntegrator.calculate_time_step(fs)
    solver.FluxComputer.compute_viscous_rhs(fs)
    if nvis == 1:
        halo.average_interface_residuals(None, fs)
    solver.InviscidFluxComputer.compute_inviscid_rhs(fs)
    halo.average_interface_residuals(None, fs)
    solver.StateUpdater.update_solution(fs)
    return solver.ResidualMonitor.compute(fs)


def main(argv=None):
    """One GPU: a configuration as N shards (LocalTransport) against the same
    case through the same per-stage entry points, wall clock per step (both
    wait for the residual every step), and the bytes the shards exchange."""
    import argparse
    import json
    import time

    from . import cases, solver

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--config", type=int, default=3)
    ap.add_argument("--shards", type=int, default=4)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "plain"])
    a = ap.parse_args(argv)
    case = cases.config(a.config)
    prec = _lib.PREC_MIXED if a.precision == "mixed" else _lib.PREC_FP64
    nvis = case.params.nvis

    fs = solver.FlowFieldSet(case, precision=prec)
    for _ in range(a.warmup):
        _per_stage_step(fs, nvis)
    t0 = time.perf_counter()
    for _ in range(a.steps):
        r1 = _per_stage_step(fs, nvis)
    single = (time.perf_counter() - t0) / a.steps
    fs.close()

    owner = partition(case, a.shards)
    shards = [Shard(case, owner, r, precision=prec) for r in range(a.shards)]
    group = ShardGroup(shards, LocalTransport())
    for _ in range(a.warmup):
        group.step()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        r2 = group.step()
    sharded = (time.perf_counter() - t0) / a.steps
    halo = sum(s.counts(HALO, p.rank)[0] for s in shards for p in shards if p.rank != s.rank)
    iface = sum(s.counts(IFACE, p.rank)[0] for s in shards for p in shards if p.rank != s.rank)
    for s in shards:
        s.close()
    print(json.dumps({
        "workload": case.name, "precision": a.precision, "shards": a.shards, "owner": owner,
        "steps": a.steps, "ms_per_step_single_per_stage": single * 1e3, "ms_per_step_sharded": sharded * 1e3,
        "exchanged_bytes_per_step": 8 * (halo + (2 if nvis == 1 else 1) * iface),
        "halo_bytes": 8 * halo, "iface_bytes_per_average": 8 * iface,
        "same_residual_max": r1.max_residual == r2.max_residual and tuple(r1.max_loc) == tuple(r2.max_loc),
        "timing": "wall clock; both paths wait for the residual every step, the sharded one also at every exchange",
    }))


if __name__ == "__main__":
    main()
