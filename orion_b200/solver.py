"""Host-side mirror of ORION's per-step solver interface over the C ABI.

``FlowFieldSet`` here is a device-resident case (the reference's
``preprocess::FlowFieldSet``, src/preprocess/FlowField.hpp:73-87, holds host
arrays; this one holds device arrays and copies on request).  The classes
below carry the reference's names and static-method signatures
(src/solver/*.hpp, src/bc/PhysicalBC.hpp) so a driver loop reads the same:

    HaloExchanger().exchange_bc(bc, fs)
    apply_physical_bc(bc, fs, params)
    StateUpdater.update_flow_states(fs, params)
    TimeIntegrator.calculate_time_step(fs, params)
    FluxComputer.compute_viscous_rhs(fs, params)
    HaloExchanger().average_interface_residuals(bc, fs)
    InviscidFluxComputer.compute_inviscid_rhs(fs, params)
    StateUpdater.update_solution(fs, bc, params)
    ResidualMonitor.compute(fs, params) -> ResidualStats

Errors raise ``OrionError`` (the reference throws std::runtime_error or exits).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from ._lib import OrionError, check
from .cases import NG, Case, FlowParams, splitmix64_uniform


@dataclass
class ResidualStats:
    """ResidualStats (src/solver/ResidualMonitor.hpp:8-12) plus phydtime."""
    rms_residual: float
    max_residual: float
    max_loc: tuple
    phydtime: float


def _params_struct(p: FlowParams) -> _lib.Params:
    s = _lib.Params()
    s.gamma, s.moo, s.reynolds, s.prl = p.gamma, p.moo, p.reynolds, p.prl
    s.cfl, s.twall, s.tref, s.visc = p.cfl, p.twall, p.tref, p.visc
    s.roo, s.uoo, s.voo, s.woo, s.poo, s.too = p.roo, p.uoo, p.voo, p.woo, p.poo, p.too
    s.nvis, s.method, s.ntmst, s.csrv = p.nvis, p.method, p.ntmst, p.csrv
    return s


def _block_descs(case: Case):
    keep = []
    descs = (_lib.BlockDesc * len(case.blocks))()
    for n, b in enumerate(case.blocks):
        regs = (_lib.Region * len(b.regions))()
        for r, g in enumerate(b.regions):
            regs[r].s_st[:] = g.s_st
            regs[r].s_ed[:] = g.s_ed
            regs[r].bctype = g.bctype
            regs[r].t_st[:] = g.t_st
            regs[r].t_ed[:] = g.t_ed
            regs[r].nbt = g.nbt
            regs[r].ibcwin = g.ibcwin
        keep.append(regs)
        descs[n].idim, descs[n].jdim, descs[n].kdim = b.idim, b.jdim, b.kdim
        descs[n].nregions = len(b.regions)
        descs[n].regions = C.cast(regs, C.POINTER(_lib.Region))
    return descs, keep


def grid_metrics(block, gcl: int = 1):
    """Metrics (9, nz, ny, nx) and vol (nz, ny, nx) of one block, padded, ghosts zero."""
    lib = _lib.load()
    nx, ny, nz = block.padded
    met = np.zeros((9, nz, ny, nx))
    vol = np.zeros((nz, ny, nx))
    x = np.ascontiguousarray(block.x, dtype=np.float64)
    y = np.ascontiguousarray(block.y, dtype=np.float64)
    z = np.ascontiguousarray(block.z, dtype=np.float64)
    check(lib.orion_grid_metrics_host(block.idim, block.jdim, block.kdim, x.ctypes.data, y.ctypes.data,
                                      z.ctypes.data, gcl, met.ctypes.data, vol.ctypes.data))
    return met, vol


def footprint_estimate(case: Case, precision: int = _lib.PREC_FP64) -> int:
    descs, _keep = _block_descs(case)
    return int(_lib.load().orion_footprint_estimate(len(case.blocks), descs, precision))


class FlowFieldSet:
    """A device-resident case.  ``precision`` is PREC_FP64 (plain) or PREC_MIXED."""

    def __init__(self, case: Case, precision: int = _lib.PREC_FP64, device: int = 0,
                 metrics: Optional[Sequence] = None, init: bool = True):
        lib = _lib.load()
        check(lib.orion_gpu_init(device))
        self.case = case
        self.precision = precision
        self.params = case.params
        descs, keep = _block_descs(case)
        h = C.c_void_p()
        check(lib.orion_case_create(len(case.blocks), descs, C.byref(_params_struct(case.params)), precision,
                                    C.byref(h)))
        self._h = h
        self._keep = keep
        if metrics is None:  # on the device, from the coordinates
            for n, b in enumerate(case.blocks):
                x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (b.x, b.y, b.z))
                check(lib.orion_case_grid_metrics(self._h, n, x.ctypes.data, y.ctypes.data, z.ctypes.data,
                                                  case.params.gcl))
        else:
            for n, (met, vol) in enumerate(metrics):
                self.upload(n, "metrics", met)
                self.upload(n, "vol", vol)
        if init:
            check(lib.orion_case_init_flow(self._h, case.noise_seed, case.noise_amp))
            self.sync()

    # ------------------------------------------------------------------
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

    def set_params(self, params: FlowParams):
        """Replaces the flow parameters for the steps enqueued from now on
        (orion_case_set_params); a grouped case keeps stepping in its group."""
        check(_lib.load().orion_case_set_params(self._h, C.byref(_params_struct(params))))
        self.params = params

    def stream_ptr(self) -> int:
        v = C.c_void_p()
        check(_lib.load().orion_case_stream(self._h, C.byref(v)))
        return int(v.value or 0)

    def step_launches(self) -> int:
        v = C.c_int()
        check(_lib.load().orion_case_step_launches(self._h, C.byref(v)))
        return int(v.value)

    def sweep_schedule(self) -> dict:
        v = (C.c_int * 5)()
        check(_lib.load().orion_case_sweep_schedule(self._h, v))
        mode = _lib.SWEEP_NAMES[v[0]]
        return {"mode": mode, "units": v[1], "cluster_size": v[2], "threads": v[3], "hyperplanes": v[4]}

    def footprint(self) -> int:
        v = C.c_size_t()
        check(_lib.load().orion_case_footprint(self._h, C.byref(v)))
        return int(v.value)

    def upload(self, block: int, field: str, arr: np.ndarray):
        fid = _lib.FIELD_NAMES[field]
        b = self.case.blocks[block]
        nx, ny, nz = b.padded
        nc = _lib.FIELD_NCOMP[fid]
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.size != nc * nx * ny * nz:
            raise OrionError(f"{field}: expected {nc * nx * ny * nz} values, got {a.size}")
        check(_lib.load().orion_case_upload(self._h, block, fid, a.ctypes.data))

    def download(self, block: int, field: str) -> np.ndarray:
        fid = _lib.FIELD_NAMES[field]
        b = self.case.blocks[block]
        nx, ny, nz = b.padded
        nc = _lib.FIELD_NCOMP[fid]
        a = np.empty((nc, nz, ny, nx) if nc > 1 else (nz, ny, nx))
        check(_lib.load().orion_case_download(self._h, block, fid, a.ctypes.data))
        return a

    def upload_state(self, state: dict):
        """Uploads every field of a reference-style state (per block dict of arrays)."""
        for n, blk in enumerate(state["blocks"]):
            for name in ("prim", "q", "dq", "metrics", "vol", "dt", "c", "mu"):
                if name in blk:
                    self.upload(n, name, blk[name])

    # ------------------------------------------------------------------
    def step(self, nsteps: int) -> np.ndarray:
        """Runs nsteps whole steps (graph-captured); returns the residual history
        as an array (nsteps, 8): rms, max, loc[5], phydtime."""
        hist = (_lib.Residual * max(nsteps, 1))()
        check(_lib.load().orion_step(self._h, nsteps, hist))
        out = np.zeros((nsteps, 8))
        for s in range(nsteps):
            r = hist[s]
            out[s, 0] = r.rms
            out[s, 1] = r.max
            out[s, 2:7] = list(r.max_loc)
            out[s, 7] = r.phydtime
        return out

    def step_async(self, nsteps: int):
        check(_lib.load().orion_step_async(self._h, nsteps))

    def get_schedule(self) -> dict:
        s = _lib.Schedule()
        check(_lib.load().orion_case_get_schedule(self._h, C.byref(s)))
        return {"sweep": _lib.SWEEP_NAMES[s.sweep_form], "cluster_size": s.cluster_size, "lanes": s.lanes}

    def set_schedule(self, sweep: str, cluster_size: int = 0, lanes: int = 32):
        """Fixes the step schedule: sweep form (tiles | planes | grid | cluster), cluster size
        (8, 16, 0 = largest co-resident) and grid lines per CTA of the line kernels."""
        form = {v: k for k, v in _lib.SWEEP_NAMES.items()}[sweep]
        s = _lib.Schedule(form, cluster_size, lanes, 0.0)
        check(_lib.load().orion_case_set_schedule(self._h, C.byref(s)))

    def autotune(self, steps_per_trial: int = 3) -> dict:
        """Times candidate schedules on this case and keeps the fastest; the
        solution is unchanged.  Returns the chosen schedule and every trial."""
        trials = (_lib.Schedule * 16)()
        n = C.c_int()
        best = _lib.Schedule()
        check(_lib.load().orion_case_autotune(self._h, steps_per_trial, trials, 16, C.byref(n), C.byref(best)))
        row = lambda s: {"sweep": _lib.SWEEP_NAMES[s.sweep_form], "cluster_size": s.cluster_size, "lanes": s.lanes,
                         "ms_per_step": round(float(s.ms_per_step), 4)}
        return {"best": row(best), "trials": [row(trials[i]) for i in range(min(n.value, 16))]}

    def submit(self, nsteps: int):
        """Enqueues nsteps steps and the asynchronous copy of their residual
        history; returns at once (orion_step_submit)."""
        check(_lib.load().orion_step_submit(self._h, nsteps))

    def poll(self, cap: int = 4096):
        """None while submitted steps run; else their history (n, 8) as step() returns it."""
        buf = getattr(self, "_poll_buf", None)
        if buf is None or len(buf) < max(cap, 1):  # one buffer per case, reused: request loops poll often
            buf = self._poll_buf = (_lib.Residual * max(cap, 1))()
        n = C.c_int()
        rc = _lib.load().orion_case_poll(self._h, buf, cap, C.byref(n))
        if rc == 0:
            return None
        check(rc if rc < 0 else 0)
        out = np.zeros((n.value, 8))
        for s in range(n.value):
            r = buf[s]
            out[s, 0] = r.rms
            out[s, 1] = r.max
            out[s, 2:7] = list(r.max_loc)
            out[s, 7] = r.phydtime
        return out

    # -- pipelined host I/O: copies overlap the steps (orion_io_*) --------
    def _prim_buffer(self, block: int, arr) -> int:
        nx, ny, nz = self.case.blocks[block].padded
        n = 6 * nx * ny * nz
        if isinstance(arr, np.ndarray):
            if arr.dtype != np.float64 or not arr.flags.c_contiguous or arr.size != n:
                raise OrionError(f"prim of block {block}: a C-contiguous float64 array of {n} values")
            return arr.ctypes.data
        if arr.dtype.itemsize != 8 or not arr.is_contiguous() or arr.numel() != n:  # a (pinned) torch tensor
            raise OrionError(f"prim of block {block}: a contiguous float64 tensor of {n} values")
        return arr.data_ptr()

    def io_put(self, block: int, prim):
        """Enqueues the copy of a block's prim from host memory (pinned: a
        torch tensor from pin_memory(), for the copy to overlap the steps)."""
        check(_lib.load().orion_io_put(self._h, block, self._prim_buffer(block, prim)))

    def io_step(self, nsteps: int = 1):
        """Installs the blocks put since the last io step, enqueues nsteps steps
        (history as submit(); poll it) and the copy of the result to staging."""
        check(_lib.load().orion_io_step(self._h, nsteps))

    def io_get(self, block: int, prim):
        """Enqueues the copy of a block's prim, as the last io step left it, into
        host memory; valid after io_wait()."""
        check(_lib.load().orion_io_get(self._h, block, self._prim_buffer(block, prim)))

    def io_wait(self):
        check(_lib.load().orion_io_wait(self._h))

    def last_residual(self) -> ResidualStats:
        r = _lib.Residual()
        check(_lib.load().orion_last_residual(self._h, C.byref(r)))
        return ResidualStats(r.rms, r.max, tuple(r.max_loc), r.phydtime)

    def conservative(self, block: int) -> np.ndarray:
        """Q from the current prim (update_conservative_block formula,
        src/solver/StateUpdater.cpp:108-124) at interior points."""
        prim = self.download(block, "prim")
        return conservative_from_prim(prim, self.params.gamma)


class CaseGroup:
    """Several device-resident cases stepped together: every stage is one
    launch over the blocks of all members (orion_group_*).  Each member's
    results are the same as when it steps alone; poll the members
    (FlowFieldSet.poll) after submit().  Close the group before closing or
    regrouping its members."""

    def __init__(self, members: Sequence[FlowFieldSet]):
        lib = _lib.load()
        self.members = list(members)
        arr = (C.c_void_p * len(self.members))(*[m.handle for m in self.members])
        h = C.c_void_p()
        check(lib.orion_group_create(len(self.members), arr, C.byref(h)))
        self._h = h

    def submit(self, nsteps: int):
        check(_lib.load().orion_group_submit(self._h, nsteps))

    def sync(self):
        check(_lib.load().orion_group_sync(self._h))

    def step_launches(self) -> int:
        v = C.c_int()
        check(_lib.load().orion_group_step_launches(self._h, C.byref(v)))
        return int(v.value)

    def step(self, nsteps: int) -> List[np.ndarray]:
        """Runs nsteps steps of every member; returns each member's history."""
        self.submit(nsteps)
        self.sync()
        return [m.poll(max(nsteps, 1)) for m in self.members]

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().orion_group_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def conservative_from_prim(prim: np.ndarray, gamma: float) -> np.ndarray:
    rho, u, v, w, p = prim[0], prim[1], prim[2], prim[3], prim[4]
    rc = np.where(rho < 0.0, np.abs(rho), rho)
    q = np.empty((5,) + rho.shape)
    q[0] = rc
    q[1] = rc * u
    q[2] = rc * v
    q[3] = rc * w
    ke = 0.5 * rc * (u * u + v * v + w * w)
    q[4] = p * (1.0 / (gamma - 1.0)) + ke
    return q


# ---------------------------------------------------------------------------
# reference-named facade
# ---------------------------------------------------------------------------
class HaloExchanger:
    """src/solver/HaloExchanger.hpp"""

    def exchange_bc(self, bc, fs: FlowFieldSet):
        check(_lib.load().orion_exchange_bc(fs.handle))

    def average_interface_residuals(self, bc, fs: FlowFieldSet):
        check(_lib.load().orion_average_interface_residuals(fs.handle))


def apply_physical_bc(bc, fs: FlowFieldSet, params=None):
    """src/bc/PhysicalBC.hpp:17-19"""
    check(_lib.load().orion_apply_physical_bc(fs.handle))


class StateUpdater:
    """src/solver/StateUpdater.hpp"""

    @staticmethod
    def update_flow_states(fs: FlowFieldSet, params=None):
        check(_lib.load().orion_update_flow_states(fs.handle))

    @staticmethod
    def update_solution(fs: FlowFieldSet, bc=None, params=None):
        check(_lib.load().orion_update_solution(fs.handle))


class TimeIntegrator:
    """src/solver/TimeIntegrator.hpp"""

    @staticmethod
    def calculate_time_step(fs: FlowFieldSet, params=None) -> float:
        lib = _lib.load()
        check(lib.orion_calculate_time_step(fs.handle))
        v = C.c_double()
        check(lib.orion_phydtime(fs.handle, C.byref(v)))
        if params is not None and hasattr(params, "phydtime"):
            params.phydtime = v.value
        return v.value


class FluxComputer:
    """src/solver/FluxComputer.hpp"""

    @staticmethod
    def compute_viscous_rhs(fs: FlowFieldSet, params=None):
        check(_lib.load().orion_compute_viscous_rhs(fs.handle))


class InviscidFluxComputer:
    """src/solver/InviscidFluxComputer.hpp"""

    @staticmethod
    def compute_inviscid_rhs(fs: FlowFieldSet, params=None):
        check(_lib.load().orion_compute_inviscid_rhs(fs.handle))


class ResidualMonitor:
    """src/solver/ResidualMonitor.hpp"""

    @staticmethod
    def compute(fs: FlowFieldSet, params=None) -> ResidualStats:
        r = _lib.Residual()
        check(_lib.load().orion_residual_compute(fs.handle, C.byref(r)))
        return ResidualStats(r.rms, r.max, tuple(r.max_loc), r.phydtime)


def initial_prim(case: Case) -> List[np.ndarray]:
    """Host restatement of the device initial state (freestream + noise + T),
    used to check orion_case_init_flow."""
    p = case.params
    out = []
    start = 0
    for b in case.blocks:
        nx, ny, nz = b.padded
        n = nx * ny * nz
        prim = np.zeros((6, nz, ny, nx))
        prim[0] = p.roo
        prim[1] = p.uoo
        prim[2] = p.voo
        prim[3] = p.woo
        prim[4] = p.poo
        if case.noise_amp != 0.0:
            r = splitmix64_uniform(case.noise_seed, 2 * start, 2 * n).reshape(n, 2)
            r1 = r[:, 0].reshape(nz, ny, nx)
            r2 = r[:, 1].reshape(nz, ny, nx)
            prim[0] = prim[0] * (1.0 + case.noise_amp * (2.0 * r1 - 1.0))
            prim[1] = prim[1] * (1.0 + case.noise_amp * (2.0 * r2 - 1.0))
        rho = np.maximum(prim[0], 1.0e-30)
        a2 = p.gamma * prim[4] / rho
        prim[5] = (p.moo * p.moo) * a2 if p.nvis == 1 else p.too
        out.append(prim)
        start += n
    return out
