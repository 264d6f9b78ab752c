"""The allocation-free residual entry point against the case-based one.

orion_residual_block_noalloc exists for callers that cannot allocate device
memory where they need a residual norm (a solver that reserved its whole
budget up front, or a step running inside another framework's memory pool):
they hand in their own dq / vol / dt device arrays and the reduction uses a
fixed array in the library's device memory instead of a cudaMalloc'd buffer.
Its statistics must equal those of orion_residual_compute on the same data,
on consecutive calls (the shared scratch keeps the previous call's contents).
"""
import ctypes as C

import numpy as np
import pytest

from orion_b200 import _lib, cases, solver

pytestmark = pytest.mark.gpu


def _noalloc(dq, vol, dt, dims):
    import torch

    lib = _lib.load()
    out = _lib.Residual()
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.orion_residual_block_noalloc(C.c_void_p(dq.data_ptr()), C.c_void_p(vol.data_ptr()),
                                          C.c_void_p(dt.data_ptr()), dims[0], dims[1], dims[2],
                                          C.c_void_p(stream), C.byref(out))
    return rc, out


def _device_copies(fs):
    import torch

    return (torch.from_numpy(fs.download(0, "dq")).cuda(), torch.from_numpy(fs.download(0, "vol")).cuda(),
            torch.from_numpy(fs.download(0, "dt")).cuda())


def test_noalloc_residual_matches_case_residual_on_consecutive_calls():
    import torch

    case = cases.small_case("noalloc", dims=(29, 21, 17), split=(1, 1, 1), noise_seed=21)
    fs = solver.FlowFieldSet(case)
    dims = case.blocks[0].dims
    for call in range(2):
        fs.step(2 + call)  # different data on each call
        ref = solver.ResidualMonitor.compute(fs)
        dq, vol, dt = _device_copies(fs)
        rc, out = _noalloc(dq, vol, dt, dims)
        assert rc == 0, _lib.load().orion_last_error()
        assert abs(out.rms - ref.rms_residual) <= 1e-12 * ref.rms_residual
        assert abs(out.max - ref.max_residual) <= 1e-12 * ref.max_residual
        assert tuple(out.max_loc) == tuple(ref.max_loc)
        torch.cuda.synchronize()
    fs.close()


def test_noalloc_residual_rejects_blocks_beyond_its_scratch():
    import torch

    t = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc, _ = _noalloc(t, t, t, (205, 205, 205))  # 8,615,125 > ORION_NOALLOC_MAX_POINTS
    assert rc == -1
    assert b"at most" in _lib.load().orion_last_error()


def test_noalloc_residual_refuses_a_capturing_stream():
    import torch

    case = cases.small_case("noalloc_cap", dims=(17, 13, 13), split=(1, 1, 1), noise_seed=3)
    fs = solver.FlowFieldSet(case)
    fs.step(1)
    dq, vol, dt = _device_copies(fs)
    dims = case.blocks[0].dims
    rc, _ = _noalloc(dq, vol, dt, dims)  # first call on the device: outside any capture
    assert rc == 0, _lib.load().orion_last_error()
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        g.capture_begin()
        try:
            rc, _ = _noalloc(dq, vol, dt, dims)
        finally:
            g.capture_end()
    assert rc == -1
    assert b"capturing" in _lib.load().orion_last_error()
    # the shared scratch still serves the next ordinary call
    ref = solver.ResidualMonitor.compute(fs)
    rc, out = _noalloc(dq, vol, dt, dims)
    assert rc == 0 and abs(out.rms - ref.rms_residual) <= 1e-12 * ref.rms_residual
    del g
    fs.close()
