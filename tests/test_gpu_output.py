"""Solution output and restart on the GPU.

* The plain path's output after N steps against the files the reference's own
  PostProcess::write_solution writes after the same N steps: identical XML and
  layout; Float32 arrays equal within 1e-6 relative (the FP64 states agree
  within 1e-10, the far-field pow to an ulp).
* A restart written after 3 steps and loaded into a fresh case continues
  bit for bit like the uninterrupted run.
* The asynchronous writer snapshots at the call: its files equal a
  synchronous write of the same state although the case kept stepping.
"""
import os
import subprocess

import numpy as np
import pytest

import refio
from orion_b200 import _lib, cases, output, solver

pytestmark = pytest.mark.gpu
needs_ref = pytest.mark.skipif(not refio.reference_available(), reason="oracle/_ref not built")


def _split_vts(raw: bytes):
    body = raw.split(b"<AppendedData encoding=\"raw\">\n    _", 1)[1]
    arrays, off = [], 0
    for _ in range(6):
        nbytes = int(np.frombuffer(body, "<u4", 1, off)[0])
        arrays.append(np.frombuffer(body, "<f4", nbytes // 4, off + 4))
        off += 4 + nbytes
    return raw.split(b"<AppendedData", 1)[0], arrays


@needs_ref
def test_device_output_matches_the_reference_writer(tmp_path):
    case = cases.small_case("gout", dims=(33, 25, 23), split=(2, 1, 1), nsteps=3, noise_seed=4)
    cdir = str(tmp_path / "case")
    case.write_reference_inputs(cdir)
    os.makedirs(tmp_path / "ref", exist_ok=True)
    subprocess.run([refio.REF_HARNESS, cdir, "3", str(tmp_path / "ref"), "--vts", str(tmp_path / "refout" / "flow")],
                   check=True, capture_output=True)
    fs = solver.FlowFieldSet(case, precision=_lib.PREC_FP64)
    fs.step(3)
    paths = output.write_solution(fs, str(tmp_path / "ours" / "flow"), 3)
    fs.close()
    for p in paths:
        ref = open(tmp_path / "refout" / os.path.basename(p), "rb").read()
        ours = open(p, "rb").read()
        if p.endswith(".vtm"):
            assert ours == ref
            continue
        hr, ar = _split_vts(ref)
        ho, ao = _split_vts(ours)
        assert ho == hr
        for a, b in zip(ao, ar):
            assert a.shape == b.shape
            assert np.all(np.abs(a - b) <= 1e-6 * np.maximum(np.abs(b), 1e-30))


def test_restart_continues_bit_for_bit(tmp_path):
    case = cases.small_case("rst", dims=(33, 25, 23), split=(2, 1, 1), noise_seed=6)
    a = solver.FlowFieldSet(case, precision=_lib.PREC_FP64)
    a.step(3)
    output.save_restart(a, str(tmp_path / "r.npz"), step=3)
    ha = a.step(4)
    b = solver.FlowFieldSet(case, precision=_lib.PREC_FP64)
    assert output.load_restart(b, str(tmp_path / "r.npz")) == 3
    hb = b.step(4)
    assert np.array_equal(ha, hb)
    for n in range(len(case.blocks)):
        assert np.array_equal(a.download(n, "prim"), b.download(n, "prim"))
    a.close()
    b.close()


def test_async_writer_snapshots_at_the_call(tmp_path):
    case = cases.small_case("asy", dims=(33, 25, 23), noise_seed=2)
    fs = solver.FlowFieldSet(case, precision=_lib.PREC_MIXED)
    fs.step(2)
    sync = output.write_solution(fs, str(tmp_path / "sync" / "flow"), 2)
    fut = output.write_solution_async(fs, str(tmp_path / "async" / "flow"), 2)
    fs.step(3)  # keeps stepping while the files are written
    for p, q in zip(sync, fut.result(timeout=60)):
        assert open(p, "rb").read() == open(q, "rb").read()
    fs.close()
