"""Solution output format against the reference's own writer (CPU).

The reference build writes its VTS/VTM files for a small case
(PostProcess::write_solution, via the oracle driver's --vts option).  From the
reference's own final state, orion_b200.output must produce the same files
byte for byte: the same XML, offsets and UInt32-framed Float32 arrays.
"""
import os
import subprocess

import numpy as np
import pytest

import refio
from orion_b200 import cases, output

needs_ref = pytest.mark.skipif(not refio.reference_available(), reason="oracle/_ref not built")


def _fields_from_prim(prim, gamma):
    """What orion_case_pack_output computes, in numpy (FP64, then float32)."""
    it = prim[:, 3:-3, 3:-3, 3:-3].reshape(6, -1)
    r, u, v, w, p, T = it
    v2 = u * u + v * v + w * w
    c2 = gamma * p / r
    mach = np.where(c2 > 1e-30, np.sqrt(v2 / np.where(c2 > 1e-30, c2, 1.0)), 0.0)
    return np.stack([r, p, T, mach, u, v, w]).astype(np.float32)


@needs_ref
def test_writer_reproduces_the_reference_files(tmp_path):
    case = cases.small_case("out", dims=(33, 25, 23), split=(2, 1, 1), nsteps=2, noise_seed=4)
    cdir = str(tmp_path / "case")
    case.write_reference_inputs(cdir)
    os.makedirs(tmp_path / "ref", exist_ok=True)
    subprocess.run([refio.REF_HARNESS, cdir, "2", str(tmp_path / "ref"), "--vts", str(tmp_path / "refout" / "flow")],
                   check=True, capture_output=True)
    state = refio.read_state(str(tmp_path / "ref" / "final.bin"))
    snap = []
    for b, blk in zip(case.blocks, state["blocks"]):
        xyz = np.stack([b.x.ravel(), b.y.ravel(), b.z.ravel()], axis=1).astype(np.float32)
        snap.append((b.dims, xyz, _fields_from_prim(blk["prim"], case.params.gamma)))
    ours = output._write(snap, str(tmp_path / "ours" / "flow"), 2)
    assert [os.path.basename(p) for p in ours] == ["flow_000002_block_0.vts", "flow_000002_block_1.vts",
                                                    "flow_000002.vtm"]
    for p in ours:
        ref = tmp_path / "refout" / os.path.basename(p)
        assert open(p, "rb").read() == open(ref, "rb").read(), os.path.basename(p)
