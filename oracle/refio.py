"""Readers for the oracle driver's output files.  TEST INFRASTRUCTURE ONLY.

State files (init.bin, final.bin, snap_<step>_<stage>.bin) hold, per block,
the padded i-fastest arrays of the reference's BlockField
(src/preprocess/FlowField.hpp:19-71): prim(6) q(5) dq(5) metrics(9) vol dt c mu
spec_radius(3) spec_radius_visc(3).  hist.bin holds per step
(rms, max, loc[5], phydtime) as written by ResidualMonitor::compute
(src/solver/ResidualMonitor.cpp:11-137) and TimeIntegrator (phydtime).
"""
from __future__ import annotations

import os
import subprocess
from typing import Dict, List

import numpy as np

FIELDS = (("prim", 6), ("q", 5), ("dq", 5), ("metrics", 9), ("vol", 1), ("dt", 1),
          ("c", 1), ("mu", 1), ("spec", 3), ("specv", 3))

HERE = os.path.dirname(os.path.abspath(__file__))


def ref_root() -> str:
    """The reference's source tree (read-only): $ORION_REF, else a directory
    `reference` beside the repository, the default of oracle/Makefile (the
    recipe compiling it).  Only CPU-side checks read it directly; a machine
    without the source tree (a GPU box) uses the prebuilt oracle/_ref."""
    env = os.environ.get("ORION_REF")
    if env:
        return env
    return os.path.normpath(os.path.join(HERE, "..", "..", "reference"))


REF_ROOT = ref_root()
REF_HARNESS = os.path.join(HERE, "_ref", "orion_ref_harness")
# The same driver source linked against the B200 path through the C++ drop-in
# layer (make -C oracle shim); it is the product under test, not the oracle.
SHIM_HARNESS = os.path.join(HERE, "_ref", "orion_shim_harness")


def read_state(path: str) -> Dict:
    with open(path, "rb") as f:
        raw = f.read()
    assert raw[:8] == b"ORSTATE1", path
    nb, ng, _ = np.frombuffer(raw, dtype="<i4", count=3, offset=8)
    phydtime = float(np.frombuffer(raw, dtype="<f8", count=1, offset=20)[0])
    off = 28
    dims = []
    for _ in range(nb):
        dims.append(tuple(int(v) for v in np.frombuffer(raw, dtype="<i4", count=3, offset=off)))
        off += 12
    blocks: List[Dict[str, np.ndarray]] = []
    for (nx, ny, nz) in dims:
        n = nx * ny * nz
        blk = {}
        for name, nc in FIELDS:
            a = np.frombuffer(raw, dtype="<f8", count=n * nc, offset=off).reshape(nc, nz, ny, nx)
            off += 8 * n * nc
            blk[name] = a[0] if nc == 1 else a
        blocks.append(blk)
    return {"ng": int(ng), "phydtime": phydtime, "dims": dims, "blocks": blocks}


def read_hist(path: str) -> np.ndarray:
    with open(path, "rb") as f:
        raw = f.read()
    n = int(np.frombuffer(raw, dtype="<i4", count=1)[0])
    return np.frombuffer(raw, dtype="<f8", offset=4).reshape(n, 8)


def run_reference(case_dir: str, nsteps: int, out_dir: str, snap_step: int = -1,
                  time_only: bool = False) -> str:
    os.makedirs(out_dir, exist_ok=True)
    cmd = [REF_HARNESS, case_dir, str(nsteps), out_dir]
    if snap_step >= 0:
        cmd += ["--snap-step", str(snap_step)]
    if time_only:
        cmd += ["--time-only"]
    r = subprocess.run(cmd, check=True, capture_output=True, text=True)
    return r.stdout


def reference_available() -> bool:
    return os.path.exists(REF_HARNESS)


def run_shim(case_dir: str, nsteps: int, out_dir: str, extra=()) -> str:
    os.makedirs(out_dir, exist_ok=True)
    r = subprocess.run([SHIM_HARNESS, case_dir, str(nsteps), out_dir, *extra], check=True, capture_output=True,
                       text=True)
    return r.stdout


def shim_available() -> bool:
    return os.path.exists(SHIM_HARNESS)
