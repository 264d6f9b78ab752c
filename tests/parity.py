"""Parity helpers: run the reference oracle on a case and compare GPU stages
with the reference's per-stage snapshots."""
from __future__ import annotations

import os
import sys
import tempfile
from typing import Dict, List, Tuple

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import refio  # noqa: E402

from orion_b200 import cases  # noqa: E402

NG = 3
STAGES = ["pre", "exchange", "bc", "state", "dt", "visc", "avg1", "inv", "avg2", "update"]


def rel_err(a: np.ndarray, b: np.ndarray) -> float:
    """max |a-b| / max(max|b|, 1e-300)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(float(np.max(np.abs(b))) if b.size else 0.0, 1e-300)
    return float(np.max(np.abs(a - b))) / scale if a.size else 0.0


def interior(a: np.ndarray) -> np.ndarray:
    return a[..., NG:-NG, NG:-NG, NG:-NG]


def run_reference_case(case: cases.Case, nsteps: int, snap_step: int = -1, workdir: str = None) -> Tuple[str, str]:
    workdir = workdir or tempfile.mkdtemp(prefix="orion_ref_")
    cdir = os.path.join(workdir, "case")
    odir = os.path.join(workdir, "out")
    case.write_reference_inputs(cdir)
    refio.run_reference(cdir, nsteps, odir, snap_step=snap_step)
    return cdir, odir


def compare_state(fs, state: Dict, fields, region="all") -> Dict[str, float]:
    """Max relative error per field over all blocks (region: all | interior)."""
    out = {}
    for f in fields:
        errs = []
        for n, blk in enumerate(state["blocks"]):
            g = fs.download(n, f)
            r = blk[f]
            if region == "interior":
                g, r = interior(g), interior(r)
            errs.append(rel_err(g, r))
        out[f] = max(errs)
    return out
