"""Generates the golden fixtures of this directory by running the reference
solver (compiled from its own sources into oracle/_ref by oracle/Makefile) on
small seeded cases.

    make -C oracle ref && python tests/golden/gen_golden.py [fixture ...]

With no arguments it regenerates the small fixtures; the configuration
horizons (c0_200, c1_25: minutes of reference CPU time) are made only when
named.

Each fixture holds the case recipe, the reference's residual history
(rms, max, max location, phydtime per step) and its final primitive state:
the full interior state for a single-block case, every 7th interior point
(flattened, blocks in order) for a multi-block case to keep the file small.
"""
from __future__ import annotations

import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import refio  # noqa: E402
from orion_b200 import cases  # noqa: E402

NG = 3

RECIPES = {
    "small_1blk": dict(name="small_1blk", dims=(17, 13, 12), split=(1, 1, 1), nsteps=20, noise_seed=11),
    "small_8blk": dict(name="small_8blk", dims=(33, 25, 23), split=(2, 2, 2), nsteps=10, noise_seed=12),
    "small_uneven": dict(name="small_uneven", dims=(41, 27, 25), split=(3, 2, 2), nsteps=8, noise_seed=13,
                         uneven_seed=5, moo=0.7, reynolds=1.0e4),
    # freestream (imin) and extrapolation (imax, kmax) faces, isothermal walls, 3 degrees of attack
    "small_bcmix": dict(name="small_bcmix", dims=(33, 25, 23), split=(2, 1, 1), nsteps=8, noise_seed=14,
                        twall=300.0, attack=3.0, physical={"imin": cases.BC_FREESTREAM, "imax": cases.BC_EXTRAPOLATION,
                                                           "kmax": cases.BC_EXTRAPOLATION}),
    # Euler: slip walls, no viscous stage; method 0
    "small_euler": dict(name="small_euler", dims=(33, 25, 23), split=(1, 2, 1), nsteps=8, noise_seed=15,
                        nvis=0, method=0),
}


def build(recipe: dict) -> cases.Case:
    r = dict(recipe)
    return cases.small_case(**r)


def interior_prim(state, sub: int = 1) -> np.ndarray:
    parts = []
    for b in state["blocks"]:
        p = b["prim"][:5, NG:-NG, NG:-NG, NG:-NG]
        parts.append(p.reshape(5, -1))
    flat = np.concatenate(parts, axis=1)
    return flat[:, ::sub]


# The benchmark configurations at their own horizons (cases.config):
#   c0_200: config 0 (one block 97x49x33) for its 200 steps;
#   c1_25:  config 1 (eight blocks 193x97x65, split 2x2x2) for 25 steps, and the
#           reference's residual history over its 300 steps (hist_long), which
#           records where the reference's own scheme leaves convergence on this
#           split.
# The state is stored sub-sampled, with per-variable sums and sums of squares
# of the whole interior state beside it.
HORIZONS = {
    "c0_200": dict(config=0, nsteps=200, sub=37, long_steps=0),
    "c1_25": dict(config=1, nsteps=25, sub=211, long_steps=300),
}


def state_sums(flat: np.ndarray) -> np.ndarray:
    """Per-variable sum and sum of squares of the interior state (5 x 2)."""
    return np.stack([flat.sum(axis=1), (flat * flat).sum(axis=1)], axis=1)


def horizon(key: str, spec: dict) -> None:
    case = cases.config(spec["config"], nsteps=spec["nsteps"])
    tmp = tempfile.mkdtemp(prefix="golden_")
    cdir = os.path.join(tmp, "case")
    case.write_reference_inputs(cdir)
    refio.run_reference(cdir, case.nsteps, os.path.join(tmp, "out"))
    hist = refio.read_hist(os.path.join(tmp, "out", "hist.bin"))
    final = refio.read_state(os.path.join(tmp, "out", "final.bin"))
    flat = interior_prim(final, 1)
    extra = {}
    if spec["long_steps"]:
        refio.run_reference(cdir, spec["long_steps"], os.path.join(tmp, "long"), time_only=True)
        extra["hist_long"] = refio.read_hist(os.path.join(tmp, "long", "hist.bin"))
    np.savez_compressed(os.path.join(HERE, key + ".npz"), hist=hist, prim=flat[:, ::spec["sub"]],
                        sums=state_sums(flat), sub=np.array([spec["sub"]]),
                        recipe=np.array([json.dumps(spec)]), **extra)
    print(key, case.npoints, "points", case.nsteps, "steps", hist[-1, :2])


# Two requests of the seeded serving stream (serving.c4_requests(24, seed=4))
# whose flows diverge: the reference's residual history over 200 steps.
DIVERGING = {"c4_diverging": dict(requests=24, seed=4, rids=(1, 18), steps=200)}


def diverging(key: str, spec: dict) -> None:
    from orion_b200 import serving

    reqs = serving.c4_requests(spec["requests"], seed=spec["seed"], mean_ms=50.0, max_steps=spec["steps"])
    hists = []
    for rid in spec["rids"]:
        case = reqs[rid].build_case()
        case.nsteps = spec["steps"]
        tmp = tempfile.mkdtemp(prefix="golden_")
        cdir = os.path.join(tmp, "case")
        case.write_reference_inputs(cdir)
        refio.run_reference(cdir, spec["steps"], os.path.join(tmp, "out"), time_only=True)
        hists.append(refio.read_hist(os.path.join(tmp, "out", "hist.bin")))
        print(key, rid, case.npoints, "points", hists[-1][[0, -1], 0])
    np.savez_compressed(os.path.join(HERE, key + ".npz"), hist=np.stack(hists), recipe=np.array([json.dumps(spec)]))


def main(keys=None):
    for key, spec in HORIZONS.items():
        if keys and key in keys:
            horizon(key, spec)
    for key, spec in DIVERGING.items():
        if keys and key in keys:
            diverging(key, spec)
    for key, recipe in RECIPES.items():
        if keys and key not in keys:
            continue
        case = build(recipe)
        tmp = tempfile.mkdtemp(prefix="golden_")
        case.write_reference_inputs(os.path.join(tmp, "case"))
        refio.run_reference(os.path.join(tmp, "case"), case.nsteps, os.path.join(tmp, "out"))
        hist = refio.read_hist(os.path.join(tmp, "out", "hist.bin"))
        final = refio.read_state(os.path.join(tmp, "out", "final.bin"))
        sub = 1 if len(case.blocks) == 1 else 7
        np.savez_compressed(os.path.join(HERE, key + ".npz"), hist=hist, prim=interior_prim(final, sub),
                            sub=np.array([sub]), recipe=np.array([json.dumps(recipe)]))
        print(key, case.npoints, "points", case.nsteps, "steps", hist[-1, :2])


if __name__ == "__main__":
    main(sys.argv[1:])
