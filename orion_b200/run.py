"""Runs one synthetic configuration through the C ABI and prints its residual
history: the command-line counterpart of the reference's driver loop
(src/core/OrionSolver.cpp:139-209) for the bump-channel configurations.

    python -m orion_b200.run --config 1 --steps 2 --warmup 1 --precision mixed
    python -m orion_b200.run --config 0 --steps 200 --every 20

Profilers wrap it (a launch list of a few steps, a one-kernel capture).
"""
from __future__ import annotations

import argparse
import json

from . import _lib, cases, solver


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=1)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "plain"])
    ap.add_argument("--small", action="store_true", help="a 2x2x2-block 97x65x49 case instead")
    ap.add_argument("--every", type=int, default=0, help="print every n-th step of the history (0: the last)")
    ap.add_argument("--time", action="store_true",
                    help="time the steps (CUDA events on the case's stream) and print cell-updates/s")
    ap.add_argument("--autotune", action="store_true",
                    help="autotune the schedule on the case first (the solution does not move) and print it")
    a = ap.parse_args()
    if a.small:
        case = cases.bump_case("profile_small", 97, 65, 49, split=(2, 2, 2), nsteps=a.steps)
    else:
        case = cases.config(a.config)
    prec = _lib.PREC_MIXED if a.precision == "mixed" else _lib.PREC_FP64
    fs = solver.FlowFieldSet(case, precision=prec)
    fs.step(a.warmup)
    if a.autotune:
        print(json.dumps({"case": case.name, "precision": a.precision, "autotune": fs.autotune(steps_per_trial=3)}))
    if a.time:
        import torch

        st = torch.cuda.ExternalStream(fs.stream_ptr())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fs.step_async(a.steps)
        e1.record(st)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / a.steps
        print(json.dumps({"case": case.name, "precision": a.precision, "points": case.npoints, "steps": a.steps,
                          "ms_per_step": ms, "cell_updates_per_s": case.npoints / (ms / 1e3),
                          "schedule": fs.sweep_schedule()}))
        fs.close()
        return
    h = fs.step(a.steps)
    if a.every > 0:
        for n in range(a.every - 1, a.steps, a.every):
            print(f"step {a.warmup + n + 1:6d}  rms {h[n, 0]:.6e}  max {h[n, 1]:.6e}")
    print(f"{case.name} {a.precision}: {a.steps} steps, rms {h[-1, 0]:.6e}")
    fs.close()


if __name__ == "__main__":
    main()
