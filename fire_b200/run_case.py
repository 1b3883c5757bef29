"""Runs one simulation for a few steps and prints its diagnostics and per-pass times.

    python -m fire_b200.run_case X Y Z [--steps N] [--jacobi auto|unblocked|zmarch|fused|resident]
                                       [--block K] [--zchunk ZC] [--pressure auto|warm_f32|f16|cold_f32]
                                       [--mixed] [--iters P R] [--profile] [--time N]
                                       [--staging auto|cpasync|tma] [--project auto|fused|separate]
                                       [--simulate-by 2|4|8]

A sphere emitter near the floor (radius X/9), seeded velocity noise and emission jitter,
dt = 1/60. Used as the command under profilers (one process, one GPU, small cases).
--time N then times N more steps as the engine runs them (graph replay) with CUDA events on
the simulation's stream and prints their mean as step_ms.
"""
from __future__ import annotations

import argparse
import json

from . import _abi as A
from .sim import FireXSim, make_options

PRESSURE = {"auto": A.PRESSURE_AUTO, "warm_f32": A.PRESSURE_WARM_F32, "f16": A.PRESSURE_F16,
            "cold_f32": A.PRESSURE_COLD_F32}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("dims", type=int, nargs=3)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--jacobi", default="auto")
    ap.add_argument("--block", type=int, default=0, help="fused sweeps per launch / resident variant + 1")
    ap.add_argument("--zchunk", type=int, default=0, help="z planes per CTA (0 = auto)")
    ap.add_argument("--pressure", default="warm_f32", choices=list(PRESSURE))
    ap.add_argument("--mixed", action="store_true")
    ap.add_argument("--iters", type=int, nargs=2, default=(96, 96))
    ap.add_argument("--profile", action="store_true", help="per-pass device times (no graph replay)")
    ap.add_argument("--time", type=int, default=0, help="then time this many steps (graph replay)")
    ap.add_argument("--staging", default="auto", choices=["auto", "cpasync", "tma"],
                    help="plane staging of the two-sweep pass (auto: cp.async)")
    ap.add_argument("--project", default="auto", choices=["auto", "fused", "separate"],
                    help="primary projection and residual divergence in one pass or two")
    ap.add_argument("--simulate-by", type=int, default=0, choices=[0, 2, 4, 8], help="source-pass brick height")
    a = ap.parse_args()
    X, Y, Z = a.dims
    opts = make_options(pressure_iterations=a.iters[0], correction_iterations=a.iters[1], seed=1, velocity_noise=0.05,
                        emission_jitter=0.1, pressure_mode=PRESSURE[a.pressure],
                        precision=A.PRECISION_MIXED if a.mixed else A.PRECISION_F32,
                        spheres=[dict(center=(X / 2, Y / 16, Z / 2), radius=X / 9)])
    s = FireXSim((X, Y, Z), opts)
    s.set_jacobi(a.jacobi, a.block, a.zchunk)
    s.set_staging({"auto": A.STAGING_AUTO, "cpasync": A.STAGING_CPASYNC, "tma": A.STAGING_TMA}[a.staging])
    s.set_tiles(a.simulate_by, {"auto": A.PROJECT_AUTO, "fused": A.PROJECT_FUSED, "separate": A.PROJECT_SEPARATE}[a.project])
    if a.profile:
        s.set_profiling(True)
        s.pass_times()
    s.step(a.steps, 1 / 60)
    s.sync()
    out = {"dims": [X, Y, Z], "steps": a.steps, "diagnostics": s.diagnostics}
    if a.profile:
        out["pass_ms"] = {k: v[0] / a.steps for k, v in s.pass_times().items()}
        s.set_profiling(False)
    if a.time > 0:
        import torch

        st = torch.cuda.ExternalStream(s.stream)
        s.step(1, 1 / 60)  # plan and graph for the unprofiled step
        s.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        s.step(a.time, 1 / 60)
        e1.record(st)
        s.sync()
        out["step_ms"] = e0.elapsed_time(e1) / a.time
    print(json.dumps(out))
    s.close()


if __name__ == "__main__":
    main()
