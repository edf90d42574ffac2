"""Run steps of one benchmark configuration on cuda:0 and report its throughput (also the
target command for ncu captures).

    python -m wmles_jax_b200.profile_case --config 2 --n 128 128 128 --steps 3 --precision fp64
    python -m wmles_jax_b200.profile_case --config 3 --steps 500 --precision mixed
    python -m wmles_jax_b200.profile_case --config 4 --steps 500 --precision fp64 --breakdown

config 2: periodic channel (KEP4 + WALE + wall model + constant mass flux), size --n
(default 256 128 128);
config 3: smooth ramp (Hybrid + Vreman + wall model + synthetic inflow + sponge), size --n
(default 384 96 64); config 4: NACA 0012 four-block C-grid (Hybrid + Vreman + wall model
+ far field), cell counts divided by --scale.  Steps go through ``Solver.step`` with the
time advanced by the returned dt, as the reference's drivers do.  --breakdown times every
launch with CUDA events and prints the device time per kernel kind.
"""
import argparse
import json
import time

import numpy as np
import torch

from . import _native as N
from .solver import Solver
from .workloads import channel_case, naca_case, ramp_case


def build(config, n=None, scale=1):
    if config == 2:
        return channel_case(2, n=tuple(n) if n else (256, 128, 128), device=True)
    if config == 3:
        mesh, gas, kw, prim, _ = ramp_case(tuple(n) if n else (384, 96, 64), device=True)
        return mesh, gas, kw, prim
    if config == 4:
        return naca_case(scale=scale, device=True)
    raise ValueError(f"unknown config {config}")


def run(config, precision, steps, n=None, scale=1, tile=None, chunk=None, breakdown=False, warmup=2):
    mesh, gas, kw, prim = build(config, n, scale)
    s = Solver(mesh, gas, **kw, precision=precision, tile=tile, chunk=chunk)
    Q = s.init_state(prim)
    t = 0.0
    for _ in range(warmup):
        Q, dt = s.step(Q, t)
        t += float(dt)
    torch.cuda.synchronize()
    s.profile(enable=breakdown)
    t0 = time.perf_counter()
    for _ in range(steps):
        Q, dt = s.step(Q, t)
        t += float(dt)
    torch.cuda.synchronize()
    el = (time.perf_counter() - t0) / steps
    cells = sum(int(np.prod(b.n)) for b in mesh.blocks)
    out = {"config": config, "precision": precision, "blocks": [list(b.n) for b in mesh.blocks], "cells": cells,
           "steps": steps, "ms_per_step": el * 1e3, "mcell_steps_per_s": cells / el / 1e6, "time": t,
           "finite": all(bool(torch.isfinite(q).all()) for q in Q)}
    if breakdown:
        # "surface": ghost cells + wall-model overrides + sponge means, one launch per stage
        names = {N.KIND_STAGE: "stage", N.KIND_GHOST: "surface", N.KIND_WALL: "wall_stats", N.KIND_DT: "dt",
                 N.KIND_SOURCE: "inflow"}
        out["device_ms_per_step"] = {names[k]: s.profile_read(k)[0] / steps for k in names}
        out["launches_per_step"] = s.profile_read(-1)[1] / steps
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, choices=[2, 3, 4], default=2)
    ap.add_argument("--n", type=int, nargs=3, default=None)
    ap.add_argument("--scale", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--tile", default=None, help="tile id 0-3 or 'auto' (autotuned, cached)")
    ap.add_argument("--chunk", type=int, default=None)
    ap.add_argument("--breakdown", action="store_true")
    a = ap.parse_args()
    tile = a.tile if a.tile in (None, "auto") else int(a.tile)
    print(json.dumps(run(a.config, a.precision, a.steps, a.n, a.scale, tile, a.chunk, a.breakdown)), flush=True)


if __name__ == "__main__":
    main()
