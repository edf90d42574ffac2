"""Run a few steps of a channel workload on cuda:0 (target for ncu captures).

    python -m wmles_jax_b200.profile_case --n 128 128 128 --steps 3 --precision fp64

Builds the config-2 channel physics (KEP4 + WALE + wall model + constant mass flux) at
the requested size, runs ``--steps`` steps through ``Solver.step`` and prints the wall
time per step.  Each step launches, in order: dt (1), then per RK stage ghost gather,
wall model, stage kernel (3 x 3), then the constraint pass (1).
"""
import argparse
import time

import numpy as np
import torch

from .solver import Solver
from .workloads import channel_case


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, nargs=3, default=(128, 128, 128))
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--precision", choices=["fp64", "mixed"], default="fp64")
    ap.add_argument("--tile", type=int, default=None)
    ap.add_argument("--chunk", type=int, default=None)
    a = ap.parse_args()
    mesh, gas, kw, prim = channel_case(2, n=tuple(a.n))
    s = Solver(mesh, gas, **kw, precision=a.precision, tile=a.tile, chunk=a.chunk)
    Q = s.init_state(prim)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        Q, dt = s.step(Q)
    torch.cuda.synchronize()
    el = (time.perf_counter() - t0) / a.steps
    cells = int(np.prod(a.n))
    print(f"{a.precision} n={tuple(a.n)}: {el * 1e3:.3f} ms/step (wall), {cells / el / 1e6:.1f} Mcell-steps/s, "
          f"dt={float(dt):.4e}")


if __name__ == "__main__":
    main()
