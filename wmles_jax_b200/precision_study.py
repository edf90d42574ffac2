"""Error of the mixed-precision form against the FP64 form on the same inputs.

    python -m wmles_jax_b200.precision_study --config 2 --steps 1000

Both forms start from the same initial state and advance ``steps`` steps, each with its own
CFL time step (the drivers' loop).  Reported, per result the mixed form is evaluated on:

* state: relative L2 difference of every conservative variable after the last step;
* mean velocity profile: the velocity averaged over the homogeneous directions (x and z
  for the channel, the span for the ramp and the airfoil), max-norm difference relative
  to the FP64 profile's max norm;
* wall shear: tau_w of every wall-modelled face, averaged the same way, max-norm relative
  difference; plus the relative L2 difference of the instantaneous tau_w field;
* dt: relative difference of the last CFL time step.

With ``--perturb eps`` the same metrics are also given for two FP64 runs whose initial
states differ by a relative N(0, eps) perturbation (eps ~ 1e-7, FP32 round-off): in an
unsteady flow that separation grows with time whatever the arithmetic, and it bounds what
any reduced-precision form can achieve at that step count.

The averages are measurement code over the device states (torch reductions), not part of
the solver.
"""
import argparse
import json

import numpy as np
import torch

from .solver import Solver
from .profile_case import build

HOMOGENEOUS = {2: (0, 2), 3: (2,), 4: (2,)}     # interior axes averaged over, per config


def _advance(mesh, gas, kw, q0, precision, steps):
    s = Solver(mesh, gas, **kw, precision=precision)
    Q = tuple(q.clone() for q in q0)
    t = 0.0
    for _ in range(steps):
        Q, dt = s.step(Q, t)
        t += float(dt)
    return s, Q, s.max_dt(Q)


def _rel(a, b):
    return float(torch.linalg.norm(a - b) / torch.linalg.norm(b))


def _rel_inf(a, b):
    return float((a - b).abs().max() / b.abs().max())


def compare(config=2, steps=1000, n=None, scale=1, perturb=0.0):
    """Metrics of mixed vs FP64; with perturb > 0 also those of FP64 from the initial state
    multiplied by (1 + perturb * N(0, 1)) vs FP64 (how far two FP64 runs drift apart from a
    relative input difference of the size of FP32 round-off: the problem's own sensitivity)."""
    mesh, gas, kw, prim = build(config, n, scale)
    dev = torch.device("cuda", torch.cuda.current_device())
    q0 = tuple(torch.from_numpy(np.ascontiguousarray(gas.prim_to_cons(np.asarray(prim(g.xc), float)))).to(dev)
               for g in mesh.geoms)
    s64, Q64, dt64 = _advance(mesh, gas, kw, q0, "fp64", steps)
    s32, Q32, dt32 = _advance(mesh, gas, kw, q0, "mixed", steps)
    out = {"config": config, "steps": steps, "cells": sum(int(np.prod(b.n)) for b in mesh.blocks)}
    out.update(_metrics(config, mesh, s64, Q64, dt64, s32, Q32, dt32))
    if perturb > 0:
        g = torch.Generator(device=dev).manual_seed(1)
        qp = tuple(q * (1.0 + perturb * torch.randn(q.shape, generator=g, device=dev, dtype=q.dtype)) for q in q0)
        sp, Qp, dtp = _advance(mesh, gas, kw, qp, "fp64", steps)
        out["fp64_input_perturbation"] = perturb
        out["fp64_perturbed_vs_fp64"] = _metrics(config, mesh, s64, Q64, dt64, sp, Qp, dtp)
    return out


def _metrics(config, mesh, s64, Q64, dt64, s32, Q32, dt32):
    axes = tuple(1 + a for a in HOMOGENEOUS[config])
    out = {"finite": all(bool(torch.isfinite(q).all()) for q in Q64 + Q32)}
    state, prof = [], []
    for blk, a, b in zip(mesh.blocks, Q32, Q64):
        ia, ib = blk.interior(a), blk.interior(b)
        state.append([_rel(ia[c], ib[c]) for c in range(5)])
        ua, ub = ia[1:4] / ia[0:1], ib[1:4] / ib[0:1]
        prof.append(_rel_inf(ua.mean(dim=axes), ub.mean(dim=axes)))
    out["state_rel_l2"] = [max(s[c] for s in state) for c in range(5)]
    out["mean_velocity_rel_inf"] = max(prof)
    t32, t64 = s32.wall_stats(Q32), s64.wall_stats(Q64)
    tau_mean, tau_l2 = [], []
    for key, (ta, _) in t32.items():
        tb = t64[key][0]
        ta, tb = torch.from_numpy(np.asarray(ta)), torch.from_numpy(np.asarray(tb))
        ib, a, s_, bc = next(w for w in s64.walls if (mesh.blocks[w[0]].name, "ijk"[w[1]] + ("min", "max")[w[2]]) == key)
        tang = [d for d in range(3) if d != a]
        hom = tuple(i for i, d in enumerate(tang) if d in HOMOGENEOUS[config])
        tau_mean.append(_rel_inf(ta.mean(dim=hom) if hom else ta, tb.mean(dim=hom) if hom else tb))
        tau_l2.append(_rel(ta, tb))
    out["wall_shear_mean_rel_inf"] = max(tau_mean) if tau_mean else None
    out["wall_shear_field_rel_l2"] = max(tau_l2) if tau_l2 else None
    out["dt_rel"] = abs(float(dt32) - float(dt64)) / float(dt64)
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--config", type=int, choices=[2, 3, 4], default=2)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--n", type=int, nargs=3, default=None)
    ap.add_argument("--scale", type=int, default=1)
    ap.add_argument("--perturb", type=float, default=0.0)
    a = ap.parse_args()
    print(json.dumps(compare(a.config, a.steps, a.n, a.scale, a.perturb)), flush=True)


if __name__ == "__main__":
    main()
