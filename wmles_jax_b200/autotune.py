"""Tile-shape autotuner for the fused stage kernel.

The stage kernel marches a TJ x TK column of cells along i (tile ids: 0 = 8x32, 1 = 16x16,
2 = 4x32, 3 = 16x32, the last built for the mixed form only).  Which shape is fastest depends
on the grid extents (partial tiles at the j/k edges, waves of CTAs over the SMs), on the
precision (registers and shared memory decide CTAs per SM) and on the scheme.  ``tune``
measures it: for each candidate tile it builds the cases with that tile, advances them
together (one batched step, as the server runs them) and times the steps with CUDA events;
the fastest tile is stored in a JSON cache keyed by GPU name, precision, scheme, SGS model
and the block extents of the workload, so each workload is tuned once per machine.

The tile shape does not change the physics; it does change the summation order of the
stage-3 mass-flux partials, so results with different tiles agree to round-off, not bitwise.
A server therefore fixes one tile for all its cases (``Server(tile="auto")`` tunes it over
its grid mix before serving).
"""
import copy
import json
import os
import threading

import numpy as np

TILE_SHAPES = {0: (8, 32), 1: (16, 16), 2: (4, 32), 3: (16, 32)}
CANDIDATES = {"fp64": (0, 1, 2), "mixed": (0, 1, 2, 3)}
_LOCK = threading.Lock()


def cache_path():
    """Cache file: $WMLES_TUNE_CACHE, else ~/.cache/wmles_jax_b200/tiles.json."""
    p = os.environ.get("WMLES_TUNE_CACHE")
    if p:
        return p
    return os.path.join(os.path.expanduser("~"), ".cache", "wmles_jax_b200", "tiles.json")


def workload_key(dims, precision, scheme, sgs, device_name):
    """Cache key of a workload: the sorted multiset of block extents plus the options."""
    ext = sorted("x".join(str(int(n)) for n in d) for d in dims)
    return f"{device_name}|{precision}|{scheme}|{sgs}|{','.join(ext)}"


def load_cache(path=None):
    path = path or cache_path()
    try:
        with open(path) as f:
            data = json.load(f)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def store(key, entry, path=None):
    path = path or cache_path()
    with _LOCK:
        data = load_cache(path)
        data[key] = entry
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        tmp = f"{path}.{os.getpid()}.tmp"
        with open(tmp, "w") as f:
            json.dump(data, f, indent=1, sort_keys=True)
        os.replace(tmp, path)


def pick(timings):
    """Fastest tile of {tile: ms per step} (ties: the lower id)."""
    return min(sorted(timings), key=lambda t: timings[t])


def _scheme_name(scheme):
    from .schemes import KEP, MUSCLHLLC, Hybrid
    if isinstance(scheme, KEP):
        return f"KEP{scheme.order}"
    if isinstance(scheme, MUSCLHLLC):
        return f"MUSCLHLLC-{scheme.limiter}"
    if isinstance(scheme, Hybrid):
        return f"Hybrid-KEP{scheme.c.order}"
    return type(scheme).__name__


def key_for(cases, precision):
    """Cache key of a list of (mesh, gas, kw, prim) cases."""
    import torch
    from .sgs import make_sgs
    mesh0, _, kw0, _ = cases[0]
    dims = [tuple(b.n) for mesh, _, _, _ in cases for b in mesh.blocks]
    sgs = make_sgs(kw0.get("sgs", "vreman"), **(kw0.get("sgs_kwargs") or {})).name
    return workload_key(dims, precision, _scheme_name(kw0["scheme"]), sgs, torch.cuda.get_device_name())


def tune(cases, precision="mixed", tiles=None, steps=20, warmup=3, use_cache=True, path=None):
    """Fastest stage-kernel tile for advancing ``cases`` (a list of (mesh, gas, kw, prim)
    with prim=None for a uniform state) together.  Returns (tile, {tile: ms per step})."""
    import torch
    from .solver import Solver
    from .serving import Batch
    key = key_for(cases, precision)
    if use_cache:
        hit = load_cache(path).get(key)
        if hit is not None:
            return int(hit["tile"]), {int(k): v for k, v in hit["ms_per_step"].items()}
    tiles = CANDIDATES[precision] if tiles is None else tuple(tiles)
    # host lowering and initial states once; device cases per tile
    prepared, q0 = [], []
    for mesh, gas, kw, prim in cases:
        s = Solver.__new__(Solver)
        s._prepare(mesh, gas, precision=precision, **kw)
        prepared.append(s)
        if prim is None:
            prim = _uniform_prim(gas)
        q0.append([np.ascontiguousarray(gas.prim_to_cons(np.asarray(prim(g.xc), float))) for g in s.host_geoms])
    timings = {}
    for tile in tiles:
        solvers = []
        for s in prepared:
            t = copy.copy(s)
            t._desc.tile = int(tile)
            t._create(release=False)
            solvers.append(t)
        qa = [tuple(torch.from_numpy(q).cuda() for q in Q) for Q in q0]
        qb = [tuple(torch.empty_like(x) for x in Q) for Q in qa]
        da = [s.max_dt(Q) for s, Q in zip(solvers, qa)]
        db = [torch.empty_like(d) for d in da]
        batch = Batch(solvers)
        bufs, dts = [qa, qb], [da, db]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for k in range(warmup + steps):
            if k == warmup:
                e0.record()
            p = k % 2
            batch.step(bufs[p], bufs[1 - p], dts[p], dts[1 - p])
        e1.record()
        torch.cuda.synchronize()
        timings[int(tile)] = e0.elapsed_time(e1) / steps
        batch.close()
        del solvers, bufs, dts, qa, qb
    best = pick(timings)
    if use_cache:
        store(key, {"tile": best, "tile_shape": list(TILE_SHAPES[best]),
                    "ms_per_step": {str(k): v for k, v in timings.items()}, "steps": steps}, path)
    return best, timings


def _uniform_prim(gas):
    """A uniform state (rho = 1, T = 1, u = 0.3 c) for timing when no initial condition is given."""
    c = float(np.sqrt(gas.gamma * gas.R))

    def prim(xc):
        one = np.ones_like(xc[0])
        return np.stack([one, 0.3 * c * one, 0 * one, 0 * one, gas.R * one])
    return prim
