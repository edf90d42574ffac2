"""Benchmark of the wmles explicit RHS + SSP-RK3 step on B200 (Mcell-steps/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (config 2): periodic channel, one 256x128x128 block (4.19M cells), tanh
stretching beta=2.5, KEP4 + WALE 0.5, equilibrium wall model on both walls (3rd cell),
constant mass flux, CFL 0.5, Ma_b 0.3, Re_b 20000; seeded log-law IC + 10 % noise.
A step is the drivers' loop body: dt = max_dt(Q); Q = advance(Q, dt).

value       whole-job Mcell-steps/s, state resident in HBM, FP64 form, CUDA events, max over
            ranks (N > 1: one replica per GPU, weak scaling, no data-path collective)
e2e         the same step through the public Solver API with the state in pinned HOST
            memory: every step copies an independent host state in, steps, copies the new
            state and dt out (copies of consecutive steps overlapped with the step between
            them; the strictly serial loop's time is reported beside it)
mixed       the mixed-precision form (FP32 fluxes/gradients/SGS, FP64 state and reductions)
roofline    the fused stage kernel: algorithmic bytes per launch / mean launch time
cpu_baseline  the CPU oracle (NumPy float64 restatement of the reference) on a slab of the
            same workload, one core
serving     config 5: 64 seeded channel requests (Poisson arrivals at 20/s; uneven grids, Re_tau,
            Ma_b), mixed precision, 2000 steps each, continuously batched on one GPU: p50/p99
            time-to-result and aggregate Mcell-steps/s (--serving-requests 0 skips it)
--impl reference  the oracle on the host cores (one process per core, each on its own slab)
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Mcell-steps/s"
CONFIG_NAME = "channel 256x128x128, KEP4 + WALE + wall model + constant mass flux, SSP-RK3"
N_CFG2 = (256, 128, 128)
# DRAM bytes (read + write) per stage-kernel launch per interior cell, mean of the three RK
# stages, from one ncu capture of the same kernel on a 128^3 case of this workload; scaled
# by the cell count for the roofline's `traffic`
TRAFFIC_PER_CELL = {"fp64": 327.0, "mixed": 229.0}
# FP64 work per interior cell per stage-kernel launch (FP64 form, mean of the three RK
# stages), from one ncu capture of the same kernel on a 128^3 case of this workload: DADD 277.8,
# DMUL 329.5, DFMA 357.0 thread instructions, i.e. 1321 flop (an FMA counts two) in 964
# FP64-pipe instructions
FP64_FLOP_PER_CELL = 1321.0
FP64_INST_PER_CELL = 964.0
# nominal FP64 rate of a B200: 148 SMs x 64 FP64 lanes x 1.965 GHz (x 2 flop per FMA)
FP64_PEAK_INST = 148 * 64 * 1.965e9
FP64_PEAK_TFLOPS = 2 * FP64_PEAK_INST / 1e12


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)["hbm_gbs"], "measured"
    return 6650.0, "fallback"


def config_dict(extra=None):
    d = {"workload": CONFIG_NAME, "cells": int(np.prod(N_CFG2)), "grid": list(N_CFG2), "ghost_layers": 3,
         "scheme": "KEP4", "sgs": "WALE Cw=0.5", "wall_model": "equilibrium (Spalding/Kader), n_match=3",
         "constraint": "constant mass flux", "cfl": 0.5, "l2": "inputs larger than L2 (state 188 MB + metrics 527 MB)"}
    if extra:
        d.update(extra)
    return d


class ClockSampler:
    """nvidia-smi clock/throttle samples during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.proc = index, None

    def __enter__(self):
        self.lines = []
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.5)                              # let the sampler start
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except (ValueError, IndexError):
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------- ranks
def rank_barrier(dist):
    """Barrier over the job's ranks (no-op for one process)."""
    if dist is not None:
        dist.barrier()


def reduce_max(x, dist, device=None):
    """Max of a per-rank float over all ranks (identity for one process): the job's time is
    the slowest rank's."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_value(cells_per_rank, world, ms_per_step_max):
    """Aggregate Mcell-steps/s of N replicas (weak scaling): every rank advances its own copy
    of the workload, the job's step time is the slowest rank's."""
    return cells_per_rank * world / (ms_per_step_max * 1e-3) / 1e6


# ----------------------------------------------------------------------------- our arm
def run_ours(args, rank, world, local_rank):
    import torch
    from wmles_jax_b200 import Solver, _native
    from wmles_jax_b200.workloads import channel_case, STAGE_BYTES, STEP_BYTES, CMF_BYTES

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    def barrier():
        rank_barrier(dist)

    def max_over_ranks(x):
        return reduce_max(x, dist, dev)

    mesh, gas, kw, prim = channel_case(2, n=N_CFG2, device=True)
    cells = int(np.prod(mesh.blocks[0].n))
    Q0h = [np.ascontiguousarray(gas.prim_to_cons(np.asarray(prim(g.xc), float))) for g in mesh.geoms]
    K, Wm = args.steps, args.warmup

    def timed(solver, Q, profile=False):
        with ClockSampler(local_rank) as clk:          # sampling covers warm-up + timed steps
            for _ in range(Wm):
                Q, _ = solver.step(Q)
            torch.cuda.synchronize()
            barrier()
            torch.cuda.synchronize()
            solver.profile(enable=profile)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(K):
                Q, dt = solver.step(Q)
            e1.record()
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        barrier()
        return Q, ms, clk

    def kernel_split(solver, Q, n):
        """Mean device time of one launch of each kernel kind over n more steps, CUDA events
        around every launch (a separate pass: the event pairs are not in the timed steps)."""
        solver.profile(enable=True)
        for _ in range(n):
            Q, _ = solver.step(Q)
        torch.cuda.synchronize()
        split = {}
        for kind, name in ((_native.KIND_STAGE, "stage"), (_native.KIND_GHOST, "surface"), (_native.KIND_DT, "dt")):
            ms, cnt = solver.profile_read(kind)
            split[name] = dict(ms_per_launch=ms / max(cnt, 1), launches=cnt)
        solver.profile(enable=False)
        return Q, split

    out = {}
    s64 = Solver(mesh, gas, **kw)
    Q = tuple(torch.from_numpy(q).to(dev) for q in Q0h)
    Q64, ms64, clk = timed(s64, Q, profile=False)       # launch counts kept, no event pairs
    all_ms, all_n = s64.profile_read(-1)
    ms64_max = max_over_ranks(ms64)
    Q64, split64 = kernel_split(s64, Q64, min(K, 20))
    out["fp64"] = dict(ms=ms64_max / K, stage_ms=split64["stage"]["ms_per_launch"], launches=all_n,
                       clk=clk.summary(), split=split64)

    # mixed precision form (same workload and IC)
    s32 = Solver(mesh, gas, **kw, precision="mixed")
    Q = tuple(torch.from_numpy(q).to(dev) for q in Q0h)
    Q32, ms32, clk32 = timed(s32, Q, profile=False)
    ms32_max = max_over_ranks(ms32)
    Q32, split32 = kernel_split(s32, Q32, min(K, 20))
    st32_ms, st32_n = split32["stage"]["ms_per_launch"], 1
    err = []
    for c in range(5):
        a = mesh.blocks[0].interior(Q32[0][c]).double()
        b = mesh.blocks[0].interior(Q64[0][c]).double()
        err.append(float(torch.linalg.norm(a - b) / torch.linalg.norm(b)))
    out["mixed"] = dict(ms=ms32_max / K, stage_ms=st32_ms / max(st32_n, 1), err=max(err), clk=clk32.summary(),
                        split=split32)

    # end to end through the public API with host buffers.  Each step takes an independent
    # host state (two pinned input buffers, alternating), and its new state goes back to a
    # pinned host buffer; the host reads every step's dt.  Pipelined: the copy-in of step k+1
    # (copy stream) runs during step k, the copy-out of step k (second copy stream) during
    # step k+1, device inputs double-buffered; every copy is inside the timed region.  The
    # state copy-out of a step is enqueued after the host has read its dt: device-to-host
    # copies share a copy engine, and the 8-byte dt read must not wait behind 188 MB.  The
    # same loop run strictly in order (copy in, step, copy out, dt) is reported beside it.
    s64.profile(enable=False)                              # the public path, no event pairs
    pin_in = [[torch.from_numpy(q).pin_memory() for q in Q0h] for _ in range(2)]
    pin_out = [[torch.empty_like(p).pin_memory() for p in pin_in[0]] for _ in range(2)]
    dbuf = [[torch.empty_like(p, device=dev) for p in pin_in[0]] for _ in range(2)]
    h2d = sum(p.numel() * 8 for p in pin_in[0])
    d2h = h2d + 8
    comp = torch.cuda.current_stream()
    s_in, s_out = torch.cuda.Stream(), torch.cuda.Stream()
    ev_in = [torch.cuda.Event() for _ in range(2)]
    ev_used = [torch.cuda.Event() for _ in range(2)]

    def copy_in(k):
        b = k % 2
        s_in.wait_event(ev_used[b])                       # the step that last read dbuf[b] is done
        with torch.cuda.stream(s_in):
            for d, p in zip(dbuf[b], pin_in[b]):
                d.copy_(p, non_blocking=True)
        ev_in[b].record(s_in)

    def pipelined(n):
        s_in.wait_stream(comp)
        copy_in(0)
        for k in range(n):
            b = k % 2
            comp.wait_event(ev_in[b])
            Qn, dt = s64.step(tuple(dbuf[b]))
            ev_used[b].record(comp)
            if k + 1 < n:
                copy_in(k + 1)                            # enqueued before the blocking dt read
            float(dt)                                     # the host reads the step's dt
            s_out.wait_stream(comp)
            with torch.cuda.stream(s_out):
                for r, q in zip(pin_out[b], Qn):
                    r.copy_(q, non_blocking=True)
                    q.record_stream(s_out)
        comp.wait_stream(s_out)

    def serial(n):
        for _ in range(n):
            for d, p in zip(dbuf[0], pin_in[0]):
                d.copy_(p, non_blocking=True)
            Qn, dt = s64.step(tuple(dbuf[0]))
            for r, q in zip(pin_out[0], Qn):
                r.copy_(q, non_blocking=True)
            float(dt)

    def timed(fn, n):
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn(n)
        e1.record()
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1)) / n

    pipelined(max(1, Wm))
    e2e_ms = timed(pipelined, K)
    serial(max(1, Wm))
    e2e_serial_ms = timed(serial, K)
    barrier()

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return None
    hbm, peak_kind = peaks()
    f = out["fp64"]
    alg_launch = np.mean(STAGE_BYTES["fp64"]) * cells
    achieved = alg_launch / (f["stage_ms"] * 1e-3) / 1e9
    tr = TRAFFIC_PER_CELL["fp64"]
    line = {
        "metric": METRIC, "value": whole_job_value(cells, world, f["ms"]), "unit": METRIC, "n_gpus": world,
        "steps": K, "warmup": Wm, "ms_per_step": f["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded log-law IC + 10% noise)",
        "config": config_dict({"parallelism": f"replicas x{world}" if world > 1 else "1 GPU", "form": "fp64"}),
        "e2e": {"value": cells * world / (e2e_ms * 1e-3) / 1e6, "unit": METRIC, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                "path": "Solver.step on an independent host state per step: state copied in from pinned "
                        "host memory, dt read by the host, new state copied out to pinned host memory, "
                        "every step; the copies of consecutive steps overlap the step between them on "
                        "two copy streams",
                "serial_ms_per_step": e2e_serial_ms},
        "gpu_launches": int(f["launches"]),
        "roofline": {"bound": "hbm", "kernel": "stage_kernel<double,KEP>", "achieved": achieved, "peak": hbm,
                     "unit": "GB/s", "frac": achieved / hbm, "peak_source": f"{peak_kind} hbm_gbs",
                     "traffic": None if tr is None else tr * cells,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum per launch on a 128^3 "
                                       "case of the workload, per interior cell x cells",
                     "alg_bytes_per_launch": alg_launch, "mean_launch_ms": f["stage_ms"],
                     "whole_step_frac": (STEP_BYTES["fp64"] + CMF_BYTES) * cells / (f["ms"] * 1e-3) / 1e9 / hbm},
        "mixed": {"value": cells * world / (out["mixed"]["ms"] * 1e-3) / 1e6, "ms_per_step": out["mixed"]["ms"],
                  "speedup_vs_fp64": f["ms"] / out["mixed"]["ms"],
                  "state_rel_l2_vs_fp64_after_steps": out["mixed"]["err"], "steps_compared": K + Wm + min(K, 20),
                  "stage_launch_ms": out["mixed"]["stage_ms"], "kernel_split": out["mixed"]["split"],
                  "roofline_frac": np.mean(STAGE_BYTES["mixed"]) * cells / (out["mixed"]["stage_ms"] * 1e-3) / 1e9 / hbm},
        "kernel_split": dict(f["split"], how="a separate pass of min(K, 20) steps with CUDA events around every "
                                              "launch; the timed steps run without them"),
        "clocks": f["clk"],
    }
    if FP64_FLOP_PER_CELL is not None:
        # the FP64 stage kernel's other roof: its FP64 instructions against the FP64 pipe
        fl = FP64_FLOP_PER_CELL * cells
        tfs = fl / (f["stage_ms"] * 1e-3) / 1e12
        inst_rate = FP64_INST_PER_CELL * cells / (f["stage_ms"] * 1e-3)
        line["roofline"]["fp64_pipe"] = {
            "achieved": tfs, "peak": FP64_PEAK_TFLOPS, "unit": "TFLOP/s", "frac": tfs / FP64_PEAK_TFLOPS,
            "flop_per_launch": fl, "flop_per_cell": FP64_FLOP_PER_CELL,
            "pipe_inst_per_cell": FP64_INST_PER_CELL, "pipe_frac": inst_rate / FP64_PEAK_INST,
            "flop_source": "ncu: 2 x dfma + dadd + dmul thread instructions per launch (mean of the three "
                           "RK stages) on a 128^3 case of the workload, per interior cell",
            "peak_source": "nominal: 148 SMs x 64 FP64 lanes x 1.965 GHz (x 2 flop per FMA); pipe_frac "
                           "counts FP64 instructions against the lanes (DADD and DMUL take a lane like DFMA)"}
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args.cpu_cells)
    if world == 1 and args.extra:
        line["diagnostics"] = diagnostics_leg(mesh, s64, Q64, cells)
        del s64, s32, Q64, Q32, dbuf, pin_in, pin_out
        line["mixed"]["error_vs_fp64"] = precision_leg()
        line["configs"] = configs_leg()
    if world == 1 and args.serving_requests > 0:
        line["serving"] = serving_leg(args)
    if dist is not None:
        dist.destroy_process_group()
    return line


# ----------------------------------------------------------------------------- configs 3 and 4, precision
def configs_leg(steps=100):
    """Throughput of the smooth ramp (config 3) and the NACA 0012 C-grid (config 4), both forms,
    tile shape from the autotuner; inputs larger than L2.  CUDA events around `steps` steps of
    the state-resident loop, as for config 2; the host's time (the synthetic inflow's phase)
    advances by the time step read back after the warm-up, so that no step waits for a
    read-back."""
    import torch
    from wmles_jax_b200.profile_case import build
    from wmles_jax_b200.solver import Solver
    out = {}
    for cfg, name in ((3, "smooth ramp 384x96x64, Hybrid + Vreman + wall model + inflow + sponge"),
                      (4, "NACA 0012 C-grid 4 blocks (576x64x40), Hybrid + Vreman + wall model + far field")):
        r = {}
        for p in ("fp64", "mixed"):
            mesh, gas, kw, prim = build(cfg, None, 1)
            cells = sum(int(np.prod(b.n)) for b in mesh.blocks)
            s = Solver(mesh, gas, **kw, precision=p, tile="auto")
            Q = s.init_state(prim)
            t = 0.0
            for _ in range(3):
                Q, dt = s.step(Q, t)
                t += float(dt)
            dt0 = float(dt)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(steps):
                Q, dt = s.step(Q, t)
                t += dt0
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            r[p] = dict(value=cells / ms / 1e3, ms=ms, finite=all(bool(torch.isfinite(q).all()) for q in Q))
        out[f"config{cfg}"] = {"workload": name, "cells": cells, "steps": steps,
                               "fp64": r["fp64"]["value"], "mixed": r["mixed"]["value"], "unit": METRIC,
                               "ms_per_step": {"fp64": r["fp64"]["ms"], "mixed": r["mixed"]["ms"]},
                               "speedup": r["mixed"]["value"] / r["fp64"]["value"],
                               "finite": r["fp64"]["finite"] and r["mixed"]["finite"],
                               "timing": "CUDA events around the steps of the state-resident loop (no read-back "
                                         "per step; the host time advances by the warm-up's last time step)"}
    return out


def diagnostics_leg(mesh, solver, Q, cells, samples=20):
    """Device cost of sampling the flow: PlaneStats.accumulate (per-plane means over the whole
    block, plus the wall shear of both walls) on the config-2 state, CUDA events around
    `samples` calls; algorithmic bytes = the state's 40 B per interior cell."""
    import torch
    from wmles_jax_b200.stats import PlaneStats
    hbm, _ = peaks()
    ps = PlaneStats(mesh, solver)
    for _ in range(3):
        ps.accumulate(Q)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(samples):
        ps.accumulate(Q)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / samples
    from wmles_jax_b200.output import derived_fields
    for _ in range(2):
        derived_fields(solver, Q, as_numpy=False)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(5):
        derived_fields(solver, Q, as_numpy=False)
    e1.record()
    torch.cuda.synchronize()
    dms = e0.elapsed_time(e1) / 5
    return {"plane_stats_ms_per_sample": ms, "plane_stats_hbm_frac": 40.0 * cells / (ms * 1e-3) / 1e9 / hbm,
            "derived_fields_ms": dms,
            "what": "wmles_jax_b200.stats.PlaneStats.accumulate (12 plane means + mean wall shear) and "
                    "wmles_jax_b200.output.derived_fields (apply_bcs + 11 fields per cell, kept on the device) "
                    "on the 256x128x128 state"}


def precision_leg():
    """Mixed vs FP64 on config 2 after 1000 steps from the same input, beside two FP64 runs whose
    inputs differ by a relative 1e-7 (the flow's own sensitivity at that step count)."""
    from wmles_jax_b200.precision_study import compare
    return compare(2, 1000, perturb=1e-7)


# ----------------------------------------------------------------------------- serving (config 5)
def serving_leg(args):
    """Continuous batching of seeded channel requests (Poisson arrivals, uneven grids, Re_tau and
    Ma_b), mixed precision; p50/p99 time-to-result and aggregate Mcell-steps/s."""
    import torch
    from wmles_jax_b200.lowering import block_metrics
    from wmles_jax_b200.serving import Server
    from wmles_jax_b200.workloads import SERVING_GRIDS, serving_mesh, serving_requests
    for g in SERVING_GRIDS:                 # grid catalogue: meshes and metrics built at server start
        m = serving_mesh(g)
        for b, geo in zip(m.blocks, m.geoms):
            block_metrics(b, geo)
    reqs = serving_requests(n=args.serving_requests, rate=args.serving_rate, steps=args.serving_steps, seed=0)
    torch.cuda.synchronize()
    srv = Server(precision="mixed", graphs=True, tile="auto", policy="srpt")
    tile, tile_ms = srv.tune(reqs)              # before the arrivals start (cached per machine)
    srv.tile = tile
    results = srv.run(reqs, timeout=1800)
    st = srv.stats
    bad = sum(1 for r in results.values() if not all(bool(torch.isfinite(q).all()) for q in r.state))
    return {"requests": st["requests"], "steps_per_request": args.serving_steps,
            "arrivals": f"Poisson, {args.serving_rate}/s, seed 0",
            "grids": [list(g) for g in SERVING_GRIDS], "re_tau": [550, 5200], "ma_b": [0.1, 0.5],
            "form": "mixed", "scheduling": "least remaining work first within an 8M-cell step budget, "
                                            "the rest paused on the device; cases built smallest first as "
                                            "free HBM allows, up to twice the step budget ahead",
            "tile": tile, "tile_ms_per_step": tile_ms,
            "p50_time_to_result_s": st["p50_s"], "p99_time_to_result_s": st["p99_s"],
            "value": st["mcell_steps_per_s"], "unit": METRIC, "wall_s": st["wall_s"],
            "device_busy_s": st["device_busy_s"], "device_value": st["device_mcell_steps_per_s"],
            "cell_steps": st["cell_steps"], "batch_steps": st["batch_steps"], "graph_steps": st["graph_steps"],
            "graph_captures": st["captures"], "memberships": st["memberships"], "pauses": st["pauses"],
            "gpu_launches": st["kernel_launches"], "peak_admitted_bytes": st["peak_admitted_bytes"],
            "nonfinite_results": bad, "failed_requests": st["failed"],
            "time_to_result": "arrival to the host seeing the last step done on the device, including "
                              "host-side case preparation (IC, ghost programs) and admission"}


# ----------------------------------------------------------------------------- CPU oracle
def _oracle_worker(n, steps, warm, seed):
    """Run the oracle on one slab of the config-2 channel; returns (cells, steps, seconds)."""
    sys.path.insert(0, ROOT)
    from wmles_jax_b200.workloads import channel_case
    from oracle.wmles_oracle import OracleSolver, init_state
    mesh, gas, kw, prim = channel_case(2, n=n)
    s = OracleSolver(mesh, gas, **kw)
    Q = init_state(s, prim)
    for _ in range(warm):
        Q = s.advance(Q, s.max_dt(Q))
    t0 = time.perf_counter()
    for _ in range(steps):
        Q = s.advance(Q, s.max_dt(Q))
    return int(np.prod(n)), steps, time.perf_counter() - t0


def cpu_baseline(nx=8):
    n = (nx, N_CFG2[1], N_CFG2[2])
    cells, steps, sec = _oracle_worker(n, 6, 1, 0)
    return {"value": cells * steps / sec / 1e6, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"{steps} steps (after 1 warm-up) of a {n[0]}x{n[1]}x{n[2]} x-periodic slab of the "
                      f"256x128x128 channel, same physics; NumPy float64 oracle, one process"}


def run_reference(args, rank, world):
    if rank != 0:
        return None
    import multiprocessing as mp
    workers = max(1, min(os.cpu_count() or 1, args.max_workers))
    # each step is one oracle step on a slab of the workload (~1.6 s on an 8-cell slab per
    # core); long runs use a 4-cell slab so that the whole run stays within a few minutes
    nx = args.cpu_cells if args.steps + args.warmup <= 100 else max(4, args.cpu_cells // 2)
    n = (nx, N_CFG2[1], N_CFG2[2])
    ctx = mp.get_context("spawn")
    t0 = time.perf_counter()
    with ctx.Pool(workers) as pool:
        res = pool.starmap(_oracle_worker, [(n, args.steps, args.warmup, i) for i in range(workers)])
    wall = time.perf_counter() - t0
    cells_steps = sum(c * s for c, s, _ in res)
    slowest = max(t for _, _, t in res)
    value = cells_steps / slowest / 1e6
    sample = (f"{workers} processes, each {args.steps} steps (after {args.warmup} warm-up) of its own "
              f"{n[0]}x{n[1]}x{n[2]} x-periodic slab of the 256x128x128 channel (same physics); "
              f"NumPy float64 oracle restating the reference")
    return {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": slowest / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded log-law IC + 10% noise)", "impl": "reference",
            "config": config_dict({"form": "fp64", "host": "CPU",
                                   "sample_per_process": f"{n[0]}x{n[1]}x{n[2]} slab ({int(np.prod(n))} cells)",
                                   "ms_per_step": "one step of every process's slab, all processes at once"}),
            "cpu_baseline": {"value": value, "unit": METRIC, "cores": workers, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "wall_s": wall}


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-cells", type=int, default=8, help="x-cells of the CPU slab sample")
    ap.add_argument("--max-workers", type=int, default=64)
    ap.add_argument("--serving-requests", type=int, default=64, help="config-5 requests (0: skip the leg)")
    ap.add_argument("--no-extra", dest="extra", action="store_false",
                    help="skip the config-3/4 throughput and the 1000-step precision study")
    ap.add_argument("--serving-steps", type=int, default=2000)
    ap.add_argument("--serving-rate", type=float, default=20.0)
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be at least 3")
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", args.gpus))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        line = run_reference(args, rank, world)
    else:
        line = run_ours(args, rank, world, local_rank)
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
