"""Generate golden fixtures by running the REFERENCE implementation (its NumPy float64
fallback) on the synthetic cases of ``tests/golden/cases.py``.

    python tests/golden/make_golden.py [--reference /root/reference]

Needs the reference source tree; it runs in the build container only and writes
``tests/golden/*.npz``, which travel with the repository.  The reference's package is
imported with WMLES_BACKEND=numpy (wmles/backend.py:18,44-49), which is the float64
path that runs here (JAX is not installed).
"""
import argparse
import os
import sys
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))     # node generators of wmles_jax_b200.workloads (NumPy only)


def load_reference(root):
    os.environ["WMLES_BACKEND"] = "numpy"
    sys.path.insert(0, root)
    import wmles
    import wmles.smooth_ramp as sr
    from wmles.wall_model import EquilibriumWallModel
    W = types.SimpleNamespace(**{k: getattr(wmles, k) for k in dir(wmles) if not k.startswith("_")})
    W.SmoothRampInflow, W.SmoothRampSponge = sr.SmoothRampInflow, sr.SmoothRampSponge
    W.EquilibriumWallModel = EquilibriumWallModel
    return W


def interior(blk, a):
    return np.asarray(blk.interior(a))


def record_case(out, tag, mesh, solver, Q, time_=0.0, geom=False, advance=True):
    """Store inputs and reference outputs of one case under keys '<tag>/...'."""
    for ib, q in enumerate(Q):
        out[f"{tag}/q{ib}"] = np.asarray(q)
    Qb = solver.apply_bcs(Q, solver.geoms, time_)
    for ib, q in enumerate(Qb):
        out[f"{tag}/bcs{ib}"] = np.asarray(q)
    R = solver.rhs(Q, time_)
    for ib, (blk, r) in enumerate(zip(solver.blocks, R)):
        out[f"{tag}/rhs{ib}"] = interior(blk, np.asarray(r))
    dt = float(solver.max_dt(Q, time_))
    out[f"{tag}/dt"] = np.array(dt)
    if advance:
        Q1 = solver.advance(Q, dt, time_)
        for ib, (blk, q) in enumerate(zip(solver.blocks, Q1)):
            out[f"{tag}/adv{ib}"] = interior(blk, np.asarray(q))
    stats = solver.wall_stats(Q)
    for (bname, face), (tau, qw) in sorted(stats.items()):
        out[f"{tag}/tau/{bname}/{face}"] = np.asarray(tau)
        out[f"{tag}/qw/{bname}/{face}"] = np.asarray(qw)
    if stats:
        loads = solver.wall_loads(Q, (0.1, 0.2, 0.3))
        for (bname, face), (force, moment) in sorted(loads.items()):
            out[f"{tag}/force/{bname}/{face}"] = np.asarray(force)
            out[f"{tag}/moment/{bname}/{face}"] = np.asarray(moment)
    if geom:
        for ib, g in enumerate(solver.geoms):
            out[f"{tag}/vol{ib}"] = np.asarray(g.vol)
            out[f"{tag}/xc{ib}"] = np.asarray(g.xc)
            for d in range(3):
                out[f"{tag}/S{d}_{ib}"] = np.asarray(g.S[d])
                out[f"{tag}/xf{d}_{ib}"] = np.asarray(g.xf[d])


def make_trajectories(W, C):
    """golden_traj.npz: the reference's own trajectories, run here.

    * <case>/...: 100 steps of the reduced config-2 channel (KEP4 + WALE + wall model +
      constant mass flux), the small smooth ramp (Hybrid + Vreman + synthetic inflow +
      sponge + characteristic outflow) and the NACA C-grid at 1/8 of its cell counts, with
      the drivers' loop (dt = max_dt(Q, t); Q = advance(Q, dt, t); t += dt): every dt, the
      final interior state, the final wall stress, and the initial state's checksums.
    * sod/<scheme>/...: the reference's Sod tube (tests/test_sod.py:7-28) run to t = 0.2 with
      MUSCL-HLLC and with Hybrid (th0 0.3, th1 0.6): the final interior state and the dts.
    * freestream/<scheme>: the reference's free-stream residual on the skewed periodic box
      (tests/test_multiblock.py:100-107), max over variables of max |RHS|.
    """
    out = {}
    for tag in C.TRAJ_CASES:
        mesh, gas, kw, prim, t = C.traj_case(W, tag)
        solver = W.Solver(mesh, gas, **kw)
        Q = solver.init_state(prim)
        out[f"{tag}/ic_sum"] = np.array([[float(np.sum(np.asarray(q)[v])) for v in range(5)] for q in Q])
        out[f"{tag}/t0"] = np.array(t)
        t0 = time.perf_counter()
        dts = []
        for _ in range(C.TRAJ_STEPS):
            dt = float(solver.max_dt(Q, t))
            Q = solver.advance(Q, dt, t)
            t += dt
            dts.append(dt)
        out[f"{tag}/dts"] = np.array(dts)
        for ib, (blk, q) in enumerate(zip(solver.blocks, Q)):
            out[f"{tag}/final{ib}"] = interior(blk, np.asarray(q))
        for (bname, face), (tau, qw) in sorted(solver.wall_stats(Q).items()):
            out[f"{tag}/tau/{bname}/{face}"] = np.asarray(tau)
        print(f"trajectory {tag}: {C.TRAJ_STEPS} steps, {time.perf_counter() - t0:.1f} s")
    for name, make in C.SOD_SCHEMES.items():
        mesh, Q, dts = C.sod_run(W, W.Solver, make(W))
        out[f"sod/{name}/final"] = interior(mesh.blocks[0], Q[0])
        out[f"sod/{name}/dts"] = dts
        print(f"sod {name}: {len(dts)} steps")
    for name, make in C.FREESTREAM_SCHEMES.items():
        mesh = C.freestream_mesh(W)
        s = W.Solver(mesh, W.Gas(), make(W), sgs="vreman", cfl=0.5)
        R = s.rhs(s.init_state(C.freestream_prim))
        out[f"freestream/{name}"] = np.array(max(float(np.abs(interior(mesh.blocks[0], np.asarray(R[0]))[v]).max())
                                                for v in range(5)))
        print(f"free stream {name}: residual {float(out[f'freestream/{name}']):.3e}")
    np.savez_compressed(os.path.join(HERE, "golden_traj.npz"), **out)
    print("wrote golden_traj.npz:", len(out), "arrays")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--skip-cfg1", action="store_true", help="keep the existing config-1 fixture")
    ap.add_argument("--traj-only", action="store_true",
                    help="write only golden_traj.npz (100-step trajectories, Sod, free stream)")
    args = ap.parse_args()
    W = load_reference(args.reference)
    sys.path.insert(0, HERE)
    sys.path.append(ROOT)
    import cases as C

    make_trajectories(W, C)
    if args.traj_only:
        return

    # ---------------------------------------------------------------- small topology/physics cases
    out = {}
    for tag in C.SMALL_CASES:
        mesh, gas, kw, prim, t = C.golden_case(W, tag)
        solver = W.Solver(mesh, gas, **kw)
        Q = solver.init_state(prim)
        record_case(out, tag, mesh, solver, Q, time_=t, geom=tag in C.GEOM_CASES)
        print("case", tag, "ok")
        if tag == "ramp_small":
            out["ramp_small/modes"] = np.array(
                [[np.asarray(v) for v in m] for m in mesh.blocks[0].faces[(0, 0)]._modes])

    # sod tube after 3 steps, hybrid with low thresholds (shock-capturing branch active)
    mesh = C.sod_case(W)
    gas = W.Gas(R=1.0, mu_ref=1e-9)
    solver = W.Solver(mesh, gas, W.Hybrid(th0=0.3, th1=0.6), sgs=None, cfl=0.5)
    Q = solver.init_state(C.sod_prim)
    for _ in range(3):
        Q = solver.advance(Q, float(solver.max_dt(Q)))
    record_case(out, "sod_hybrid", mesh, solver, Q)

    # known-answer tests of the wall model (Spalding inversion and Kader), reference API
    wm = W.EquilibriumWallModel()
    rng = np.random.default_rng(7)
    h = 10 ** rng.uniform(-4, -1, 64)
    U = 10 ** rng.uniform(-1, 2, 64)
    Th = rng.uniform(250, 350, 64)
    ph = rng.uniform(5e4, 1.5e5, 64)
    for Tw, name in ((300.0, "iso"), (None, "adia")):
        tau, qw = wm(W.Gas(), h, U, Th, ph, Tw)
        out[f"kat_wall/{name}/tau"], out[f"kat_wall/{name}/qw"] = np.asarray(tau), np.asarray(qw * np.ones_like(tau))
    out["kat_wall/h"], out["kat_wall/U"], out["kat_wall/Th"], out["kat_wall/ph"] = h, U, Th, ph

    np.savez_compressed(os.path.join(HERE, "golden_cases.npz"), **out)
    print("wrote golden_cases.npz:", len(out), "arrays")

    # ---------------------------------------------------------------- plane statistics
    # the reference's PlaneStats (wmles/channel5200.py:121-199) over two samples of the
    # small constant-mass-flux channel: the initial state and the state after one step
    from wmles.channel5200 import PlaneStats
    mesh, gas, kw, prim, t = C.golden_case(W, "channel_small_cmf")
    solver = W.Solver(mesh, gas, **kw)
    Q0 = solver.init_state(prim)
    Q1 = solver.advance(Q0, float(solver.max_dt(Q0)))
    ps = PlaneStats(mesh, solver)
    ps.accumulate(Q0)
    ps.accumulate(Q1)
    y, avg = ps.result()
    outp = {"y": np.asarray(y), "mean_tau_w": np.array(ps.mean_tau_w), "mu_ref": np.array(gas.mu_ref)}
    for ib, (a, b) in enumerate(zip(Q0, Q1)):
        outp[f"q0_{ib}"], outp[f"q1_{ib}"] = np.asarray(a), np.asarray(b)
    for k, v in avg.items():
        outp[f"avg/{k}"] = np.asarray(v)
    u_tau, wu = ps.wall_units(ps.mean_tau_w, 1.0, gas.mu_ref, 1.0)
    outp["wu/u_tau"] = np.array(u_tau)
    for k, v in wu.items():
        outp[f"wu/{k}"] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, "golden_planestats.npz"), **outp)
    print("wrote golden_planestats.npz:", len(outp), "arrays")

    # ---------------------------------------------------------------- derived output fields
    # the reference's derived_fields (wmles/io_vtk.py:269-293; pyvista is not needed for it)
    # on two skewed split blocks with the wall model and WALE, and on the NACA C-grid (Vreman)
    from wmles.io_vtk import derived_fields
    outd = {}
    for tag in ("split_wm_hybrid", "naca_small"):
        mesh, gas, kw, prim, t = C.golden_case(W, tag)
        solver = W.Solver(mesh, gas, **kw)
        Q = tuple(out[f"{tag}/q{ib}"] for ib in range(len(mesh.blocks)))
        for ib, fields in derived_fields(solver, Q).items():
            for k, v in fields.items():
                outd[f"{tag}/{ib}/{k}"] = np.asarray(v)
    np.savez_compressed(os.path.join(HERE, "golden_derived.npz"), **outd)
    print("wrote golden_derived.npz:", len(outd), "arrays")

    # ---------------------------------------------------------------- config-1 channel, 100 steps
    if args.skip_cfg1:
        return
    mesh, gas, kw, prim = C.cfg1_case(W)
    solver = W.Solver(mesh, gas, **kw)
    Q = solver.init_state(prim)
    q0 = [np.asarray(q).copy() for q in Q]
    t0 = time.perf_counter()
    dts, t = [], 0.0
    for _ in range(args.steps):
        dt = solver.max_dt(Q)
        Q = solver.advance(Q, dt)
        dts.append(float(dt))
        t += float(dt)
    wall = time.perf_counter() - t0
    out1 = {"dts": np.array(dts), "t": np.array(t), "steps": np.array(args.steps),
            "ic_checksum": np.array([float(np.sum(q)) for q in q0]), "cpu_seconds": np.array(wall)}
    for ib, (blk, q) in enumerate(zip(solver.blocks, Q)):
        out1[f"final{ib}"] = interior(blk, np.asarray(q))
    stats = solver.wall_stats(Q)
    for (bname, face), (tau, qw) in sorted(stats.items()):
        out1[f"tau/{bname}/{face}"] = np.asarray(tau)
        out1[f"qw/{bname}/{face}"] = np.asarray(qw)
    np.savez_compressed(os.path.join(HERE, "golden_channel_cfg1.npz"), **out1)
    print(f"wrote golden_channel_cfg1.npz ({args.steps} steps, {wall:.1f} s)")


if __name__ == "__main__":
    main()
