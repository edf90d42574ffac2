"""A driver written against the reference's public API runs unchanged on the cuda backend.

The driver below follows the call sequence of the reference's channel example
(examples/channel_wmles.py:34-59,121-145): ``from wmles import ...`` and ``from
wmles.backend import xp, HAS_JAX, device_info``; a two-block periodic channel with
wall-modelled walls, Hybrid KEP4 / MUSCL-HLLC, Vreman and constant mass flux; an initial
condition written with ``xp`` on the cell centres; the loop ``dt = max_dt(Q); Q =
advance(Q, dt); t += float(dt)``; and the diagnostics ``wall_stats``, ``xp.min`` of the
interior density, ``xp.sum`` of the kinetic energy over ``solver.geoms`` volumes, and
``wall_loads``.  ``wmles`` is the binding package under tests/shim.  Its results are
checked against the CPU oracle driven through the same steps: state within 1e-10 relative
L2, the diagnostics within 1e-10.
"""
import os
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

SHIM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "shim")


def driver(steps, every):
    if SHIM not in sys.path:
        sys.path.insert(0, SHIM)
    from wmles import (Gas, Block, Mesh, Solver, KEP, Hybrid, WallModel, EquilibriumWallModel,
                       ConstantMassFlux)
    from wmles.backend import xp, HAS_JAX, device_info

    gas = Gas()
    h = 0.01
    Lx, Ly, Lz = 2 * np.pi * h, 2 * h, np.pi * h
    nx, ny, nz = 16, 16, 12
    T0, rho0 = 300.0, 1.2
    Ub = 0.3 * float(gas.sound_speed(T0))
    p0 = rho0 * gas.R * T0

    def nodes(x0, x1, ncells):
        x = np.linspace(x0, x1, ncells + 1)
        eta = np.linspace(0, 1, ny + 1)
        y = h * (1 + np.tanh(1.6 * (2 * eta - 1)) / np.tanh(1.6))
        z = np.linspace(0, Lz, nz + 1)
        return np.stack(np.meshgrid(x, y, z, indexing="ij"))

    A, B = Block("A", nodes(0, Lx / 2, nx // 2)), Block("B", nodes(Lx / 2, Lx, nx // 2))
    mesh = Mesh([A, B])
    mesh.connect(A, "imax", B, "imin")
    mesh.connect(B, "imax", A, "imin", shift=(Lx, 0, 0))
    wm = EquilibriumWallModel()
    for b in (A, B):
        mesh.connect(b, "kmin", b, "kmax", shift=(0, 0, -Lz))
        b.set_bc("jmin", WallModel(wm, T_wall=T0, n_match=1))
        b.set_bc("jmax", WallModel(wm, T_wall=T0, n_match=1))
    mesh.finalize()
    kw = dict(scheme=Hybrid(KEP(4)), sgs="vreman", cfl=0.7, constraints=[ConstantMassFlux(0, rho0 * Ub)])
    solver = Solver(mesh, gas, **kw)

    def initial(xc):
        x, y, z = xc
        yn = xp.clip(xp.minimum(y, 2 * h - y) / h, 1e-3, 1.0)
        u = 1.15 * Ub * yn ** (1 / 7)
        k = 2 * np.pi
        u = u + 0.08 * Ub * xp.sin(k * z / Lz * 2) * xp.sin(k * x / Lx)
        v = 0.05 * Ub * xp.sin(k * x / Lx * 2) * xp.sin(k * z / Lz)
        w = 0.05 * Ub * xp.cos(k * x / Lx) * xp.sin(k * y / Ly)
        return xp.stack([rho0 + 0 * x, u, v, w, p0 + 0 * x])

    Q, t = solver.init_state(initial), 0.0
    assert not HAS_JAX and device_info().startswith("cuda")
    log = []
    for it in range(1, steps + 1):
        dt = solver.max_dt(Q)
        Q = solver.advance(Q, dt)
        t += float(dt)
        if it % every == 0:
            st = solver.wall_stats(Q)
            tau = np.mean([np.mean(v[0]) for v in st.values()])
            rmin = min(float(xp.min(b.interior(q[0]))) for b, q in zip(mesh.blocks, Q))
            ke = sum(float(xp.sum(b.interior(0.5 * xp.sum(q[1:4] ** 2, axis=0) / q[0] * g.vol)))
                     for b, q, g in zip(mesh.blocks, Q, solver.geoms))
            loads = solver.wall_loads(Q, (0.0, 0.0, 0.0))
            log.append((it, t, tau, rmin, ke, loads))
    return mesh, gas, kw, initial, Q, log


def test_reference_style_driver_runs_unchanged(W):
    from oracle.wmles_oracle import OracleSolver, init_state
    steps, every = 12, 4
    mesh, gas, kw, initial, Q, log = driver(steps, every)
    assert [row[0] for row in log] == [4, 8, 12]
    ref = OracleSolver(mesh, gas, **kw)
    Qr = init_state(ref, initial)
    t = 0.0
    for it in range(1, steps + 1):
        dt = ref.max_dt(Qr)
        Qr = ref.advance(Qr, dt)
        t += dt
        if it % every == 0:
            _, tg, tau, rmin, ke, loads = log[it // every - 1]
            assert abs(tg - t) <= 1e-12 * t
            st = ref.wall_stats(Qr)
            assert abs(tau - np.mean([np.mean(v[0]) for v in st.values()])) <= 1e-9 * abs(tau)
            rmin_r = min(float(np.min(b.interior(q[0]))) for b, q in zip(mesh.blocks, Qr))
            ke_r = sum(float(np.sum(b.interior(0.5 * np.sum(q[1:4] ** 2, axis=0) / q[0] * g.vol)))
                       for b, q, g in zip(mesh.blocks, Qr, mesh.geoms))
            assert abs(rmin - rmin_r) <= 1e-10 * rmin_r and abs(ke - ke_r) <= 1e-10 * ke_r
            for key, (force, moment) in ref.wall_loads(Qr, (0.0, 0.0, 0.0)).items():
                np.testing.assert_allclose(loads[key][0], force, rtol=1e-9, atol=1e-12)
    for blk, a, b in zip(mesh.blocks, Q, Qr):
        a, b = blk.interior(a.cpu().numpy()), blk.interior(b)
        for c in range(5):
            assert np.linalg.norm(a[c] - b[c]) / np.linalg.norm(b[c]) < 1e-10


def test_whole_array_reductions_are_finite(W):
    """Reductions over whole states (ghost cells included) see defined values."""
    mesh, gas, kw, initial, Q, log = driver(3, 3)
    from wmles.backend import xp
    for q in Q:
        assert bool(torch.isfinite(q).all())
        assert float(xp.min(q[0])) > 0.0
    w, T = gas.cons_to_prim(Q[0])                     # on the device state (tests/test_sod.py:25)
    assert w.is_cuda and float(xp.min(T)) > 0.0
