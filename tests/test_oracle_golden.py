"""Pin the CPU oracle and this package's host set-up to the reference's own outputs.

The golden fixtures were produced by the reference implementation itself
(tests/golden/make_golden.py, NumPy float64 backend).  Geometry and ghost fills must be
bit-identical; RHS, dt, one RK3 step and wall diagnostics agree to round-off.
"""
import numpy as np
import pytest

import cases as C
from oracle.wmles_oracle import OracleSolver, init_state, equilibrium_wall


def _build(W, tag):
    mesh, gas, kw, prim, t = C.golden_case(W, tag)
    return mesh, OracleSolver(mesh, gas, **kw), prim, t


def _rel(a, b):
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(np.asarray(a) - np.asarray(b)).max() / scale


@pytest.mark.parametrize("tag", sorted(C.GEOM_CASES))
def test_geometry_bit_identical(W, golden, tag):
    mesh, solver, _, _ = _build(W, tag)
    for ib, g in enumerate(mesh.geoms):
        assert np.array_equal(g.vol, golden[f"{tag}/vol{ib}"])
        assert np.array_equal(g.xc, golden[f"{tag}/xc{ib}"])
        for d in range(3):
            assert np.array_equal(g.S[d], golden[f"{tag}/S{d}_{ib}"])
            assert np.array_equal(g.xf[d], golden[f"{tag}/xf{d}_{ib}"])


@pytest.mark.parametrize("tag", C.SMALL_CASES)
def test_initial_state_and_ghost_fill_bit_identical(W, golden, tag):
    mesh, solver, prim, t = _build(W, tag)
    Q = init_state(solver, prim)
    for ib, q in enumerate(Q):
        assert np.array_equal(q, golden[f"{tag}/q{ib}"]), "initial state differs"
    Qb = solver.apply_bcs(Q, t)
    for ib, q in enumerate(Qb):
        assert np.array_equal(q, golden[f"{tag}/bcs{ib}"]), f"ghost fill of block {ib} differs"


@pytest.mark.parametrize("tag", C.SMALL_CASES)
def test_rhs_dt_step_match_reference(W, golden, tag):
    mesh, solver, _, t = _build(W, tag)
    Q = tuple(golden[f"{tag}/q{ib}"] for ib in range(len(mesh.blocks)))
    R = solver.rhs(Q, t)
    for ib, (blk, r) in enumerate(zip(mesh.blocks, R)):
        ref = golden[f"{tag}/rhs{ib}"]
        for c in range(5):
            assert _rel(blk.interior(r)[c], ref[c]) < 1e-13, (ib, c)
    dt = solver.max_dt(Q, t)
    assert dt == golden[f"{tag}/dt"]
    Q1 = solver.advance(Q, float(dt), t)
    for ib, (blk, q) in enumerate(zip(mesh.blocks, Q1)):
        ref = golden[f"{tag}/adv{ib}"]
        for c in range(5):
            assert _rel(blk.interior(q)[c], ref[c]) < 1e-13, (ib, c)


@pytest.mark.parametrize("tag", ["split_wm_hybrid", "flip_wmad_kep2", "zoo_hybrid", "ramp_small",
                                 "channel_small_cmf"])
def test_wall_diagnostics_match_reference(W, golden, tag):
    mesh, solver, _, _ = _build(W, tag)
    Q = tuple(golden[f"{tag}/q{ib}"] for ib in range(len(mesh.blocks)))
    stats = solver.wall_stats(Q)
    assert stats
    for (bname, face), (tau, qw) in stats.items():
        assert _rel(tau, golden[f"{tag}/tau/{bname}/{face}"]) < 1e-13
        np.testing.assert_allclose(qw, golden[f"{tag}/qw/{bname}/{face}"], rtol=1e-12, atol=1e-12)
    loads = solver.wall_loads(Q, (0.1, 0.2, 0.3))
    for (bname, face), (force, moment) in loads.items():
        np.testing.assert_allclose(force, golden[f"{tag}/force/{bname}/{face}"], rtol=1e-12, atol=1e-9)
        np.testing.assert_allclose(moment, golden[f"{tag}/moment/{bname}/{face}"], rtol=1e-12, atol=1e-9)


def test_inflow_modes_identical(W, golden):
    mesh, solver, _, _ = _build(W, "ramp_small")
    modes = mesh.blocks[0].faces[(0, 0)].mode_table()
    assert np.array_equal(modes, golden["ramp_small/modes"])


def test_sod_after_three_steps(W, golden):
    mesh = C.sod_case(W)
    gas = W.Gas(R=1.0, mu_ref=1e-9)
    solver = OracleSolver(mesh, gas, W.Hybrid(th0=0.3, th1=0.6), sgs=None, cfl=0.5)
    Q = tuple(golden[f"sod_hybrid/q{ib}"] for ib in range(1))
    R = solver.rhs(Q)
    ref = golden["sod_hybrid/rhs0"]
    scale = np.abs(ref).max()
    assert np.abs(mesh.blocks[0].interior(R[0]) - ref).max() / scale < 1e-13
    assert solver.max_dt(Q) == golden["sod_hybrid/dt"]


def test_wall_model_known_answers(W, golden):
    wm = W.EquilibriumWallModel()
    args = [golden[f"kat_wall/{k}"] for k in ("h", "U", "Th", "ph")]
    for Tw, name in ((300.0, "iso"), (None, "adia")):
        tau, qw = equilibrium_wall(wm, W.Gas(), *args, Tw)
        np.testing.assert_allclose(tau, golden[f"kat_wall/{name}/tau"], rtol=1e-14)
        np.testing.assert_allclose(qw * np.ones_like(tau), golden[f"kat_wall/{name}/qw"], rtol=1e-13, atol=1e-12)


def test_spalding_inversion_recovers_utau(W):
    """Known answer of tests/test_multiblock.py:134-149: a bisection-inverted Spalding
    profile gives back u_tau to 1e-6."""
    from oracle.wmles_oracle import spalding_utau
    wm = W.EquilibriumWallModel()
    k, B = wm.kappa, wm.B
    nu, ut, h = 1.5e-5, 2.0, 0.003
    yp = h * ut / nu
    f = lambda up: up + np.exp(-k * B) * (np.exp(k * up) - 1 - k * up - (k * up) ** 2 / 2 - (k * up) ** 3 / 6) - yp
    lo, hi = 1e-6, 60.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if f(mid) < 0 else (lo, mid)
    U = ut * 0.5 * (lo + hi)
    got = spalding_utau(wm, np.array([h]), np.array([U]), np.array([1.2]), np.array([nu * 1.2]))
    assert abs(got[0] - ut) < 1e-6


def test_cfg1_oracle_100_steps(W, golden_cfg1):
    """The oracle reproduces the reference's 100-step config-1 channel trajectory."""
    mesh, gas, kw, prim = C.cfg1_case(W)
    solver = OracleSolver(mesh, gas, **kw)
    Q = init_state(solver, prim)
    assert np.allclose([q.sum() for q in Q], golden_cfg1["ic_checksum"], rtol=0, atol=0)
    steps = int(golden_cfg1["steps"])
    for n in range(steps):
        dt = solver.max_dt(Q)
        assert abs(dt - golden_cfg1["dts"][n]) <= 1e-12 * dt
        Q = solver.advance(Q, dt)
    for ib, (blk, q) in enumerate(zip(mesh.blocks, Q)):
        ref = golden_cfg1[f"final{ib}"]
        for c in range(5):
            err = np.linalg.norm(blk.interior(q)[c] - ref[c]) / np.linalg.norm(ref[c])
            assert err < 1e-12, (ib, c, err)
