"""CUDA backend parity with the reference (golden fixtures) and the CPU oracle.

Tolerances: ghost fills bit-exact; one RHS / dt / RK3 step within 1e-11 relative to the
field's max (FP64 with FMA contraction and CUDA's pow/exp differ from NumPy by a few ulp);
the config-1 channel after 100 steps within 1e-10 relative L2 per conservative variable.
"""
import numpy as np
import pytest

import cases as C
from oracle.wmles_oracle import OracleSolver, init_state

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

RHS_TOL = 1e-11
STEP_TOL = 1e-11


def _solver(mesh, gas, kw, **extra):
    from wmles_jax_b200 import Solver
    return Solver(mesh, gas, **kw, **extra)


def _dev(Q):
    return tuple(torch.from_numpy(np.ascontiguousarray(q)).cuda() for q in Q)


def _host(Q):
    return [q.cpu().numpy() for q in Q]


def _maxrel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("tag", C.SMALL_CASES)
def test_golden_case(W, golden, tag):
    mesh, gas, kw, prim, t = C.golden_case(W, tag)
    nb = len(mesh.blocks)
    Qh = tuple(golden[f"{tag}/q{ib}"] for ib in range(nb))
    gpu = _solver(mesh, gas, kw)
    Q = _dev(Qh)
    # ghost fill
    full = _host(gpu.apply_bcs(Q, gpu.geoms, t))
    for ib in range(nb):
        ref = golden[f"{tag}/bcs{ib}"]
        if tag == "ramp_small":
            np.testing.assert_allclose(full[ib], ref, rtol=1e-12, atol=0)
        else:
            assert np.array_equal(full[ib], ref), f"ghost fill block {ib}"
    # RHS
    R = _host(gpu.rhs(Q, t))
    for ib, blk in enumerate(mesh.blocks):
        ref = golden[f"{tag}/rhs{ib}"]
        got = blk.interior(R[ib])
        for c in range(5):
            assert _maxrel(got[c], ref[c]) < RHS_TOL, (ib, c, _maxrel(got[c], ref[c]))
        assert np.all(R[ib][:, :blk.ng] == 0.0)
    # dt and one step
    dt = gpu.max_dt(Q, t)
    assert abs(float(dt) - golden[f"{tag}/dt"]) <= 1e-13 * golden[f"{tag}/dt"]
    Q1 = _host(gpu.advance(Q, float(golden[f"{tag}/dt"]), t))
    for ib, blk in enumerate(mesh.blocks):
        ref = golden[f"{tag}/adv{ib}"]
        got = blk.interior(Q1[ib])
        for c in range(5):
            assert _maxrel(got[c], ref[c]) < STEP_TOL, (ib, c, _maxrel(got[c], ref[c]))
    # wall statistics and loads
    stats = gpu.wall_stats(Q)
    for (bname, face), (tau, qw) in stats.items():
        rt = golden[f"{tag}/tau/{bname}/{face}"]
        assert _maxrel(tau, rt) < 1e-12
        np.testing.assert_allclose(qw, golden[f"{tag}/qw/{bname}/{face}"], rtol=1e-11, atol=1e-9)
    if stats:
        loads = gpu.wall_loads(Q, (0.1, 0.2, 0.3))
        for (bname, face), (force, moment) in loads.items():
            np.testing.assert_allclose(force, golden[f"{tag}/force/{bname}/{face}"], rtol=1e-11, atol=1e-8)
            np.testing.assert_allclose(moment, golden[f"{tag}/moment/{bname}/{face}"], rtol=1e-11, atol=1e-8)


def test_cfg1_channel_100_steps_matches_reference(W, golden_cfg1):
    """The FP64 parity bar: FP64 step within 1e-10 relative L2 of the reference after
    100 steps of the config-1 channel (2 blocks of 16x32x16, KEP2, Smagorinsky, wall model,
    constant mass flux)."""
    mesh, gas, kw, prim = C.cfg1_case(W)
    ref = OracleSolver(mesh, gas, **kw)
    Q = _dev(init_state(ref, prim))
    gpu = _solver(mesh, gas, kw)
    steps = int(golden_cfg1["steps"])
    dts = []
    for _ in range(steps):
        Q, dt = gpu.step(Q)
        dts.append(dt)
    dts = np.array([float(d) for d in dts])
    np.testing.assert_allclose(dts, golden_cfg1["dts"], rtol=1e-10)
    for ib, blk in enumerate(mesh.blocks):
        got = blk.interior(Q[ib].cpu().numpy())
        want = golden_cfg1[f"final{ib}"]
        for c in range(5):
            err = np.linalg.norm(got[c] - want[c]) / np.linalg.norm(want[c])
            assert err < 1e-10, (ib, c, err)
    stats = gpu.wall_stats(Q)
    for (bname, face), (tau, qw) in stats.items():
        assert _maxrel(tau, golden_cfg1[f"tau/{bname}/{face}"]) < 1e-9


@pytest.mark.parametrize("scheme_name,sgs,tile", [
    ("kep4", "wale", 0), ("kep2", "smagorinsky", 1), ("muscl", "vreman", 2),
    ("hybrid", "vreman", 0), ("minmod", None, 1)])
def test_oracle_parity_ragged_tiles(W, scheme_name, sgs, tile):
    """Block sizes that are not multiples of the tile shape, every tile variant."""
    sch = {"kep4": lambda: W.KEP(4), "kep2": lambda: W.KEP(2), "muscl": lambda: W.MUSCLHLLC(),
           "hybrid": lambda: W.Hybrid(W.KEP(4), th0=0.02, th1=0.2), "minmod": lambda: W.MUSCLHLLC("minmod")}
    mesh = C.skew_case(W, "flip", n=(14, 11, 37), ybc="wm")
    gas = W.Gas()
    kw = dict(scheme=sch[scheme_name](), sgs=sgs, cfl=0.5)
    ref = OracleSolver(mesh, gas, **kw)
    Qh = init_state(ref, C.skew_prim)
    gpu = _solver(mesh, gas, kw, tile=tile, chunk=5)
    Q = _dev(Qh)
    R = _host(gpu.rhs(Q))
    Rr = ref.rhs(Qh)
    for ib, blk in enumerate(mesh.blocks):
        for c in range(5):
            assert _maxrel(blk.interior(R[ib])[c], blk.interior(Rr[ib])[c]) < RHS_TOL
    dt = ref.max_dt(Qh)
    Q1 = _host(gpu.advance(Q, dt))
    Q1r = ref.advance(Qh, dt)
    for ib, blk in enumerate(mesh.blocks):
        for c in range(5):
            assert _maxrel(blk.interior(Q1[ib])[c], blk.interior(Q1r[ib])[c]) < STEP_TOL


def test_minimum_block_size(W):
    """Blocks of exactly ng cells per direction (the reference's minimum)."""
    mesh = C.skew_case(W, "rot_cyc", n=(6, 3, 3), ybc="slip")
    gas = W.Gas()
    kw = dict(scheme=W.KEP(4), sgs="vreman", cfl=0.5)
    ref = OracleSolver(mesh, gas, **kw)
    Qh = init_state(ref, C.skew_prim)
    gpu = _solver(mesh, gas, kw)
    R = _host(gpu.rhs(_dev(Qh)))
    Rr = ref.rhs(Qh)
    for ib, blk in enumerate(mesh.blocks):
        for c in range(5):
            assert _maxrel(blk.interior(R[ib])[c], blk.interior(Rr[ib])[c]) < RHS_TOL


def test_mixed_precision_close_to_fp64(W):
    mesh, gas, kw, prim = C.cfg1_case(W)
    ref = OracleSolver(mesh, gas, **kw)
    Qh = init_state(ref, prim)
    g64 = _solver(mesh, gas, kw)
    g32 = _solver(mesh, gas, kw, precision="mixed")
    Q = _dev(Qh)
    R64, R32 = _host(g64.rhs(Q)), _host(g32.rhs(Q))
    for ib, blk in enumerate(mesh.blocks):
        for c in range(1, 5):
            a, b = blk.interior(R32[ib])[c], blk.interior(R64[ib])[c]
            assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-3
    Qa, Qb = Q, Q
    for _ in range(10):
        Qa, _ = g64.step(Qa)
        Qb, _ = g32.step(Qb)
    for ib, blk in enumerate(mesh.blocks):
        for c in range(5):
            a = blk.interior(Qb[ib].cpu().numpy())[c]
            b = blk.interior(Qa[ib].cpu().numpy())[c]
            assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-4


def test_input_state_interior_unchanged(W):
    """advance/step refresh ghost cells of the input in place but never its interior."""
    mesh, gas, kw, prim = C.cfg1_case(W)
    ref = OracleSolver(mesh, gas, **kw)
    Qh = init_state(ref, prim)
    gpu = _solver(mesh, gas, kw)
    Q = _dev(Qh)
    gpu.step(Q)
    for blk, q, qh in zip(mesh.blocks, Q, Qh):
        assert np.array_equal(blk.interior(q.cpu().numpy()), blk.interior(qh))


def test_bad_state_rejected(W):
    mesh, gas, kw, prim = C.cfg1_case(W)
    gpu = _solver(mesh, gas, kw)
    with pytest.raises(ValueError):
        gpu.rhs(tuple(torch.zeros((5, 4, 4, 4), dtype=torch.float64, device="cuda") for _ in mesh.blocks))
    with pytest.raises(TypeError):
        gpu.rhs(tuple(torch.zeros((5,) + b.N, dtype=torch.float64) for b in mesh.blocks))


@pytest.mark.parametrize("tag", ["split_wm_hybrid", "channel_small_cmf"])
def test_output_ghost_cells_defined(W, golden, tag):
    """Ghost cells of a returned state: the input's (after the step's boundary fill) plus
    the constraint's shift, never uninitialised memory."""
    mesh, gas, kw, prim, t = C.golden_case(W, tag)
    nb = len(mesh.blocks)
    gpu = _solver(mesh, gas, kw)
    for path in ("advance", "step"):
        Q = _dev(tuple(golden[f"{tag}/q{ib}"] for ib in range(nb)))
        # poison the memory the outputs will come from
        junk = [torch.full_like(q, float("nan")) for q in Q]
        del junk
        Q1 = gpu.advance(Q, gpu.max_dt(Q), t) if path == "advance" else gpu.step(Q, t)[0]
        for blk, q, q1 in zip(mesh.blocks, Q, Q1):
            ghost = torch.ones(q.shape[1:], dtype=torch.bool, device=q.device)
            blk.interior(ghost)[...] = False
            a, b = q[:, ghost], q1[:, ghost]
            assert bool(torch.isfinite(b).all())
            if "cmf" in tag:
                shift = b[1] - a[1]                 # uniform momentum shift of the constraint
                assert float((shift - shift[0]).abs().max()) <= 1e-12 * float(a[1].abs().max())
                assert torch.equal(b[0], a[0]) and torch.equal(b[2:4], a[2:4])
            else:
                assert torch.equal(a, b)
