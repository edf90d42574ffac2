"""Multi-step parity of the CUDA path with the reference's own runs
(tests/golden/golden_traj.npz, written by the reference's NumPy float64 path).

Tolerances:
* FP64, 100 steps of the reduced config-2 channel (KEP4 + WALE + wall model + constant mass
  flux), the small smooth ramp (Hybrid + Vreman + synthetic inflow + sponge +
  characteristic outflow) and the NACA C-grid at 1/8 of its cells (four blocks, transposed
  and flipped interfaces, far field): every dt within 1e-10 relative, the final state within
  1e-10 relative L2 per conservative variable, the final wall stress within 1e-9 — through
  the drivers' loop (max_dt + advance, examples/channel_wmles.py:124-126) and through the
  fused ``step``;
* ``Solver.init_state`` bit-identical to the reference's (wmles/solver.py:54-56);
* Sod tube (tests/test_sod.py:7-28) to t = 0.2, FP64: the same number of steps, every dt
  within 1e-11, the final state within 1e-11 of the field's max (the momentum's max for the
  three momentum components); the mixed form within 1e-4 of the FP64 state and on the exact
  plateaus;
* free stream on the skewed periodic box (tests/test_multiblock.py:100-107): FP64 below
  the reference's bound of 0.1; the mixed form (FP32 metrics and fluxes) below 1e-6 of the
  energy-flux scale (E + p) |u| |S| / V of the case.
"""
import os

import numpy as np
import pytest

import cases as C

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_traj.npz")
TRAJ_TOL = 1e-10


@pytest.fixture(scope="module")
def traj():
    return dict(np.load(GOLDEN))


def _solver(mesh, gas, kw, **extra):
    from wmles_jax_b200 import Solver
    return Solver(mesh, gas, **kw, **extra)


def _Solver(*args, **kw):
    from wmles_jax_b200 import Solver
    return Solver(*args, **kw)


def _l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("path", ["advance", "step"])
@pytest.mark.parametrize("tag", C.TRAJ_CASES)
def test_fp64_trajectory_matches_reference(W, traj, tag, path):
    mesh, gas, kw, prim, t = C.traj_case(W, tag)
    s = _solver(mesh, gas, kw)
    Q = s.init_state(prim)
    ic = np.array([[float(np.sum(q[v].cpu().numpy())) for v in range(5)] for q in Q])
    assert np.array_equal(ic, traj[f"{tag}/ic_sum"]), "initial state differs from the reference's"
    dts = []
    for _ in range(C.TRAJ_STEPS):
        if path == "advance":
            dt = s.max_dt(Q, t)
            Q = s.advance(Q, dt, t)
        else:
            Q, dt = s.step(Q, t)
        dts.append(float(dt))
        t += dts[-1]
    np.testing.assert_allclose(dts, traj[f"{tag}/dts"], rtol=TRAJ_TOL, atol=0)
    for ib, blk in enumerate(mesh.blocks):
        got = blk.interior(Q[ib].cpu().numpy())
        ref = traj[f"{tag}/final{ib}"]
        for c in range(5):
            err = _l2(got[c], ref[c])
            assert err < TRAJ_TOL, (ib, c, err)
    for (bname, face), (tau, _) in s.wall_stats(Q).items():
        ref = traj[f"{tag}/tau/{bname}/{face}"]
        assert np.abs(tau - ref).max() <= 1e-9 * np.abs(ref).max()


@pytest.mark.parametrize("tag", C.SMALL_CASES)
def test_init_state_bit_identical(W, golden, tag):
    """Solver.init_state (wmles/solver.py:54-56) against the reference's initial states."""
    mesh, gas, kw, prim, _ = C.golden_case(W, tag)
    s = _solver(mesh, gas, kw)
    for ib, q in enumerate(s.init_state(prim)):
        assert q.dtype == torch.float64 and q.is_cuda
        assert np.array_equal(q.cpu().numpy(), golden[f"{tag}/q{ib}"])


def _host(q):
    return q.cpu().numpy()


@pytest.mark.parametrize("name", sorted(C.SOD_SCHEMES))
def test_sod_fp64_matches_reference(W, traj, name):
    mesh, Q, dts = C.sod_run(W, _Solver, C.SOD_SCHEMES[name](W), to_host=_host)
    ref_dts = traj[f"sod/{name}/dts"]
    assert len(dts) == len(ref_dts)
    np.testing.assert_allclose(dts, ref_dts, rtol=1e-11, atol=0)
    got, ref = mesh.blocks[0].interior(Q[0]), traj[f"sod/{name}/final"]
    for c in range(5):
        # momentum components against the momentum magnitude: the tube's rho v and rho w are
        # round-off (~1e-17) in the reference, their own maximum is no scale
        scale = np.abs(ref[1:4]).max() if c in (1, 2, 3) else np.abs(ref[c]).max()
        err = np.abs(got[c] - ref[c]).max() / scale
        assert err < 1e-11, (c, err)


@pytest.mark.parametrize("name", sorted(C.SOD_SCHEMES))
def test_sod_mixed_on_plateaus(W, traj, name):
    """The mixed form through the shock, contact and rarefaction (MUSCL positivity fallback
    and HLLC branches active): within 1e-4 of the FP64 reference state, on the exact
    plateaus of tests/test_sod.py:33-36."""
    mesh, Q, dts = C.sod_run(W, _Solver, C.SOD_SCHEMES[name](W), to_host=_host, precision="mixed")
    got, ref = mesh.blocks[0].interior(Q[0]), traj[f"sod/{name}/final"]
    for c in (0, 1, 4):
        err = np.abs(got[c] - ref[c]).max() / np.abs(ref[c]).max()
        assert err < 1e-4, (c, err)
    x = (np.arange(C.SOD_NX) + 0.5) / C.SOD_NX
    i = np.argmin(np.abs(x - 0.75))
    q = got[:, :, 1, 1]
    rho, u = q[0], q[1] / q[0]
    p = 0.4 * (q[4] - 0.5 * rho * u * u)
    assert abs(p[i] - 0.3031) < 2e-3 and abs(u[i] - 0.9275) < 2e-3


def _freestream_scale(mesh, gas):
    """(E + p) |u| max|S| / min V over the box: the size of one face's energy flux per
    volume, against which free-stream round-off is measured."""
    rho, u, v, w, p = C.FREESTREAM_PRIM
    speed = np.sqrt(u * u + v * v + w * w)
    E = p / (gas.gamma - 1.0) + 0.5 * rho * speed ** 2
    g = mesh.geoms[0]
    smax = max(float(np.sqrt(np.sum(np.asarray(S) ** 2, axis=0)).max()) for S in g.S)
    return (E + p) * speed * smax / float(np.asarray(g.vol).min())


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name", sorted(C.FREESTREAM_SCHEMES))
def test_freestream_preserved(W, traj, name, precision):
    mesh = C.freestream_mesh(W)
    gas = W.Gas()
    s = _solver(mesh, gas, dict(scheme=C.FREESTREAM_SCHEMES[name](W), sgs="vreman", cfl=0.5), precision=precision)
    R = s.rhs(s.init_state(C.freestream_prim))
    r = max(float(mesh.blocks[0].interior(R[0])[v].abs().max()) for v in range(5))
    if precision == "fp64":
        assert r < 0.1, r                                   # the reference's bound
        assert float(traj[f"freestream/{name}"]) < 0.1
    else:
        assert r < 1e-6 * _freestream_scale(mesh, gas), (r, _freestream_scale(mesh, gas))


@pytest.mark.parametrize("config,n,steps", [(2, (48, 48, 32), 500), (3, (48, 24, 16), 500)])
def test_mixed_precision_error_bound(config, n, steps):
    """The mixed form against the FP64 form after `steps` steps from the same state: mean
    velocity profile and mean wall shear (averaged over the homogeneous directions) within
    1e-4 relative (max norm), the bound the mixed form is specified to."""
    from wmles_jax_b200.precision_study import compare
    m = compare(config=config, steps=steps, n=n)
    assert m["finite"]
    assert m["mean_velocity_rel_inf"] <= 1e-4, m
    assert m["wall_shear_mean_rel_inf"] <= 1e-4, m
