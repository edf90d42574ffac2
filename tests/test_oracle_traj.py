"""Pin the CPU oracle to the reference's own multi-step runs (tests/golden/golden_traj.npz,
written by tests/golden/make_golden.py from the reference's NumPy float64 path).

* 100 steps of the reduced config-2 channel, the small smooth ramp and the NACA C-grid with
  the drivers' loop (examples/channel_wmles.py:124-126): every dt within 1e-12 and the final
  state within 1e-12 relative L2 per conservative variable;
* the Sod tube of tests/test_sod.py:7-28 (MUSCL-HLLC and Hybrid, to t = 0.2): same number of
  steps, final state within 1e-12;
* free-stream preservation on the skewed box (tests/test_multiblock.py:100-107): below the
  reference's bound of 0.1.
"""
import os

import numpy as np
import pytest

import cases as C
from oracle.wmles_oracle import OracleSolver, init_state

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_traj.npz")


@pytest.fixture(scope="module")
def traj():
    return dict(np.load(GOLDEN))


def _l2(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("tag", C.TRAJ_CASES)
def test_oracle_trajectory(W, traj, tag):
    mesh, gas, kw, prim, t = C.traj_case(W, tag)
    s = OracleSolver(mesh, gas, **kw)
    Q = init_state(s, prim)
    ic = np.array([[float(np.sum(q[v])) for v in range(5)] for q in Q])
    assert np.array_equal(ic, traj[f"{tag}/ic_sum"])
    dts = traj[f"{tag}/dts"]
    for n in range(C.TRAJ_STEPS):
        dt = s.max_dt(Q, t)
        assert abs(dt - dts[n]) <= 1e-12 * dts[n], (n, dt, dts[n])
        Q = s.advance(Q, dt, t)
        t += dt
    for ib, (blk, q) in enumerate(zip(mesh.blocks, Q)):
        ref = traj[f"{tag}/final{ib}"]
        for c in range(5):
            assert _l2(blk.interior(q)[c], ref[c]) < 1e-12, (ib, c)


@pytest.mark.parametrize("name", sorted(C.SOD_SCHEMES))
def test_oracle_sod(W, traj, name):
    mesh, Q, dts = C.sod_run(W, OracleSolver, C.SOD_SCHEMES[name](W), init=init_state)
    assert len(dts) == len(traj[f"sod/{name}/dts"])
    np.testing.assert_allclose(dts, traj[f"sod/{name}/dts"], rtol=1e-12)
    got, ref = mesh.blocks[0].interior(Q[0]), traj[f"sod/{name}/final"]
    for c in range(5):
        scale = np.abs(ref[1:4]).max() if c in (1, 2, 3) else np.abs(ref[c]).max()
        assert np.abs(got[c] - ref[c]).max() <= 1e-12 * scale, c


def test_reference_sod_plateaus(traj):
    """The reference's Sod states sit on the exact plateaus its test prints
    (tests/test_sod.py:33-36): p 0.3031, u 0.9275 at x = 0.75."""
    x = (np.arange(C.SOD_NX) + 0.5) / C.SOD_NX
    i = np.argmin(np.abs(x - 0.75))
    for name in C.SOD_SCHEMES:
        q = traj[f"sod/{name}/final"][:, :, 1, 1]
        rho, u = q[0], q[1] / q[0]
        p = 0.4 * (q[4] - 0.5 * rho * u * u)
        assert abs(p[i] - 0.3031) < 2e-3 and abs(u[i] - 0.9275) < 2e-3


@pytest.mark.parametrize("name", sorted(C.FREESTREAM_SCHEMES))
def test_oracle_freestream(W, traj, name):
    mesh = C.freestream_mesh(W)
    s = OracleSolver(mesh, W.Gas(), C.FREESTREAM_SCHEMES[name](W), sgs="vreman", cfl=0.5)
    R = s.rhs(init_state(s, C.freestream_prim))
    r = max(float(np.abs(mesh.blocks[0].interior(R[0])[v]).max()) for v in range(5))
    assert r < 0.1
    assert float(traj[f"freestream/{name}"]) < 0.1
