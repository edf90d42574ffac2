"""Plane statistics (PlaneStats, wmles/channel5200.py:121-199) against the reference's own
PlaneStats run on two samples of the small constant-mass-flux channel
(tests/golden/golden_planestats.npz): the oracle on CPU, and the device accumulation of
wmles_jax_b200.stats on a GPU."""
import os

import numpy as np
import pytest

import cases as C
from oracle.wmles_oracle import OracleSolver, plane_means

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden_planestats.npz")
KEYS = ("rho", "u", "v", "w", "uu", "vv", "ww", "uv", "uw", "vw", "T", "p")


@pytest.fixture(scope="module")
def gp():
    return dict(np.load(GOLDEN))


def _states(gp, nb):
    return [tuple(gp[f"q{s}_{ib}"] for ib in range(nb)) for s in (0, 1)]


def test_oracle_plane_means_match_reference(W, gp):
    mesh, gas, kw, prim, t = C.golden_case(W, "channel_small_cmf")
    samples = _states(gp, len(mesh.blocks))
    sums = {k: 0.0 for k in KEYS}
    for Q in samples:
        for k, v in plane_means(gas, mesh.blocks[0], Q[0]).items():
            sums[k] = sums[k] + v
    avg = {k: v / len(samples) for k, v in sums.items()}
    for a, b in (("u", "u"), ("v", "v"), ("w", "w"), ("u", "v"), ("u", "w"), ("v", "w")):
        avg[a + b] = avg[a + b] - avg[a] * avg[b]
    for k in KEYS:
        np.testing.assert_allclose(avg[k], gp[f"avg/{k}"], rtol=1e-12, atol=1e-14, err_msg=k)
    # mean wall shear stress: mean over walls of each wall's mean, averaged over the samples
    o = OracleSolver(mesh, gas, **kw)
    taus = [np.mean([np.mean(v[0]) for v in o.wall_stats(Q).values()]) for Q in samples]
    assert abs(np.mean(taus) - gp["mean_tau_w"]) <= 1e-12 * abs(gp["mean_tau_w"])


@pytest.mark.gpu
def test_device_plane_stats_match_reference(W, gp):
    torch = pytest.importorskip("torch")
    from wmles_jax_b200 import Solver
    from wmles_jax_b200.stats import PlaneStats
    mesh, gas, kw, prim, t = C.golden_case(W, "channel_small_cmf")
    s = Solver(mesh, gas, **kw)
    ps = PlaneStats(mesh, s)
    for Q in _states(gp, len(mesh.blocks)):
        ps.accumulate(tuple(torch.from_numpy(np.ascontiguousarray(q)).cuda() for q in Q))
    y, avg = ps.result()
    np.testing.assert_array_equal(y, gp["y"])
    for k in KEYS:
        np.testing.assert_allclose(avg[k], gp[f"avg/{k}"], rtol=1e-12, atol=1e-14, err_msg=k)
    assert abs(ps.mean_tau_w - gp["mean_tau_w"]) <= 1e-12 * abs(gp["mean_tau_w"])
    u_tau, wu = ps.wall_units(ps.mean_tau_w, 1.0, float(gp["mu_ref"]), 1.0)
    assert abs(u_tau - gp["wu/u_tau"]) <= 1e-12 * gp["wu/u_tau"]
    for k, v in wu.items():
        np.testing.assert_allclose(v, gp[f"wu/{k}"], rtol=1e-9, atol=1e-12, err_msg=k)
