"""Synthetic inflow fills on the device against the oracle (SmoothRampInflow.fill_at_time,
wmles/smooth_ramp.py:150-197).  The smooth ramp's inflow plane is extruded (z a function of
k alone, y constant along k), which selects the factored mode sums (one sincos per mode and
ghost row); shearing the span with height makes it general, which selects one cosine per
mode and ghost cell.  Both are checked at several times, the latest one with mode arguments
in the hundreds (the factored sums round the argument as two parts)."""
import numpy as np
import pytest

import cases as C
from oracle.wmles_oracle import OracleSolver, init_state

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("skew", [0.0, 0.2])
def test_inflow_fill_matches_oracle(W, skew):
    from wmles_jax_b200 import Solver
    mesh, gas, props, profile, kw = C.ramp_case(W, skew_z=skew)
    ref = OracleSolver(mesh, gas, **kw)
    Qh = init_state(ref, C.ramp_prim(props, profile))
    gpu = Solver(mesh, gas, **kw)
    Q = tuple(torch.from_numpy(np.ascontiguousarray(q)).cuda() for q in Qh)
    ng = mesh.blocks[0].ng
    T = props["L"] / props["U_inf"]
    for t in (0.0, 0.37 * T, 40.0 * T):
        want = ref.apply_bcs(Qh, t)[0][:, :ng]
        got = gpu.apply_bcs(Q, time=t)[0][:, :ng].cpu().numpy()
        for c in range(5):
            err = np.abs(got[c] - want[c]).max() / np.abs(want[c]).max()
            assert err < 1e-11, (t, c, err)
