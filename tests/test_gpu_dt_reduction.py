"""The CFL reduction's NaN handling and per-case independence.

The time step is the minimum over a case's cells, taken with one 64-bit atomicMin per warp
on an order-preserving key of the case; a NaN gets the lowest key, so a NaN cell gives a
NaN time step as np.min does (the reference's Solver._dt, wmles/solver.py:135-151).  The
keys are reset by the launch's last CTA, so the next call starts clean.  In a batch each
case has its own key: one case's NaN leaves the others' time steps bit-identical.
"""
import math

import numpy as np
import pytest

import cases as C

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _dev(Q):
    return tuple(torch.from_numpy(np.ascontiguousarray(q)).cuda() for q in Q)


def _poison(Q, blk, value=float("nan")):
    """Copy of Q with one interior cell's density set to `value`."""
    out = tuple(q.clone() for q in Q)
    ng = blk.ng
    i, j, k = ng + blk.n[0] // 2, ng + blk.n[1] // 2, ng + blk.n[2] // 2
    out[0][0, i, j, k] = value
    return out


def test_nan_cell_gives_nan_dt_and_the_next_call_is_clean(W, golden):
    from wmles_jax_b200 import Solver
    tag = "split_wm_hybrid"
    mesh, gas, kw, prim, t = C.golden_case(W, tag)
    s = Solver(mesh, gas, **kw)
    Q = _dev(tuple(golden[f"{tag}/q{ib}"] for ib in range(len(mesh.blocks))))
    dt0 = float(s.max_dt(Q))
    assert math.isfinite(dt0) and dt0 > 0.0
    assert math.isnan(float(s.max_dt(_poison(Q, mesh.blocks[0]))))
    assert math.isnan(float(s.max_dt(_poison(Q, mesh.blocks[-1]))))
    # the per-case key was reset after the NaN call: the same bits as before
    assert float(s.max_dt(Q)) == dt0
    assert float(s.max_dt(Q)) == dt0


def test_nan_in_one_case_of_a_batch_leaves_the_others(W, golden):
    from wmles_jax_b200 import Solver
    from wmles_jax_b200.serving import Batch
    tag = "single_slip_kep4"
    solvers, states = [], []
    for _ in range(3):
        mesh, gas, kw, prim, t = C.golden_case(W, tag)
        solvers.append(Solver(mesh, gas, **kw))
        states.append(_dev(tuple(golden[f"{tag}/q{ib}"] for ib in range(len(mesh.blocks)))))
    blk = mesh.blocks[0]
    dts_alone = [s.max_dt(q) for s, q in zip(solvers, states)]
    batch = Batch(solvers)
    try:
        q_in = [states[0], _poison(states[1], blk), states[2]]
        q_out = [tuple(torch.empty_like(x) for x in q) for q in q_in]
        dt_in = [d.clone() for d in dts_alone]
        dt_next = [torch.empty_like(d) for d in dts_alone]
        batch.step(q_in, q_out, dt_in, dt_next)
        torch.cuda.synchronize()
        # the same step alone for the clean cases
        for c in (0, 2):
            Q1, _ = solvers[c].step(states[c])
            ref = solvers[c].max_dt(Q1)
            assert torch.equal(dt_next[c], ref), f"case {c}: dt changed by another case's NaN"
        assert math.isnan(float(dt_next[1]))
    finally:
        batch.close()
