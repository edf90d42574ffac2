"""CPU checks of the host lowering: the traced ghost-cell programs reproduce the
reference's ghost fill bit for bit, and the metric/wall-geometry packing is consistent."""
import numpy as np
import pytest

import cases as C
from oracle.wmles_oracle import (OracleSolver, init_state, slip_map, noslip_map, farfield_map,
                                 inflow_fill)
from wmles_jax_b200.lowering import (lower_ghost_programs, rhs_ghost_mask, block_metrics,
                                     SRC_CELL, SRC_INFLOW, SRC_CONST, OP_SLIP, OP_NOSLIP, OP_FARFIELD)
from wmles_jax_b200.smooth_ramp import SmoothRampInflow


def run_program(prog, table, gas, Q, inflow=None):
    """Execute a ghost program on host arrays with the oracle's per-cell maps
    (the same arithmetic the device kernel performs)."""
    out = [q.copy() for q in Q]
    n = prog.count
    kind = prog.src[:, 0] >> 24
    sb = prog.src[:, 0] & 0xFFFFFF
    val = np.zeros((5, n))
    for ib, q in enumerate(Q):
        m = (kind == SRC_CELL) & (sb == ib)
        val[:, m] = q.reshape(5, -1)[:, prog.src[m, 1]]
    m = kind == SRC_INFLOW
    if m.any():
        for ib in np.unique(sb[m]):
            mm = m & (sb == ib)
            val[:, mm] = inflow[ib].reshape(5, -1)[:, prog.src[mm, 1]]
    m = kind == SRC_CONST
    val[:, m] = table[sb[m], :5].T
    start, depth = prog.ops[:, 0], prog.ops[:, 1]
    for level in range(int(depth.max()) if n else 0):
        has = depth > level
        code = prog.op_code[start[has] + level]
        nrm = prog.op_nrm[start[has] + level].T
        sub = val[:, has]
        res = sub.copy()
        for c in np.unique(code):
            sel = code == c
            op, bc, side = c & 0xFF, (c >> 8) & 0xFF, (c >> 16) & 1
            if op == OP_SLIP:
                res[:, sel] = slip_map(gas, sub[:, sel], nrm[:, sel])
            elif op == OP_NOSLIP:
                Tw = table[bc, 5] if table[bc, 6] else None
                res[:, sel] = noslip_map(gas, sub[:, sel], Tw)
            elif op == OP_FARFIELD:
                res[:, sel] = farfield_map(gas, sub[:, sel], nrm[:, sel], table[bc, :5], side)
        val[:, has] = res
    for ib in range(len(Q)):
        m = prog.dst[:, 0] == ib
        out[ib].reshape(5, -1)[:, prog.dst[m, 1]] = val[:, m]
    return out


def _inflow_values(solver, Q, t):
    """Oracle inflow ghost values per block (the device computes them in a separate kernel)."""
    res = {}
    for ib, blk in enumerate(solver.blocks):
        bc = blk.faces.get((0, 0))
        if isinstance(bc, SmoothRampInflow):
            res[ib] = inflow_fill(bc, solver.gas, np.zeros_like(Q[ib]), blk, solver.geoms[ib], t)
    return res


@pytest.mark.parametrize("tag", C.SMALL_CASES)
def test_ghost_program_matches_reference_fill(W, golden, tag):
    mesh, gas, kw, prim, t = C.golden_case(W, tag)
    solver = OracleSolver(mesh, gas, **kw)
    Q = tuple(golden[f"{tag}/q{ib}"] for ib in range(len(mesh.blocks)))
    prog_rhs, prog_all, table = lower_ghost_programs(mesh.blocks, mesh.geoms, gas, 2)
    inflow = _inflow_values(solver, Q, t)
    full = run_program(prog_all, table, gas, Q, inflow)
    for ib in range(len(Q)):
        ref = golden[f"{tag}/bcs{ib}"]
        if inflow:   # inflow values: cos() of the oracle vs the reference agree to round-off
            np.testing.assert_allclose(full[ib], ref, rtol=1e-13, atol=0)
        else:
            assert np.array_equal(full[ib], ref), f"block {ib}"
    # the RHS program writes exactly the needed subset, with the same values
    part = run_program(prog_rhs, table, gas, Q, inflow)
    for ib, blk in enumerate(mesh.blocks):
        need = rhs_ghost_mask(blk)
        assert np.array_equal(part[ib][:, need], full[ib][:, need])
        assert int(need.sum()) == int((prog_rhs.dst[:, 0] == ib).sum())


def test_cfg1_programs_cover_needed_cells(W):
    mesh, gas, kw, prim = C.cfg1_case(W)
    prog_rhs, prog_all, table = lower_ghost_programs(mesh.blocks, mesh.geoms, gas, 2)
    solver = OracleSolver(mesh, gas, **kw)
    Q = init_state(solver, prim)
    ref = solver.apply_bcs(Q)
    got = run_program(prog_all, table, gas, Q)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


def test_metric_packing(W):
    mesh = C.skew_case(W, "flip")
    for blk, g in zip(mesh.blocks, mesh.geoms):
        M = block_metrics(blk, g)
        Ni, Nj, Nk = blk.N
        assert M.shape == (27,) + blk.N
        assert np.array_equal(M[0:3], g.S[0][:, :Ni])
        assert np.array_equal(M[5], g.S[1][2, :, :Nj])
        assert np.array_equal(M[13], g.vol ** (1.0 / 3.0))
