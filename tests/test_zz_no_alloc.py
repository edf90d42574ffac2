"""wm_max_dt_noalloc: the CFL time step for callers that cannot allocate device memory.

Such callers (code living inside another framework's memory pool, or under a fixed
device-memory budget) pass the state, the metrics and the output slot; the entry point's
reduction scratch is a static array inside the library.  This test calls it through the C
ABI and checks it against the allocating entry point (wm_max_dt via Solver.max_dt) on two
calls in a row.  The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import cases as C_cases
from oracle.wmles_oracle import OracleSolver, init_state

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_no_alloc_cfl_matches_allocating_entry_point(W):
    from wmles_jax_b200 import Solver, _native as N
    from wmles_jax_b200.lowering import block_metrics

    mesh, gas, kw, prim = C_cases.cfg1_case(W)
    ref = OracleSolver(mesh, gas, **kw)
    solver = Solver(mesh, gas, **kw)
    Q = tuple(torch.from_numpy(q).cuda() for q in init_state(ref, prim))
    # the caller owns every buffer: metrics, state and the output slot
    mets = [torch.from_numpy(np.ascontiguousarray(block_metrics(b, g))).cuda()
            for b, g in zip(mesh.blocks, mesh.geoms)]
    dims = np.array([[*b.n, b.ng] for b in mesh.blocks], dtype=np.int32).ravel()
    gas_c = N.WmGas(gas.gamma, gas.R, gas.Pr, gas.Pr_t, gas.mu_ref, gas.T_ref, gas.S_suth)
    out = torch.full((), float("nan"), dtype=torch.float64, device="cuda")
    lib = N.load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def noalloc(state):
        rc = lib.wm_max_dt_noalloc(len(mesh.blocks), N.as_int_p(dims), N.ptr_array([q.data_ptr() for q in state]),
                                   N.ptr_array([m.data_ptr() for m in mets]), C.byref(gas_c), float(kw["cfl"]),
                                   N.ptr_array([out.data_ptr()])[0], stream)
        N.check(rc, "wm_max_dt_noalloc")
        return float(out)

    states = [Q, solver.step(Q)[0]]           # two calls in a row, on different states
    for state in states:
        got = noalloc(state)
        want = float(solver.max_dt(state))
        assert np.isfinite(got)
        assert abs(got - want) <= 1e-13 * want, (got, want)

    # the property the entry point exists for: once the first call has loaded the library's
    # module (and with it the static array), further calls take no device memory
    ptrs = (N.ptr_array([q.data_ptr() for q in states[1]]), N.ptr_array([m.data_ptr() for m in mets]))
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(5):
        N.check(lib.wm_max_dt_noalloc(len(mesh.blocks), N.as_int_p(dims), ptrs[0], ptrs[1], C.byref(gas_c),
                                      float(kw["cfl"]), N.ptr_array([out.data_ptr()])[0], stream), "wm_max_dt_noalloc")
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before, (free_before, free_after)


def test_no_alloc_rejects_oversized_input():
    from wmles_jax_b200 import _native as N
    lib = N.load()
    n = 4096                                   # 4096^2 x 16 cells: more than the static scratch holds
    dims = np.array([n, n, 16, 3], dtype=np.int32)
    gas_c = N.WmGas(1.4, 287.05, 0.72, 0.9, 1.716e-5, 273.15, 110.4)
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")    # the size check rejects before any read
    p = N.ptr_array([buf.data_ptr()])
    rc = lib.wm_max_dt_noalloc(1, N.as_int_p(dims), p, p, C.byref(gas_c), 0.5, p[0], None)
    assert rc == -1
    assert b"static scratch" in lib.wm_last_error()
    assert torch.all(buf == 0)
