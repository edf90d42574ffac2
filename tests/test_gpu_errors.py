"""Error paths at the C boundary with a live case: null per-block pointers are rejected
before any launch (a null state pointer would otherwise become a device fault), and the
case stays usable afterwards."""
import ctypes

import pytest

import cases as C

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_null_block_pointers_rejected(W):
    from wmles_jax_b200 import Solver
    from wmles_jax_b200 import _native as N
    from wmles_jax_b200.serving import Batch
    mesh, gas, kw, prim, t = C.golden_case(W, "split_slip_kep4")
    s = Solver(mesh, gas, **kw)
    Q = s.init_state(prim)
    out = tuple(torch.empty_like(q) for q in Q)
    dt, dn = s.max_dt(Q), torch.empty((), dtype=torch.float64, device="cuda")
    lib, stream = N.load(), s._stream()
    one = N.ptr_array([dt.data_ptr()])[0]
    two = N.ptr_array([dn.data_ptr()])[0]
    holey = N.ptr_array([Q[0].data_ptr(), 0])
    assert lib.wm_step_fused(s._case, holey, s._ptrs(out), one, two, 0.0, stream) == -1
    assert b"q_in[1]" in lib.wm_last_error()
    assert lib.wm_rhs(s._case, s._ptrs(Q), N.ptr_array([out[0].data_ptr(), 0]), 0.0, stream) == -1
    assert lib.wm_apply_bcs(s._case, None, 0.0, stream) == -1
    b = Batch([s])
    qi, qo, di, dnx, tt = b.args([Q], [out], [dt], [dn])
    assert lib.wm_batch_step(b._h, qi, qo, N.ptr_array([0]), dnx, N.as_double_p(tt), stream) == -1
    b.close()
    # the case still steps correctly
    Q1, _ = s.step(Q)
    torch.cuda.synchronize()
    assert all(bool(torch.isfinite(q[:, 3:-3, 3:-3, 3:-3]).all()) for q in Q1)
