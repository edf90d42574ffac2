"""Checkpoint / restart of a device state (the (Q, step, time) contract of read_restart,
wmles/io_vtk.py:118-193; driver wiring examples/channel_wmles.py:85-119): k steps, write,
read back, k more steps is bit-identical to 2k steps without the interruption."""
import numpy as np
import pytest

import cases as C

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag,precision", [("cfg2_small", "fp64"), ("ramp_small", "mixed")])
def test_restart_continues_bit_identical(W, tmp_path, tag, precision):
    from wmles_jax_b200 import Solver
    from wmles_jax_b200.restart import read_restart, write_restart
    mesh, gas, kw, prim, t0 = C.traj_case(W, tag)
    s = Solver(mesh, gas, **kw, precision=precision)
    k = 10

    def run(Q, t, n):
        for _ in range(n):
            Q, dt = s.step(Q, t)
            t += float(dt)
        return Q, t

    Q0 = s.init_state(prim)
    Qa, ta = run(Q0, t0, 2 * k)                     # uninterrupted
    Qk, tk = run(Q0, t0, k)
    path = tmp_path / "restart.npz"
    write_restart(path, s, Qk, k, tk)
    del Qk
    Qr, step, tr = read_restart(path, s)
    assert step == k and tr == tk
    Qb, tb = run(Qr, tr, k)
    assert tb == ta
    for blk, a, b in zip(mesh.blocks, Qa, Qb):
        assert torch.equal(blk.interior(a), blk.interior(b))
