"""Restart files round-trip a multiblock state exactly and refuse a mismatching solver."""
import types

import numpy as np
import pytest

import cases as C

torch = pytest.importorskip("torch")


def _fake_solver(mesh):
    return types.SimpleNamespace(blocks=mesh.blocks, device=torch.device("cpu"))


def test_round_trip_and_checks(W, tmp_path):
    from wmles_jax_b200.restart import read_restart, write_restart
    mesh = C.skew_case(W, "split")
    s = _fake_solver(mesh)
    rng = np.random.default_rng(3)
    Q = tuple(torch.from_numpy(rng.normal(size=(5,) + tuple(b.N))) for b in mesh.blocks)
    path = tmp_path / "chk.npz"
    write_restart(path, s, Q, 1234, 5.5e-3)
    Q2, step, time = read_restart(path, s)
    assert step == 1234 and time == 5.5e-3
    assert all(torch.equal(a, b) for a, b in zip(Q, Q2))
    other = _fake_solver(C.skew_case(W, "single"))
    with pytest.raises(ValueError):
        read_restart(path, other)
    with pytest.raises(ValueError):
        write_restart(path, s, Q[:1], 0, 0.0)
