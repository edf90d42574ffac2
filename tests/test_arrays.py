"""The backend's ``xp`` namespace (wmles_jax_b200/arrays.py) and its backend switch, on CPU.

Host arrays must go through NumPy unchanged (bit for bit: initial conditions are compared
with the reference's); torch tensors (CPU tensors here, CUDA tensors on the GPU) select torch
with NumPy's keywords translated.  The driver idioms are those of the reference's channel
example (examples/channel_wmles.py:53-59,141-143)."""
import os
import subprocess
import sys

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from wmles_jax_b200 import _native as N  # noqa: E402
from wmles_jax_b200.arrays import xp  # noqa: E402
from wmles_jax_b200.gas import Gas  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_host_arrays_run_numpy_unchanged():
    x = np.linspace(0.0, 0.02, 11)
    got = xp.clip(xp.minimum(x, 0.02 - x) / 0.01, 1e-3, 1.0)
    want = np.clip(np.minimum(x, 0.02 - x) / 0.01, 1e-3, 1.0)
    assert type(got) is np.ndarray and np.array_equal(got, want)
    st = xp.stack([x, xp.sin(x), xp.cos(x)])
    assert type(st) is np.ndarray and np.array_equal(st, np.stack([x, np.sin(x), np.cos(x)]))
    assert xp.pi == np.pi and xp.float64 is np.float64


def test_tensors_select_torch():
    rng = np.random.default_rng(1)
    a = rng.normal(size=(5, 6, 7, 8)) + 3.0
    t = torch.from_numpy(a)
    # the reference driver's reductions on a state
    assert float(xp.min(t[0])) == a[0].min()
    ke_t = float(xp.sum(0.5 * xp.sum(t[1:4] ** 2, axis=0) / t[0]))
    ke_n = float(np.sum(0.5 * np.sum(a[1:4] ** 2, axis=0) / a[0]))
    assert abs(ke_t - ke_n) <= 1e-12 * abs(ke_n)
    assert isinstance(xp.sum(t, axis=(1, 2)), torch.Tensor) and tuple(xp.sum(t, axis=(1, 2)).shape) == (5, 8)
    assert tuple(xp.max(t, axis=0).shape) == (6, 7, 8) and tuple(xp.mean(t, axis=-1, keepdims=True).shape) == (5, 6, 7, 1)
    assert torch.equal(xp.clip(t, 2.0, 4.0), torch.clamp(t, 2.0, 4.0))
    assert torch.equal(xp.minimum(t, 3.0), torch.clamp(t, max=3.0))
    assert torch.equal(xp.where(t > 3.0, 1.0, t), torch.where(t > 3.0, 1.0, t))
    assert torch.equal(xp.stack([t[0], t[1]]), torch.stack([t[0], t[1]]))
    assert torch.allclose(xp.sqrt(t.abs()), torch.sqrt(t.abs())) and xp.asarray(t, dtype=xp.float32).dtype == torch.float32
    # NumPy arrays mixed with a tensor are moved to the tensor's device and dtype
    w = np.ones((6, 7, 8))
    assert torch.equal(xp.maximum(t[0], w), torch.maximum(t[0], torch.ones(6, 7, 8, dtype=t.dtype)))


def test_gas_on_tensors_and_arrays():
    gas = Gas()
    w = np.stack([np.full(4, 1.2), np.full(4, 30.0), np.zeros(4), np.full(4, -5.0), np.full(4, 1e5)])
    q = gas.prim_to_cons(w)
    assert type(q) is np.ndarray
    w2, T = gas.cons_to_prim(torch.from_numpy(q))
    assert isinstance(w2, torch.Tensor) and torch.allclose(w2, torch.from_numpy(w), rtol=1e-14, atol=0)
    assert abs(float(gas.sound_speed(300.0)) - np.sqrt(1.4 * 287.05 * 300.0)) < 1e-12


def test_backend_switch_other_than_cuda_refuses_the_solver():
    code = ("import wmles_jax_b200.backend as b\n"
            "try:\n    b.require_gpu()\nexcept RuntimeError as e:\n    print('refused:', e)\n")
    env = dict(os.environ, WMLES_BACKEND="numpy", PYTHONPATH=ROOT)
    out = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=300)
    assert "refused:" in out.stdout and "WMLES_BACKEND=numpy" in out.stdout, out.stdout + out.stderr


def test_backend_helpers():
    from wmles_jax_b200.backend import fori_loop, jit, set_at
    a = np.zeros(4)
    b = set_at(a, 1, 5.0)
    assert a[1] == 0.0 and b[1] == 5.0
    t = torch.zeros(4)
    u = set_at(t, 2, 3.0)
    assert float(t[2]) == 0.0 and float(u[2]) == 3.0
    assert fori_loop(0, 4, lambda i, x: x + i, 0) == 6
    f = lambda x: x + 1  # noqa: E731
    assert jit(f) is f


def test_status_bits_decode():
    assert N.status_names(0) == []
    assert N.status_names(N.ST_NONFINITE | N.ST_PRESSURE) == ["non-finite state", "non-positive pressure"]
    assert N.ST_FATAL & N.ST_WALL == 0
    assert issubclass(N.NonFiniteStateError, RuntimeError)
