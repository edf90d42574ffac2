"""Mesh.finalize(device=True) on the host side: malformed node arrays are rejected before any
device call, and without a GPU the device path fails loudly instead of falling back to the
host metrics."""
import numpy as np
import pytest

import cases as C

torch = pytest.importorskip("torch")


def test_bad_node_array_rejected_before_the_device():
    from wmles_jax_b200.device_geometry import block_geometry
    for shape in [(3, 4, 4), (2, 4, 4, 4), (3, 1, 4, 4)]:
        with pytest.raises(ValueError):
            block_geometry(np.zeros(shape))


def test_device_finalize_without_gpu_fails_loudly(W):
    if torch.cuda.is_available():
        pytest.skip("checks the host without a GPU")
    mesh, gas, kw, prim, t = C.golden_case(W, "single_slip_kep4")
    with pytest.raises(RuntimeError, match="CUDA device"):
        mesh.finalize(device=True)
