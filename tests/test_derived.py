"""Derived output fields (derived_fields, wmles/io_vtk.py:269-293) against the reference's own
derived_fields on two golden states (tests/golden/golden_derived.npz): the oracle on CPU and
the device kernel behind wm_derived_fields on a GPU.  Tolerance: 1e-11 of each field's max
(FP64 Green-Gauss gradients; Q-criterion and mu_t are differences / ratios of them)."""
import os

import numpy as np
import pytest

import cases as C
from oracle.wmles_oracle import OracleSolver, derived_fields as oracle_derived

HERE = os.path.dirname(os.path.abspath(__file__))
TAGS = ("split_wm_hybrid", "naca_small")
TOL = 1e-11


@pytest.fixture(scope="module")
def gd():
    return dict(np.load(os.path.join(HERE, "golden", "golden_derived.npz")))


def _check(got, gd, tag):
    for ib, fields in got.items():
        for k, v in fields.items():
            ref = gd[f"{tag}/{ib}/{k}"]
            err = np.abs(np.asarray(v) - ref).max() / max(np.abs(ref).max(), 1e-300)
            assert err < TOL, (tag, ib, k, err)


@pytest.mark.parametrize("tag", TAGS)
def test_oracle_derived_fields(W, golden, gd, tag):
    mesh, gas, kw, prim, t = C.golden_case(W, tag)
    Q = tuple(golden[f"{tag}/q{ib}"] for ib in range(len(mesh.blocks)))
    _check(oracle_derived(OracleSolver(mesh, gas, **kw), Q), gd, tag)


@pytest.mark.gpu
@pytest.mark.parametrize("tag", TAGS)
def test_device_derived_fields(W, golden, gd, tag):
    torch = pytest.importorskip("torch")
    from wmles_jax_b200 import Solver
    from wmles_jax_b200.output import derived_fields
    mesh, gas, kw, prim, t = C.golden_case(W, tag)
    s = Solver(mesh, gas, **kw)
    Q = tuple(torch.from_numpy(np.ascontiguousarray(golden[f"{tag}/q{ib}"])).cuda() for ib in range(len(mesh.blocks)))
    _check(derived_fields(s, Q), gd, tag)
