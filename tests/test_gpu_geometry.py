"""Mesh metrics on the device (wm_block_geometry, Mesh.finalize(device=True)) against the
host restatement of wmles/mesh.py:53-73 and the host packing of the metric table.

Tolerances: the Geom arrays (vol, xc, S, xf) bit-identical (compared as 64-bit patterns);
the packed table bit-identical except the filter width V^(1/3), within 4 ulp (device pow
against the C library's).  A solver built on device metrics steps like one built on host
metrics: within 1e-13 of the field's max after three FP64 steps, 1e-9 in the mixed form
(there a few-ulp change of V^(1/3) may move the rounding of its FP32 copy).
"""
import numpy as np
import pytest

import cases as C

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DELTA = 13          # WM_MET_DELTA


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float64).view(np.uint64)


@pytest.mark.parametrize("tag", C.SMALL_CASES)
def test_block_geometry_matches_host(W, tag):
    from wmles_jax_b200.device_geometry import block_geometry
    from wmles_jax_b200.lowering import _block_metrics
    mesh, gas, kw, prim, t = C.golden_case(W, tag)
    for b in mesh.blocks:
        (vol, xc, S, xf), met = block_geometry(b.X)
        g = b.geom
        assert np.array_equal(_bits(vol), _bits(g.vol)), (b.name, "vol")
        assert np.array_equal(_bits(xc), _bits(g.xc)), (b.name, "xc")
        for d in range(3):
            assert np.array_equal(_bits(S[d]), _bits(g.S[d])), (b.name, "S", d)
            assert np.array_equal(_bits(xf[d]), _bits(g.xf[d])), (b.name, "xf", d)
        ref = _block_metrics(b, g)
        got = met.cpu().numpy()
        assert got.shape == ref.shape
        for m in range(ref.shape[0]):
            if m == DELTA:
                assert np.all(np.abs(got[m] - ref[m]) <= 4 * np.spacing(ref[m])), (b.name, m)
            else:
                assert np.array_equal(_bits(got[m]), _bits(ref[m])), (b.name, m)


def test_cgrid_finalize_on_device_keeps_tables(W):
    """The four-block C-grid (reversed and transposed interfaces): finalize(device=True)
    gives the host Geom bits and leaves one device table per block for the solver."""
    from wmles_jax_b200.lowering import block_metrics
    mesh, gas, kw, prim, t = C.golden_case(W, "naca_small")
    host = [(b.geom.vol.copy(), b.geom.xc.copy()) for b in mesh.blocks]
    mesh.finalize(device=True)
    for b, (vol, xc) in zip(mesh.blocks, host):
        assert np.array_equal(_bits(b.geom.vol), _bits(vol))
        assert np.array_equal(_bits(b.geom.xc), _bits(xc))
        m = block_metrics(b, b.geom)
        assert isinstance(m, torch.Tensor) and m.is_cuda and m.shape == (27,) + b.geom.vol.shape
    mesh.release_device_metrics()
    assert all(b.metrics_dev is None for b in mesh.blocks)
    assert isinstance(block_metrics(mesh.blocks[0], mesh.blocks[0].geom), np.ndarray)


def _run(mesh, gas, kw, Qh, t, precision, steps=3):
    from wmles_jax_b200 import Solver
    s = Solver(mesh, gas, **kw, precision=precision)
    Q = tuple(torch.from_numpy(np.ascontiguousarray(q)).cuda() for q in Qh)
    for _ in range(steps):
        Q, dt = s.step(Q, t)
        t += float(dt)
    return [q.cpu().numpy() for q in Q]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-13), ("mixed", 1e-9)])
@pytest.mark.parametrize("tag", ["split_wm_hybrid", "naca_small", "rotcyc_slip_kep4"])
def test_solver_on_device_metrics(W, golden, tag, precision, tol):
    mesh, gas, kw, prim, t = C.golden_case(W, tag)
    Qh = tuple(golden[f"{tag}/q{ib}"] for ib in range(len(mesh.blocks)))
    ref = _run(mesh, gas, kw, Qh, t, precision)
    mesh.finalize(device=True)
    got = _run(mesh, gas, kw, Qh, t, precision)
    for ib, blk in enumerate(mesh.blocks):
        a, b = blk.interior(got[ib]), blk.interior(ref[ib])
        for c in range(5):
            err = np.abs(a[c] - b[c]).max() / np.abs(b[c]).max()
            assert err <= tol, (tag, precision, ib, c, err)


def test_block_geometry_rejects_bad_arguments():
    import ctypes
    from wmles_jax_b200 import _native as N
    lib = N.load()
    x = torch.zeros(3, 3, 3, 3, dtype=torch.float64, device="cuda")
    p = ctypes.cast(ctypes.c_void_p(x.data_ptr()), N.c_double_p)
    faces = N.ptr_array([x.data_ptr()] * 3)
    assert lib.wm_block_geometry(p, (ctypes.c_int * 3)(2, 0, 2), p, p, faces, faces, None, None) == -1
    assert lib.wm_block_geometry(None, (ctypes.c_int * 3)(2, 2, 2), p, p, faces, faces, None, None) == -1
    assert lib.wm_block_geometry(p, (ctypes.c_int * 3)(2, 2, 2), p, p, N.ptr_array([x.data_ptr(), 0, 0]),
                                 faces, None, None) == -1
