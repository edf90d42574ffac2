"""wm_case_create rejects malformed descriptors before any device call (no GPU needed): a
real descriptor lowered from a golden case passes validation and fails only at the first
CUDA call on a host without a GPU, while each corruption of it returns WM_E_INVALID or
WM_E_UNSUPPORTED.  The ghost-program checks matter most: the gather kernel trusts every
index, so an out-of-range one must never reach the device."""
import ctypes
import os

import pytest

import cases as C

torch = pytest.importorskip("torch")

E_INVALID, E_CUDA, E_UNSUPPORTED = -1, -2, -4


@pytest.fixture()
def lowered(W, monkeypatch):
    if torch.cuda.is_available():
        pytest.skip("checks the path that stops before any device call")
    from wmles_jax_b200 import _native as N
    from wmles_jax_b200 import solver as S
    if not os.path.exists(N.LIB_PATH):
        from wmles_jax_b200.build import build
        build()
    monkeypatch.setattr(S, "require_gpu", lambda: torch.device("cpu"))
    mesh, gas, kw, prim, t = C.golden_case(W, "split_wm_hybrid")
    s = S.Solver.__new__(S.Solver)
    s._prepare(mesh, gas, **kw)
    lib = N.load()

    def create():
        h = ctypes.c_void_p()
        return lib.wm_case_create(ctypes.byref(s._desc), ctypes.byref(h))
    return s, create, lib


def test_valid_descriptor_reaches_the_device_call(lowered):
    s, create, lib = lowered
    assert create() == E_CUDA
    assert b"cuda" in lib.wm_last_error().lower() or lib.wm_last_error()


@pytest.mark.parametrize("field,value,code", [
    ("nblocks", 0, E_INVALID), ("scheme", 7, E_INVALID), ("kep_order", 3, E_INVALID),
    ("sgs", 9, E_INVALID), ("precision", 5, E_INVALID), ("tile", 4, E_INVALID), ("cfl", 0.0, E_INVALID),
    ("cmf_dir", 3, E_INVALID), ("nbc", -1, E_INVALID)])
def test_bad_fields(lowered, field, value, code):
    s, create, lib = lowered
    setattr(s._desc, field, value)
    assert create() == code, lib.wm_last_error()


def test_fp64_tile_and_ghost_layers_unsupported(lowered):
    s, create, lib = lowered
    s._desc.tile = 3                       # built for the mixed form only
    assert create() == E_UNSUPPORTED
    s._desc.tile = -1
    s._desc.blocks[0].ng = 2
    assert create() == E_UNSUPPORTED


def test_bad_wall(lowered):
    s, create, lib = lowered
    s._desc.walls[0].n_match = 10 ** 6
    assert create() == E_INVALID
    s._desc.walls[0].n_match = 1
    s._desc.walls[0].axis = 5
    assert create() == E_INVALID


@pytest.mark.parametrize("prog", ["ghost_rhs", "ghost_all"])
@pytest.mark.parametrize("corrupt", ["dst_cell", "dst_block", "src_cell", "src_kind", "const_id", "ops",
                                     "op_code"])
def test_ghost_program_indices_checked(lowered, prog, corrupt):
    s, create, lib = lowered
    p = getattr(s._desc, prog)
    assert p.count > 0 and p.nops > 0
    if corrupt == "dst_cell":
        p.dst[1] = 10 ** 9
    elif corrupt == "dst_block":
        p.dst[0] = 7
    elif corrupt == "src_cell":
        p.src[1] = -1
    elif corrupt == "src_kind":
        p.src[0] = 9 << 24
    elif corrupt == "const_id":
        p.src[0] = (2 << 24) | 200
    elif corrupt == "ops":
        p.ops[0], p.ops[1] = p.nops, 1
    else:
        p.op_code[0] = 77
    assert create() == E_INVALID, lib.wm_last_error()
    assert prog.encode() in lib.wm_last_error()


def test_inflow_span_limit(W, monkeypatch):
    """The synthetic inflow's row launch keeps a ghost row's three noise fields in 48 KB of
    shared memory: a wider inflow block is refused at creation, not at the first fill."""
    if torch.cuda.is_available():
        pytest.skip("checks the path that stops before any device call")
    from wmles_jax_b200 import _native as N
    from wmles_jax_b200 import solver as S
    if not os.path.exists(N.LIB_PATH):
        from wmles_jax_b200.build import build
        build()
    monkeypatch.setattr(S, "require_gpu", lambda: torch.device("cpu"))
    mesh, gas, kw, prim, t = C.golden_case(W, "ramp_small")
    s = S.Solver.__new__(S.Solver)
    s._prepare(mesh, gas, **kw)
    lib = N.load()
    h = ctypes.c_void_p()
    assert s._desc.inflow
    assert lib.wm_case_create(ctypes.byref(s._desc), ctypes.byref(h)) == E_CUDA
    s._desc.blocks[s._desc.inflow.contents.block].n[2] = 2048
    assert lib.wm_case_create(ctypes.byref(s._desc), ctypes.byref(h)) == E_UNSUPPORTED
    assert b"inflow" in lib.wm_last_error()
