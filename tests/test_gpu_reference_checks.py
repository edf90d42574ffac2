"""The reference's own physical checks of tests/test_multiblock.py, run on the CUDA path.

* characteristic far field (tests/test_multiblock.py:110-131): supersonic inflow takes the
  free stream, supersonic outflow the interior state, a subsonic boundary at the free
  stream keeps it; ghost primitives within 1e-12 relative, the reference's tolerance;
* wall-model self-consistency (tests/test_multiblock.py:134-149): a uniform stream at the
  speed Spalding's law gives for a chosen friction velocity at the first cell centre; the
  device wall model recovers that friction velocity within the reference's 1e-6 (and within
  1e-9 relative), on an isothermal and on an adiabatic wall;
* wall-load integration (tests/test_multiblock.py:161-190): uniform stream in a unit box
  with wall-modelled j faces; force and moment per face against the closed forms;
* multiblock consistency (tests/test_multiblock.py:88-98,216-219): two-block splits, and a
  periodic chain of eight blocks, give the single block's RHS cell by cell;
* sponge mean preservation (tests/test_smooth_ramp.py:74-96);
* device placement (tests/test_multiblock.py:152-157): metrics and states on the device.

The expected values are closed forms, an independent bisection written here or the single
block's own result, not the oracle.
"""
import numpy as np
import pytest

import cases as C

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _Solver(*args, **kw):
    from wmles_jax_b200 import Solver
    return Solver(*args, **kw)


# ----------------------------------------------------------------------- far field
FF_CASES = [
    # interior primitives, side (0 = jmin, 1 = jmax), expected ghost primitives
    ("supersonic_inflow", [1.0, 0.0, 500.0, 0.0, 8e4], 0, None),
    ("supersonic_outflow", [1.0, 0.0, 1000.0, 0.0, 8e4], 1, [1.0, 0.0, 1000.0, 0.0, 8e4]),
    ("subsonic_free_stream_min", None, 0, None),
    ("subsonic_free_stream_max", None, 1, None),
]
PRIM_INF = np.array([1.2, 10.0, 0.0, 0.0, 1e5])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("name,prim,side,expected", FF_CASES, ids=[c[0] for c in FF_CASES])
def test_characteristic_farfield_regimes(W, name, prim, side, expected, precision):
    n = (12, 10, 8)
    ix, iy, iz = (np.arange(m + 1) for m in n)
    blk = W.Block("ff", C.skew_nodes(ix, iy, iz, n))
    mesh = W.Mesh([blk])
    mesh.connect(blk, "imin", blk, "imax", shift=(-C.LBOX[0], 0, 0))
    mesh.connect(blk, "kmin", blk, "kmax", shift=(0, 0, -C.LBOX[2]))
    blk.set_bc("jmin", W.CharacteristicFarfield(PRIM_INF))
    blk.set_bc("jmax", W.CharacteristicFarfield(PRIM_INF))
    mesh.finalize()
    gas = W.Gas()
    s = _Solver(mesh, gas, W.KEP(2), sgs=None, precision=precision)
    state = PRIM_INF if prim is None else np.asarray(prim, float)
    want = PRIM_INF if expected is None else np.asarray(expected, float)
    Q = s.init_state(lambda xc: state.reshape(5, 1, 1, 1) * np.ones((1,) + xc.shape[1:]))
    assert Q[0].device.type == "cuda"
    F = s.apply_bcs(Q)
    ng, nj = blk.ng, blk.n[1]
    gj = ng - 1 if side == 0 else ng + nj
    ghost = F[0][:, ng, gj, ng].cpu().numpy()
    got = np.asarray(gas.cons_to_prim(ghost)[0])
    np.testing.assert_allclose(got, want, rtol=1e-12)


# ----------------------------------------------------------------------- wall model
def _spalding_yplus(up, kappa, B):
    ku = kappa * up
    return up + np.exp(-kappa * B) * (np.exp(ku) - 1.0 - ku - ku ** 2 / 2.0 - ku ** 3 / 6.0)


def _utau_bisection(U, h, nu, kappa, B):
    """u_tau with Spalding's y+(U/u_tau) = h u_tau / nu, by bisection on u_tau (the left side
    falls and the right side grows with u_tau)."""
    lo, hi = 1e-9, U
    for _ in range(300):
        mid = 0.5 * (lo + hi)
        g = _spalding_yplus(U / mid, kappa, B) - h * mid / nu
        lo, hi = (mid, hi) if g > 0 else (lo, mid)
    return 0.5 * (lo + hi)


@pytest.mark.parametrize("wall", ["isothermal", "adiabatic"])
def test_wall_model_recovers_spalding_utau(W, wall):
    gas = W.Gas()
    n, dy = (6, 8, 6), 0.006
    axes = [np.arange(n[0] + 1) * 0.01, np.arange(n[1] + 1) * dy, np.arange(n[2] + 1) * 0.01]
    blk = W.Block("wm", np.stack(np.meshgrid(*axes, indexing="ij")))
    mesh = W.Mesh([blk])
    mesh.connect(blk, "imin", blk, "imax", shift=(-0.01 * n[0], 0, 0))
    mesh.connect(blk, "kmin", blk, "kmax", shift=(0, 0, -0.01 * n[2]))
    model = W.EquilibriumWallModel()
    T_h, p = 300.0, 1e5
    T_wall = 300.0 if wall == "isothermal" else None
    blk.set_bc("jmin", W.WallModel(model, T_wall=T_wall, n_match=1))
    blk.set_bc("jmax", W.SlipWall())
    mesh.finalize()
    s = _Solver(mesh, gas, W.KEP(2), sgs=None)

    U = 39.0
    rho = p / (gas.R * T_h)
    T_w = T_h if T_wall is not None else T_h + gas.Pr ** (1.0 / 3.0) * U ** 2 / (2.0 * gas.cp)
    rho_w = p / (gas.R * T_w)
    nu_w = float(gas.mu(T_w)) / rho_w
    h = 0.5 * dy                                            # first cell centre over the wall
    ut = _utau_bisection(U, h, nu_w, model.kappa, model.B)

    prim = np.array([rho, U, 0.0, 0.0, p])
    Q = s.init_state(lambda xc: prim.reshape(5, 1, 1, 1) * np.ones((1,) + xc.shape[1:]))
    tau, qw = s.wall_stats(Q)[("wm", "jmin")]
    got = np.sqrt(tau / rho_w)
    assert np.all(np.abs(got - ut) < 1e-6), (got.min(), got.max(), ut)   # the reference's bound
    np.testing.assert_allclose(got, ut, rtol=1e-9)
    if T_wall is None:
        assert np.all(qw == 0.0)


# ----------------------------------------------------------------------- wall loads
def test_wall_load_integration(W):
    gas = W.Gas()
    axes = [np.linspace(0.0, 1.0, 5)] * 3
    blk = W.Block("wall", np.stack(np.meshgrid(*axes, indexing="ij")))
    mesh = W.Mesh([blk])
    for face in ("imin", "imax", "jmin", "jmax", "kmin", "kmax"):
        blk.set_bc(face, W.SlipWall())
    blk.set_bc("jmin", W.WallModel(W.EquilibriumWallModel(), T_wall=300.0))
    blk.set_bc("jmax", W.WallModel(W.EquilibriumWallModel(), T_wall=300.0))
    mesh.finalize()
    s = _Solver(mesh, gas, W.KEP(2), sgs=None)
    prim = np.array([1.2, 30.0, 0.0, 0.0, 1e5])
    Q = s.init_state(lambda xc: prim.reshape(5, 1, 1, 1) * np.ones((1,) + xc.shape[1:]))
    loads = s.wall_loads(Q, (0.5, 0.5, 0.5))
    stats = s.wall_stats(Q)
    assert set(loads) == {("wall", "jmin"), ("wall", "jmax")}
    for name, normal_y in (("jmin", -1.0), ("jmax", 1.0)):
        force, moment = loads[("wall", name)]
        np.testing.assert_allclose(force[0], np.sum(stats[("wall", name)][0]) / 16.0)
        np.testing.assert_allclose(force[1], normal_y * 1e5)
        np.testing.assert_allclose(force[2], 0.0, atol=1e-10)
        np.testing.assert_allclose(moment[:2], 0.0, atol=1e-8)
        np.testing.assert_allclose(moment[2], -normal_y * 0.5 * force[0])
    np.testing.assert_allclose(sum(v[1] for v in loads.values()), 0.0, atol=1e-8)


# ----------------------------------------------------------------------- multiblock
def _gather(mesh, R):
    """Interior RHS values keyed by rounded cell-centre coordinates."""
    out = {}
    for blk, r, g in zip(mesh.blocks, R, mesh.geoms):
        xc = np.asarray(blk.interior(g.xc)).reshape(3, -1).T
        rr = blk.interior(r.cpu().numpy()).reshape(5, -1).T
        for c, v in zip(xc, rr):
            out[tuple(np.round(c, 8))] = v
    return out


MB_CASES = [("split", "kep4", "slip"), ("flip", "kep4", "slip"), ("rot_cyc", "kep4", "slip"),
            ("split", "hybrid", "slip"), ("split", "kep4", "wm")]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-5)])
@pytest.mark.parametrize("kind,scheme,ybc", MB_CASES, ids=["-".join(c) for c in MB_CASES])
def test_multiblock_matches_single_block(W, kind, scheme, ybc, precision, tol):
    """tests/test_multiblock.py:88-98,216-219: the RHS of a two-block split (straight,
    flipped, cyclically rotated index axes) equals the single block's cell by cell, relative
    to the RHS's max; the reference's bound 1e-9 in FP64, 1e-5 in the mixed form (FP32 face
    fluxes summed in another order where the axes are permuted)."""
    make = {"kep4": lambda: W.KEP(4), "hybrid": lambda: W.Hybrid()}[scheme]
    R = []
    for k in ("single", kind):
        mesh = C.skew_case(W, k, n=(12, 10, 8), ybc=ybc)
        s = _Solver(mesh, W.Gas(), make(), sgs="vreman", cfl=0.5, precision=precision)
        R.append(_gather(mesh, s.rhs(s.init_state(C.skew_prim))))
    assert R[0].keys() == R[1].keys()
    scale = np.max(np.abs(np.array(list(R[0].values()))))
    err = max(np.max(np.abs(R[0][c] - R[1][c])) for c in R[0]) / scale
    assert err < tol, err


def _chain_case(W, pieces, n=(40, 10, 8)):
    """The skewed periodic box cut into `pieces` blocks along i (uneven widths), each
    connected to the next, the last to the first across the periodic shift; slip walls in y."""
    cuts = np.linspace(0, n[0], pieces + 1).round().astype(int)
    cuts[1:-1] += np.arange(1, pieces) % 2                  # uneven widths
    assert np.all(np.diff(cuts) >= 3)
    iy, iz = np.arange(n[1] + 1), np.arange(n[2] + 1)
    blocks = [W.Block(f"b{p}", C.skew_nodes(np.arange(cuts[p], cuts[p + 1] + 1), iy, iz, n))
              for p in range(pieces)]
    mesh = W.Mesh(blocks)
    for p in range(pieces - 1):
        mesh.connect(blocks[p], "imax", blocks[p + 1], "imin")
    mesh.connect(blocks[-1], "imax", blocks[0], "imin", shift=(C.LBOX[0], 0, 0))
    for b in blocks:
        mesh.connect(b, "kmin", b, "kmax", shift=(0, 0, -C.LBOX[2]))
        b.set_bc("jmin", W.SlipWall())
        b.set_bc("jmax", W.SlipWall())
    mesh.finalize()
    return mesh


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-5)])
def test_many_blocks_match_single_block(W, precision, tol):
    """Eight blocks of uneven widths in a periodic chain: the RHS and one step equal the
    single block's (the gather keys by cell centre)."""
    out = []
    for pieces in (1, 8):
        mesh = _chain_case(W, pieces)
        s = _Solver(mesh, W.Gas(), W.KEP(4), sgs="wale", cfl=0.5, precision=precision)
        Q = s.init_state(C.skew_prim)
        Q1, dt = s.step(Q)
        out.append((_gather(mesh, s.rhs(Q)), _gather(mesh, Q1), float(dt)))
    for a, b in ((out[0][0], out[1][0]), (out[0][1], out[1][1])):
        assert a.keys() == b.keys()
        scale = np.max(np.abs(np.array(list(a.values()))))
        err = max(np.max(np.abs(a[c] - b[c])) for c in a) / scale
        assert err < tol, err
    dt_tol = 1e-12 if precision == "fp64" else 1e-6      # the mixed form's CFL rates are FP32
    assert abs(out[0][2] - out[1][2]) <= dt_tol * out[0][2]


# ----------------------------------------------------------------------- sponge
def test_sponge_preserves_the_span_mean(W):
    """tests/test_smooth_ramp.py:74-96 on the device: the sponge source (the RHS with the
    sponge minus the RHS without it, same kernel and state) is exactly zero upstream of the
    sponge start, nonzero inside, and its volume-weighted span sum vanishes to round-off."""
    mesh, gas, props, profile, kw = C.ramp_case(W)
    prim = C.ramp_prim(props, profile)
    with_sp = _Solver(mesh, gas, **kw)
    without = _Solver(mesh, gas, **dict(kw, sources=()))
    Q = with_sp.init_state(prim)
    Rs = with_sp.rhs(Q)[0].cpu().numpy()
    R0 = without.rhs(Q)[0].cpu().numpy()
    blk, geo = mesh.blocks[0], mesh.geoms[0]
    g = blk.ng
    inner = (slice(None), slice(g, -g), slice(g, -g), slice(g, -g))
    src, rs = (Rs - R0)[inner], Rs[inner]
    vol = np.asarray(geo.vol)[inner[1:]]
    x_l = np.asarray(geo.xc[0])[inner[1:]][:, 0, 0] / props["L"]
    start = kw["sources"][0].x_start_l
    before, after = np.where(x_l < start)[0], np.where(x_l > start)[0]
    assert before.size and after.size
    assert np.all(src[:, before] == 0.0)
    assert np.any(np.abs(src[1, after]) > 0.0)
    span = np.sum(src * vol, axis=3)
    bound = 8 * np.finfo(float).eps * np.sum(np.abs(rs) * vol, axis=3)
    assert np.all(np.abs(span) <= bound), float(np.max(np.abs(span) - bound))


def test_device_placement(W):
    mesh = C.skew_case(W, "single", n=(4, 4, 4))
    s = _Solver(mesh, W.Gas(), W.KEP(2), sgs=None)
    Q = s.init_state(C.skew_prim)
    assert all(q.device.type == "cuda" for q in Q)
    assert all(g.vol.device.type == "cuda" for g in s.geoms)
