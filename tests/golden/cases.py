"""Case builders shared by the golden-fixture generator and the tests.

Every builder takes an API namespace ``W`` exposing the reference's public classes
(Gas, Block, Mesh, SlipWall, NoSlipWall, Dirichlet, CharacteristicFarfield, Extrapolate,
WallModel, EquilibriumWallModel, KEP, MUSCLHLLC, Hybrid, ConstantMassFlux,
SmoothRampInflow, SmoothRampSponge).  ``make_golden.py`` passes the reference's own
modules; the tests pass ``wmles_jax_b200``'s.  The same nodes, BCs and initial states
therefore reach both implementations.

Inputs are seeded and synthetic.  The skewed periodic node map has the form used by the
reference's multiblock consistency test (tests/test_multiblock.py:14-20); the smooth-ramp
inflow profile is an analytic boundary-layer table, not the DNS data.
"""
import numpy as np

LBOX = (1.0, 0.6, 0.5)


# ----------------------------------------------------------------------------- skewed box
def skew_nodes(ix, iy, iz, n, L=LBOX, skew=0.04):
    X, Y, Z = np.meshgrid(ix / n[0] * L[0], iy / n[1] * L[1], iz / n[2] * L[2], indexing="ij")
    x = X + skew * np.sin(2 * np.pi * Y / L[1]) * np.sin(2 * np.pi * Z / L[2])
    y = Y + skew * 0.5 * np.sin(2 * np.pi * X / L[0])
    z = Z + skew * 0.5 * np.sin(2 * np.pi * X / L[0]) * np.cos(2 * np.pi * Y / L[1])
    return np.stack([x, y, z])


def skew_prim(xc, L=LBOX):
    x, y, z = xc
    k = 2 * np.pi
    rho = 1.2 * (1 + 0.05 * np.sin(k * x / L[0]) * np.cos(k * z / L[2]))
    u = 60 * np.sin(k * y / L[1]) + 20 * np.cos(k * z / L[2])
    v = 15 * np.sin(k * x / L[0]) * np.sin(k * z / L[2])
    w = 10 * np.cos(k * x / L[0]) + 5 * np.sin(k * y / L[1])
    p = 1e5 * (1 + 0.03 * np.cos(k * x / L[0]) * np.sin(k * y / L[1]))
    return np.stack([rho, u, v, w, p])


def skew_case(W, kind, n=(8, 6, 6), ybc="slip"):
    """kind: single | split | flip | rot_cyc.  x and z periodic; y faces get ``ybc``:
    slip | wm (isothermal 300 K) | wm_adiabatic | periodic."""
    ix, iy, iz = (np.arange(m + 1) for m in n)
    if ybc == "slip":
        make_y = W.SlipWall
    elif ybc == "wm":
        make_y = lambda: W.WallModel(W.EquilibriumWallModel(), T_wall=300.0)
    elif ybc == "wm_adiabatic":
        make_y = lambda: W.WallModel(W.EquilibriumWallModel(), T_wall=None, n_match=2)
    else:
        make_y = None
    if kind == "single":
        A = W.Block("all", skew_nodes(ix, iy, iz, n))
        blocks = [A]
        mesh = W.Mesh(blocks)
        mesh.connect(A, "imin", A, "imax", shift=(-LBOX[0], 0, 0))
        zpair, yfaces = {A: ("kmin", "kmax")}, {A: ("jmin", "jmax")}
    else:
        h = n[0] // 2
        nA = skew_nodes(ix[:h + 1], iy, iz, n)
        nB = skew_nodes(ix[h:], iy, iz, n)
        if kind == "rot_cyc":
            nB = np.transpose(nB, (0, 2, 3, 1))
        elif kind == "flip":
            nB = nB[:, ::-1, ::-1, :]
        A, B = W.Block("A", nA), W.Block("B", nB)
        blocks = [A, B]
        mesh = W.Mesh(blocks)
        fx = {"split": ("imin", "imax"), "flip": ("imax", "imin"), "rot_cyc": ("kmin", "kmax")}[kind]
        fz = {"split": ("kmin", "kmax"), "flip": ("kmin", "kmax"), "rot_cyc": ("jmin", "jmax")}[kind]
        fy = {"split": ("jmin", "jmax"), "flip": ("jmax", "jmin"), "rot_cyc": ("imin", "imax")}[kind]
        mesh.connect(A, "imax", B, fx[0])
        mesh.connect(B, fx[1], A, "imin", shift=(LBOX[0], 0, 0))
        zpair, yfaces = {A: ("kmin", "kmax"), B: fz}, {A: ("jmin", "jmax"), B: fy}
    for b in blocks:
        mesh.connect(b, zpair[b][0], b, zpair[b][1], shift=(0, 0, -LBOX[2]))
        if make_y is None:
            mesh.connect(b, yfaces[b][0], b, yfaces[b][1], shift=(0, -LBOX[1], 0))
        else:
            for f in yfaces[b]:
                b.set_bc(f, make_y())
    mesh.finalize()
    return mesh


def zoo_case(W, n=(7, 6, 5)):
    """One skewed block with a different non-periodic BC on every face."""
    ix, iy, iz = (np.arange(m + 1) for m in n)
    A = W.Block("zoo", skew_nodes(ix, iy, iz, n))
    mesh = W.Mesh([A])
    prim_inf = np.array([1.1, 40.0, -5.0, 3.0, 9.5e4])
    A.set_bc("imin", W.Dirichlet(prim_inf))
    A.set_bc("imax", W.CharacteristicFarfield(prim_inf))
    A.set_bc("jmin", W.NoSlipWall(T_wall=290.0))
    A.set_bc("jmax", W.NoSlipWall())
    A.set_bc("kmin", W.Extrapolate())
    A.set_bc("kmax", W.WallModel(W.EquilibriumWallModel(), T_wall=310.0, n_match=2))
    mesh.finalize()
    return mesh


def zoo_prim(xc):
    """Non-uniform state with inflow on the far field and strong shear near the walls."""
    x, y, z = xc
    rho = 1.15 + 0.1 * np.sin(5 * x) * np.cos(7 * z) + 0.05 * y
    u = 45 + 25 * np.sin(9 * y) + 10 * np.cos(8 * z)
    v = 12 * np.sin(6 * x) * np.sin(5 * z) - 4
    w = 8 * np.cos(7 * x) + 6 * np.sin(8 * y)
    p = 9.7e4 * (1 + 0.04 * np.cos(6 * x) * np.sin(9 * y) + 0.02 * z)
    return np.stack([rho, u, v, w, p])


def sod_case(W, nx=24):
    x = np.linspace(0, 1, nx + 1)
    y = np.linspace(0, 0.1, 4)
    z = np.linspace(0, 0.1, 4)
    b = W.Block("tube", np.stack(np.meshgrid(x, y, z, indexing="ij")))
    mesh = W.Mesh([b])
    b.set_bc("imin", W.Extrapolate())
    b.set_bc("imax", W.Extrapolate())
    mesh.connect(b, "jmin", b, "jmax", shift=(0, -0.1, 0))
    mesh.connect(b, "kmin", b, "kmax", shift=(0, 0, -0.1))
    mesh.finalize()
    return mesh


def sod_prim(xc):
    z = 0 * xc[0]
    return np.stack([np.where(xc[0] < 0.5, 1.0, 0.125), z, z, z, np.where(xc[0] < 0.5, 1.0, 0.1)])


# ----------------------------------------------------------------------------- channel
def channel_gas(W, Ma_b=0.3, Re_b=20000.0, gamma=1.4):
    """Nondimensional gas: rho = T = 1 gives U_b = 1 at Ma_b, Re_b on the half-height."""
    return W.Gas(gamma=gamma, R=1.0 / (gamma * Ma_b ** 2), mu_ref=1.0 / Re_b, T_ref=1.0,
                 S_suth=110.4 / 300.0)


def channel_y(ny, beta):
    eta = np.linspace(0.0, 1.0, ny + 1)
    return 1.0 + np.tanh(beta * (2.0 * eta - 1.0)) / np.tanh(beta)


def channel_case(W, n=(32, 32, 16), blocks=2, beta=2.0, n_match=3, T_wall=1.0,
                 Lx=2 * np.pi, Lz=np.pi):
    """Periodic channel (x, z) with wall-modelled walls at y = 0 and y = 2, split into
    ``blocks`` equal blocks along x."""
    nx, ny, nz = n
    if nx % blocks:
        raise ValueError("nx must divide into the blocks")
    y = channel_y(ny, beta)
    z = np.linspace(0.0, Lz, nz + 1)
    xs = np.linspace(0.0, Lx, nx + 1)
    per = nx // blocks
    blks = []
    for b in range(blocks):
        x = xs[b * per:(b + 1) * per + 1]
        blks.append(W.Block(f"B{b}", np.stack(np.meshgrid(x, y, z, indexing="ij"))))
    mesh = W.Mesh(blks)
    for b in range(blocks - 1):
        mesh.connect(blks[b], "imax", blks[b + 1], "imin")
    mesh.connect(blks[-1], "imax", blks[0], "imin", shift=(Lx, 0, 0))
    wm = W.EquilibriumWallModel()
    for blk in blks:
        mesh.connect(blk, "kmin", blk, "kmax", shift=(0, 0, -Lz))
        blk.set_bc("jmin", W.WallModel(wm, T_wall=T_wall, n_match=n_match))
        blk.set_bc("jmax", W.WallModel(wm, T_wall=T_wall, n_match=n_match))
    mesh.finalize()
    return mesh


def channel_laminar_prim(gas, seed=0, noise=0.05):
    """u = 1.5 y (2 - y) plus N(0, noise) in u, v, w drawn per block in block order;
    rho = T = 1."""
    rng = np.random.default_rng(seed)

    def prim(xc):
        y = xc[1]
        pert = rng.normal(0.0, noise, size=(3,) + y.shape)
        one = np.ones_like(y)
        return np.stack([one, 1.5 * y * (2.0 - y) + pert[0], pert[1], pert[2], gas.R * one])
    return prim


# ----------------------------------------------------------------------------- smooth ramp
from wmles_jax_b200.workloads import RAMP_H, RAMP_SPAN, RAMP_TOP, ramp_nodes, ramp_profile, ramp_props  # noqa: E402,F401


def ramp_case(W, n=(12, 8, 6), scheme_factory=None, sgs="vreman", seed=0, n_modes=16,
              scales=(0.1, 0.02, 0.03), sponge_start_l=3.0, x_range=(-0.76, 4.0), skew_z=0.0):
    """Single-block smooth ramp: synthetic inflow (i-min), characteristic outflow (i-max),
    adiabatic wall model (j-min), slip top (j-max), periodic span; spanwise sponge.
    ``skew_z`` shears the span with height (z += skew_z * y), so that the cell centres' z
    depends on j as well as k (an inflow plane that is not extruded)."""
    gas = W.Gas()
    props = ramp_props(gas)
    profile = ramp_profile()
    L = props["L"]
    nodes = ramp_nodes(n, x_range=x_range, L=L)
    if skew_z:
        nodes = nodes.copy()
        nodes[2] = nodes[2] + skew_z * nodes[1]
    blk = W.Block("ramp", nodes)
    mesh = W.Mesh([blk])
    mesh.connect(blk, "kmin", blk, "kmax", shift=(0.0, 0.0, -RAMP_SPAN * L))
    prim_inf = np.array([props["rho_inf"], props["U_inf"], 0.0, 0.0, props["p_inf"]])
    blk.set_bc("imin", W.SmoothRampInflow(props, profile, scales, seed, n_modes, n[2]))
    blk.set_bc("imax", W.CharacteristicFarfield(prim_inf))
    blk.set_bc("jmin", W.WallModel(W.EquilibriumWallModel(), T_wall=None, n_match=1))
    blk.set_bc("jmax", W.SlipWall())
    mesh.finalize()
    sponge = W.SmoothRampSponge(props, sponge_start_l, x_range[1], 1.0)
    scheme = scheme_factory() if scheme_factory else W.Hybrid(W.KEP(4))
    return mesh, gas, props, profile, dict(scheme=scheme, sgs=sgs, cfl=0.5, sources=(sponge,))


def ramp_prim(props, profile, seed=0):
    """Profile-table mean (shifted to the local wall height) plus seeded 2% noise."""
    rng = np.random.default_rng(seed)

    def prim(xc):
        x, y, _ = xc
        L = props["L"]
        xi = np.clip(x / L, 0.0, 1.0)
        wall = RAMP_H * (1.0 - (10.0 * xi ** 3 - 15.0 * xi ** 4 + 6.0 * xi ** 5))
        yd = y / L - wall + RAMP_H
        U = props["U_inf"] * np.interp(yd, profile[:, 0], profile[:, 1])
        pert = rng.normal(0.0, 0.02 * props["U_inf"], size=(3,) + x.shape)
        one = np.ones_like(x)
        return np.stack([props["rho_inf"] * one, U + pert[0], pert[1], pert[2], props["p_inf"] * one])
    return prim


# ----------------------------------------------------------------------------- golden table
SMALL_CASES = ["single_slip_kep4", "split_slip_kep4", "flip_slip_kep4", "rotcyc_slip_kep4",
               "split_wm_hybrid", "flip_wmad_kep2", "single_per_muscl", "rotcyc_per_minmod",
               "zoo_hybrid", "zoo_kep4", "ramp_small", "channel_small_cmf", "naca_small"]
GEOM_CASES = {"single_slip_kep4", "split_slip_kep4", "flip_slip_kep4", "rotcyc_slip_kep4",
              "zoo_hybrid", "ramp_small", "naca_small"}


def golden_case(W, tag):
    """(mesh, gas, solver kwargs, prim_fn, time) of one small golden case."""
    skew = {
        "single_slip_kep4": (("single", "slip"), lambda: W.KEP(4), "vreman", None),
        "split_slip_kep4": (("split", "slip"), lambda: W.KEP(4), "vreman", None),
        "flip_slip_kep4": (("flip", "slip"), lambda: W.KEP(4), "vreman", None),
        "rotcyc_slip_kep4": (("rot_cyc", "slip"), lambda: W.KEP(4), "vreman", None),
        "split_wm_hybrid": (("split", "wm"), lambda: W.Hybrid(), "wale", None),
        "flip_wmad_kep2": (("flip", "wm_adiabatic"), lambda: W.KEP(2), "smagorinsky", None),
        "single_per_muscl": (("single", "periodic"), lambda: W.MUSCLHLLC(), None, None),
        "rotcyc_per_minmod": (("rot_cyc", "periodic"), lambda: W.MUSCLHLLC("minmod"), "wale", None),
    }
    if tag in skew:
        (kind, ybc), sch, sgs, kw = skew[tag]
        mesh = skew_case(W, kind, ybc=ybc)
        return mesh, W.Gas(), dict(scheme=sch(), sgs=sgs, sgs_kwargs=kw, cfl=0.5), skew_prim, 0.0
    if tag == "zoo_hybrid":
        return zoo_case(W), W.Gas(), dict(scheme=W.Hybrid(W.KEP(2), th0=0.05, th1=0.3), sgs="vreman",
                                          cfl=0.5), zoo_prim, 0.0
    if tag == "zoo_kep4":
        return zoo_case(W), W.Gas(), dict(scheme=W.KEP(4), sgs="smagorinsky", cfl=0.5), zoo_prim, 0.0
    if tag == "ramp_small":
        mesh, gas, props, profile, kw = ramp_case(W)
        return mesh, gas, kw, ramp_prim(props, profile), 0.05 * props["L"] / props["U_inf"]
    if tag == "naca_small":
        # the config-4 C-grid with every cell count divided by 8 (four blocks, transposed and
        # flipped interfaces, wall model on two blocks, far field and outflow)
        from wmles_jax_b200.workloads import naca_case
        mesh, gas, kw, prim = naca_case(scale=8, api=W)
        return mesh, gas, kw, prim, 0.0
    if tag == "channel_small_cmf":
        gas = channel_gas(W)
        mesh = channel_case(W, n=(8, 8, 6), blocks=2)
        kw = dict(scheme=W.KEP(4), sgs="wale", sgs_kwargs=dict(Cw=0.5), cfl=0.5,
                  constraints=[W.ConstantMassFlux(0, 1.0)])
        return mesh, gas, kw, channel_laminar_prim(gas, seed=3), 0.0
    raise KeyError(tag)


def cfg2_small_case(W, n=(32, 32, 16)):
    """The config-2 channel physics on a reduced grid: one block, tanh stretching beta=2.5,
    KEP4, WALE Cw=0.5, wall model at the 3rd cell (isothermal), constant mass flux, CFL 0.5;
    Spalding-law IC with 10 % seeded noise tapered towards the walls (seed 0)."""
    from wmles_jax_b200.workloads import loglaw_prim
    gas = channel_gas(W)
    mesh = channel_case(W, n=n, blocks=1, beta=2.5)
    kw = dict(scheme=W.KEP(4), sgs="wale", sgs_kwargs=dict(Cw=0.5), cfl=0.5,
              constraints=[W.ConstantMassFlux(0, 1.0)])
    return mesh, gas, kw, loglaw_prim(gas, mesh, seed=0)


# 100-step trajectories recorded from the reference: (mesh, gas, kw, prim, t0) per case
TRAJ_CASES = ["cfg2_small", "ramp_small", "naca_small"]
TRAJ_STEPS = 100


def traj_case(W, tag):
    if tag == "cfg2_small":
        mesh, gas, kw, prim = cfg2_small_case(W)
        return mesh, gas, kw, prim, 0.0
    return golden_case(W, tag)


# Sod shock tube of the reference's shock test (tests/test_sod.py:7-28): 100 cells,
# Extrapolate ends, periodic y/z, R = 1, mu_ref = 1e-9, CFL 0.5, run to t = 0.2
SOD_NX, SOD_TEND = 100, 0.2
SOD_SCHEMES = {"muscl": lambda W: W.MUSCLHLLC(), "hybrid": lambda W: W.Hybrid(th0=0.3, th1=0.6)}


def sod_run(W, solver_cls, scheme, to_host=np.asarray, init=None, **solver_kw):
    """Run the Sod tube with the reference's loop (dt = min(max_dt, t_end - t)); returns
    (mesh, final state, dts).  ``to_host`` turns a state array into NumPy; ``init(solver,
    prim_fn)`` builds the initial state (default: ``solver.init_state(prim_fn)``)."""
    mesh = sod_case(W, nx=SOD_NX)
    gas = W.Gas(R=1.0, mu_ref=1e-9)
    s = solver_cls(mesh, gas, scheme, sgs=None, cfl=0.5, **solver_kw)
    Q = init(s, sod_prim) if init else s.init_state(sod_prim)
    t, dts = 0.0, []
    while t < SOD_TEND - 1e-12:
        dt = min(float(s.max_dt(Q)), SOD_TEND - t)
        Q = s.advance(Q, dt)
        t += dt
        dts.append(dt)
    return mesh, [to_host(q) for q in Q], np.array(dts)


# free-stream preservation on the skewed periodic box (tests/test_multiblock.py:100-107):
# uniform state, every direction periodic, residual bound 0.1 (energy flux scale ~1e7)
FREESTREAM_PRIM = (1.2, 50.0, -20.0, 30.0, 1e5)
FREESTREAM_SCHEMES = {"kep2": lambda W: W.KEP(2), "kep4": lambda W: W.KEP(4),
                      "muscl": lambda W: W.MUSCLHLLC(), "hybrid": lambda W: W.Hybrid()}


def freestream_prim(xc):
    return np.stack([v + 0 * xc[0] for v in FREESTREAM_PRIM])


def freestream_mesh(W):
    return skew_case(W, "single", n=(12, 10, 8), ybc="periodic")


def cfg1_case(W):
    """Config-1 channel: 2 blocks of 16x32x16, KEP2, Smagorinsky 0.1, wall model at the 3rd
    cell (isothermal), constant mass flux, CFL 0.5; laminar IC + 5% seeded noise."""
    gas = channel_gas(W)
    mesh = channel_case(W)
    kw = dict(scheme=W.KEP(2), sgs="smagorinsky", sgs_kwargs=dict(Cs=0.1), cfl=0.5,
              constraints=[W.ConstantMassFlux(0, 1.0)])
    return mesh, gas, kw, channel_laminar_prim(gas, seed=0)
