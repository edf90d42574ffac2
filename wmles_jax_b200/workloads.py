"""Seeded synthetic workloads with the shapes and physics of the benchmark configurations.

* ``channel(...)``: periodic channel (x, z), wall-modelled isothermal walls at y = 0, 2,
  nondimensional gas (rho = T = 1 gives U_b = 1 at Ma_b; Re_b on the half-height),
  constant mass flux, SSP-RK3 at CFL 0.5.  Config 1 is 2 blocks of 16x32x16, KEP2 +
  Smagorinsky 0.1; config 2 is one 256x128x128 block, tanh stretching beta = 2.5, KEP4 +
  WALE 0.5, wall model sampled at the 3rd cell.
* ``loglaw_prim``: config-2 initial condition, a Spalding-law mean profile whose friction
  velocity is chosen so the bulk velocity is 1, plus seeded Gaussian noise of 10 % of U_b
  in the core, tapered to zero at the walls with the mean-velocity shape.

No external data: every input is generated here from formulas and a NumPy seed.
"""
import functools

import numpy as np

from .bc import WallModel
from .constraints import ConstantMassFlux
from .gas import Gas
from .mesh import Block, Mesh
from .schemes import KEP
from .wall_model import EquilibriumWallModel


def channel_gas(Ma_b=0.3, Re_b=20000.0, gamma=1.4):
    return Gas(gamma=gamma, R=1.0 / (gamma * Ma_b ** 2), mu_ref=1.0 / Re_b, T_ref=1.0, S_suth=110.4 / 300.0)


def channel_mesh(n, blocks=1, beta=2.0, n_match=3, T_wall=1.0, Lx=2 * np.pi, Lz=np.pi, device=False):
    nx, ny, nz = n
    if nx % blocks:
        raise ValueError("nx must divide into the blocks")
    eta = np.linspace(0.0, 1.0, ny + 1)
    y = 1.0 + np.tanh(beta * (2.0 * eta - 1.0)) / np.tanh(beta)
    z = np.linspace(0.0, Lz, nz + 1)
    xs = np.linspace(0.0, Lx, nx + 1)
    per = nx // blocks
    blks = [Block(f"B{b}", np.stack(np.meshgrid(xs[b * per:(b + 1) * per + 1], y, z, indexing="ij")))
            for b in range(blocks)]
    mesh = Mesh(blks)
    for b in range(blocks - 1):
        mesh.connect(blks[b], "imax", blks[b + 1], "imin")
    mesh.connect(blks[-1], "imax", blks[0], "imin", shift=(Lx, 0, 0))
    wm = EquilibriumWallModel()
    for blk in blks:
        mesh.connect(blk, "kmin", blk, "kmax", shift=(0, 0, -Lz))
        blk.set_bc("jmin", WallModel(wm, T_wall=T_wall, n_match=n_match))
        blk.set_bc("jmax", WallModel(wm, T_wall=T_wall, n_match=n_match))
    return mesh.finalize(device=device)


def spalding_uplus(yp, kappa=0.41, B=5.2, iters=60):
    """Invert Spalding's law y+(u+) for u+ (vectorised bisection)."""
    lo, hi = np.zeros_like(yp), np.full_like(yp, 60.0)
    ekb = np.exp(-kappa * B)
    for _ in range(iters):
        mid = 0.5 * (lo + hi)
        k = kappa * mid
        f = mid + ekb * (np.exp(k) - 1 - k - k * k / 2 - k ** 3 / 6) - yp
        lo, hi = np.where(f < 0, mid, lo), np.where(f < 0, hi, mid)
    return 0.5 * (lo + hi)


def loglaw_prim(gas, mesh, noise=0.1, seed=0):
    """Spalding mean profile with bulk velocity 1 plus N(0, noise) in u, v, w."""
    nu = gas.mu_ref           # T = T_ref = 1, rho = 1
    blk, geo = mesh.blocks[0], mesh.geoms[0]
    # the wall distance depends on y only: bisect on the distinct y values, weighted by volume
    yu, inv = np.unique(blk.interior(geo.xc[1]), return_inverse=True)
    wts = np.bincount(inv.ravel(), weights=blk.interior(geo.vol).ravel())
    ywall = np.minimum(yu, 2.0 - yu)
    lo, hi = 1e-4, 1.0
    for _ in range(60):                                   # u_tau giving a bulk velocity of 1
        ut = 0.5 * (lo + hi)
        ub = np.sum(ut * spalding_uplus(ywall * ut / nu) * wts) / np.sum(wts)
        lo, hi = (ut, hi) if ub < 1.0 else (lo, ut)
    ut = 0.5 * (lo + hi)
    rng = np.random.default_rng(seed)

    u_core = ut * spalding_uplus(np.array([ywall.max()]) * ut / nu)[0]

    def prim(xc):
        y = xc[1]
        # on a grid extruded in x and z (every channel grid here) y is one j-line repeated:
        # the profile is evaluated on that line and broadcast, the same values as over all cells
        line = y[:1, :, :1] if y.ndim == 3 else None
        if line is not None and np.array_equal(y, np.broadcast_to(line, y.shape)):
            ys, yi = np.unique(line, return_inverse=True)
            u = np.broadcast_to((ut * spalding_uplus(np.clip(np.minimum(ys, 2.0 - ys), 0.0, None) * ut / nu))
                                [yi.reshape(line.shape)], y.shape)
        else:
            ys, yi = np.unique(y, return_inverse=True)
            u = (ut * spalding_uplus(np.clip(np.minimum(ys, 2.0 - ys), 0.0, None) * ut / nu))[yi.reshape(y.shape)]
        # noise of std `noise` U_b in the core, scaled by the mean-velocity shape towards the
        # walls: grid-scale noise at y+ ~ 1 gives an SGS viscosity far above the molecular
        # one, which the reference's CFL estimate (molecular viscosity only) does not cover
        pert = rng.normal(0.0, 1.0, size=(3,) + y.shape) * (noise * np.clip(u / u_core, 0.0, 1.0))
        one = np.ones_like(y)
        return np.stack([one, u + pert[0], pert[1], pert[2], gas.R * one])
    return prim


def channel_case(config=2, n=None, blocks=None, device=False):
    """(mesh, gas, solver kwargs, prim_fn) of channel config 1 or 2 (optionally resized);
    device=True computes the mesh metrics on the GPU (Mesh.finalize)."""
    gas = channel_gas()
    if config == 1:
        mesh = channel_mesh(n or (32, 32, 16), blocks=blocks or 2, beta=2.0, device=device)
        from .sgs import make_sgs  # noqa: F401  (names resolved by the solver)
        kw = dict(scheme=KEP(2), sgs="smagorinsky", sgs_kwargs=dict(Cs=0.1), cfl=0.5,
                  constraints=[ConstantMassFlux(0, 1.0)])
        rng = np.random.default_rng(0)

        def prim(xc):
            y = xc[1]
            pert = rng.normal(0.0, 0.05, size=(3,) + y.shape)
            one = np.ones_like(y)
            return np.stack([one, 1.5 * y * (2.0 - y) + pert[0], pert[1], pert[2], gas.R * one])
        return mesh, gas, kw, prim
    mesh = channel_mesh(n or (256, 128, 128), blocks=blocks or 1, beta=2.5, device=device)
    kw = dict(scheme=KEP(4), sgs="wale", sgs_kwargs=dict(Cw=0.5), cfl=0.5,
              constraints=[ConstantMassFlux(0, 1.0)])
    return mesh, gas, kw, loglaw_prim(gas, mesh)


# ---------------------------------------------------------------------------- smooth ramp (config 3)
RAMP_H, RAMP_TOP, RAMP_SPAN = 0.22, 0.74, 0.288


def ramp_props(gas, Ma=0.2, Re_L=667000.0, T_inf=300.0, p_inf=101325.0):
    rho = p_inf / (gas.R * T_inf)
    mu = gas.mu_ref * (T_inf / gas.T_ref) ** 1.5 * (gas.T_ref + gas.S_suth) / (T_inf + gas.S_suth)
    U = Ma * float(np.sqrt(gas.gamma * gas.R * T_inf))
    L = Re_L * (mu / rho) / U
    return dict(gas=gas, Ma_inf=Ma, Re_L=Re_L, T_inf=T_inf, p_inf=p_inf, rho_inf=rho,
                mu_inf=mu, nu_inf=mu / rho, U_inf=U, L=L)


def ramp_profile(n=80, delta=0.028, y0=RAMP_H, intensity=0.05):
    """Analytic inflow table [y/L, U, V, uu, vv, ww, uv] (normalised by U_inf): a 1/7-power
    boundary layer of thickness ``delta`` with Reynolds stresses peaking near the wall at
    ``intensity``^2 and vanishing outside the layer."""
    y = y0 + np.concatenate([np.linspace(0.0, 2 * delta, n - 10), np.linspace(2.2 * delta, 0.6, 10)])
    eta = np.clip((y - y0) / delta, 0.0, 1.0)
    U = eta ** (1.0 / 7.0)
    V = 0.002 * eta
    shape = np.exp(-((eta - 0.1) / 0.35) ** 2) * (eta < 1.0) + 1e-6
    uu = (intensity ** 2) * shape * 2.0
    vv = (intensity ** 2) * shape * 0.6
    ww = (intensity ** 2) * shape * 1.0
    uv = -0.4 * np.sqrt(uu * vv)
    return np.stack([y, U, V, uu, vv, ww, uv], axis=1)


def ramp_nodes(n, x_range=(-0.76, 4.0), ratio=1.08, L=1.0):
    """Structured ramp nodes: quintic ramp wall from y=0.22 (x<=0) to 0 (x>=1), slip top
    at 0.74, geometric wall-normal stretching ``ratio``, periodic span 0.288 (all / L)."""
    ni, nj, nk = n
    x = np.linspace(x_range[0], x_range[1], ni + 1)
    xi = np.clip(x, 0.0, 1.0)
    wall = RAMP_H * (1.0 - (10.0 * xi ** 3 - 15.0 * xi ** 4 + 6.0 * xi ** 5))
    s = np.concatenate([[0.0], np.cumsum(ratio ** np.arange(nj))])
    s = s / s[-1]
    y = wall[:, None] + (RAMP_TOP - wall[:, None]) * s[None, :]
    z = np.linspace(0.0, RAMP_SPAN, nk + 1)
    shape = (ni + 1, nj + 1, nk + 1)
    X = np.broadcast_to(x[:, None, None], shape)
    Y = np.broadcast_to(y[:, :, None], shape)
    Z = np.broadcast_to(z[None, None, :], shape)
    return np.stack((X, Y, Z)) * L


def ramp_case(n=(384, 96, 64), n_modes=64, seed=0, sponge_start_l=3.0, x_range=(-0.76, 4.0), device=False):
    """(mesh, gas, solver kwargs, prim_fn, props) of the smooth-ramp configuration (config 3
    at the default size): quintic ramp wall with the equilibrium wall model (adiabatic,
    sampled at the first cell), slip top at y = 0.74 L, periodic span 0.288 L, geometric
    wall-normal ratio 1.08, Ma_inf 0.2, Re_L 667000; Fourier-mode synthetic inflow with 5 %
    intensity and scales (0.1, 0.02, 0.03) L on i-min, characteristic outflow on i-max, a
    spanwise-mean sponge over the last 1 L; Hybrid Ducros KEP4 / MUSCL-HLLC, Vreman.  The
    inflow profile is the analytic boundary-layer table of ``ramp_profile``."""
    from .bc import CharacteristicFarfield, SlipWall
    from .schemes import Hybrid
    from .smooth_ramp import SmoothRampInflow, SmoothRampSponge
    gas = Gas()
    props = ramp_props(gas)
    profile = ramp_profile()
    L = props["L"]
    blk = Block("ramp", ramp_nodes(n, x_range=x_range, L=L))
    mesh = Mesh([blk])
    mesh.connect(blk, "kmin", blk, "kmax", shift=(0.0, 0.0, -RAMP_SPAN * L))
    prim_inf = np.array([props["rho_inf"], props["U_inf"], 0.0, 0.0, props["p_inf"]])
    blk.set_bc("imin", SmoothRampInflow(props, profile, (0.1, 0.02, 0.03), seed, n_modes, n[2]))
    blk.set_bc("imax", CharacteristicFarfield(prim_inf))
    blk.set_bc("jmin", WallModel(EquilibriumWallModel(), T_wall=None, n_match=1))
    blk.set_bc("jmax", SlipWall())
    mesh.finalize(device=device)
    sponge = SmoothRampSponge(props, sponge_start_l, x_range[1], 1.0)
    kw = dict(scheme=Hybrid(KEP(4)), sgs="vreman", cfl=0.5, sources=(sponge,))
    rng = np.random.default_rng(seed)

    def prim(xc):
        x, y, _ = xc
        xi = np.clip(x / L, 0.0, 1.0)
        wall = RAMP_H * (1.0 - (10.0 * xi ** 3 - 15.0 * xi ** 4 + 6.0 * xi ** 5))
        yd = y / L - wall + RAMP_H
        U = props["U_inf"] * np.interp(yd, profile[:, 0], profile[:, 1])
        pert = rng.normal(0.0, 0.02 * props["U_inf"], size=(3,) + x.shape)
        one = np.ones_like(x)
        return np.stack([props["rho_inf"] * one, U + pert[0], pert[1], pert[2], props["p_inf"] * one])
    return mesh, gas, kw, prim, props


# ---------------------------------------------------------------------------- NACA 0012 C-grid (config 4)
NACA_SPAN, NACA_FAR = 0.0481, 20.0


def naca0012_half_thickness(x):
    """Half thickness of the NACA 0012 section, chord 1: the 4-digit thickness formula with
    the closed-trailing-edge x^4 coefficient (-0.1036)."""
    return 0.6 * (0.2969 * np.sqrt(x) - 0.1260 * x - 0.3516 * x ** 2 + 0.2843 * x ** 3 - 0.1036 * x ** 4)


def geometric_spacing(n, first, total):
    """n+1 increasing coordinates from 0 to `total` whose intervals grow by a constant ratio
    from `first` (uniform when `first` is already the mean interval)."""
    if first * n >= total:
        return np.linspace(0.0, total, n + 1)
    lo, hi = 1.0 + 1e-12, 4.0
    for _ in range(200):
        r = 0.5 * (lo + hi)
        if first * (r ** n - 1.0) / (r - 1.0) < total:
            lo = r
        else:
            hi = r
    x = np.concatenate([[0.0], np.cumsum(first * (0.5 * (lo + hi)) ** np.arange(n))])
    return x * (total / x[-1])


def naca_cgrid_nodes(scale=1, far=NACA_FAR, span=NACA_SPAN, wall_spacing=2e-3):
    """Nodes (3, ni+1, nj+1, nk+1) of a four-block C-grid around the NACA 0012 section.

    One algebraic C-mesh: its inner line runs along the lower wake cut (x = far -> 1), around
    the section (lower surface, leading edge, upper surface; clustered at the leading edge)
    and along the
    upper wake cut (1 -> far); its outer line is y = -far, a half circle of radius `far`
    about the trailing edge, and y = +far; nodes lie on straight lines between the two with
    geometric wall-normal spacing (first interval ~ wall_spacing).  It is cut into blocks
    of (at scale 1) 128 x 64 (lower wake, i and j reversed), 256 x 64 (section, trailing
    edge lower -> leading edge -> upper surface at x ~ 0.65), 64 x 64 (rest of the upper
    surface, with i and j transposed so its wall is an i face) and 128 x 64 (upper wake);
    40 spanwise cells over `span`.  `scale` divides every cell count."""
    n_wake, n_af, n_aft, nj, nk = 128 // scale, 320 // scale, 64 // scale, 64 // scale, 40 // scale
    s = np.linspace(0.0, 1.0, n_af + 1)
    # per side x = 1 - sin(pi t / 2), t = distance from the trailing edge in index space:
    # clustered at the leading edge, ~ chord / n_af at the trailing edge (a trailing-edge
    # clustering would carry its fine x spacing out to the far field along the C-grid's
    # trailing-edge lines, with cells of extreme aspect ratio there)
    xa = 1.0 - np.sin(0.5 * np.pi * (1.0 - np.abs(1.0 - 2.0 * s)))  # 1 -> 0 -> 1
    ya = np.where(s <= 0.5, -1.0, 1.0) * naca0012_half_thickness(xa)
    xw = 1.0 + geometric_spacing(n_wake, 1.0 - xa[1], far - 1.0)     # 1 -> far
    phi = -0.5 * np.pi - np.pi * s
    inner = np.stack([np.concatenate([xw[::-1], xa[1:-1], xw]), np.concatenate([0 * xw, ya[1:-1], 0 * xw])])
    outer = np.stack([np.concatenate([xw[::-1], 1.0 + far * np.cos(phi[1:-1]), xw]),
                      np.concatenate([-far + 0 * xw, far * np.sin(phi[1:-1]), far + 0 * xw])])
    sig = geometric_spacing(nj, wall_spacing / far, 1.0)
    xy = inner[:, :, None] + sig[None, None, :] * (outer - inner)[:, :, None]      # (2, NI+1, nj+1)
    z = np.linspace(0.0, span, nk + 1)
    shp = xy.shape[1:] + (nk + 1,)
    C = np.stack([np.broadcast_to(xy[0][:, :, None], shp), np.broadcast_to(xy[1][:, :, None], shp),
                  np.broadcast_to(z[None, None, :], shp)])
    a0, a1, a2 = n_wake, n_wake + n_af - n_aft, n_wake + n_af
    return {
        "wake_lower": np.ascontiguousarray(C[:, a0::-1, ::-1]),
        "section": np.ascontiguousarray(C[:, a0:a1 + 1]),
        "section_aft": np.ascontiguousarray(C[:, a1:a2 + 1][:, ::-1].transpose(0, 2, 1, 3)),
        "wake_upper": np.ascontiguousarray(C[:, a2:]),
    }


def _classes(api):
    """The public classes a builder needs: `api` (any namespace with the reference's class
    names, e.g. to feed the same case to another implementation) or this package's."""
    if api is not None:
        return api
    import types
    from .bc import CharacteristicFarfield
    from .schemes import Hybrid
    return types.SimpleNamespace(Gas=Gas, Block=Block, Mesh=Mesh, WallModel=WallModel, KEP=KEP, Hybrid=Hybrid,
                                 EquilibriumWallModel=EquilibriumWallModel,
                                 CharacteristicFarfield=CharacteristicFarfield)


def naca_case(scale=1, alpha_deg=4.0, Ma=0.15, Re_c=1e6, noise=0.01, seed=0, n_match=3, api=None,
              device=False):
    """(mesh, gas, solver kwargs, prim_fn) of the NACA 0012 C-grid (config 4 at scale 1):
    nondimensional gas (rho = T = 1 gives |U| = 1 at Ma, Re on the chord), angle of attack
    `alpha_deg`, adiabatic equilibrium wall model on the section, characteristic far field
    and outflow, periodic span; Hybrid Ducros KEP4 / MUSCL-HLLC with Vreman; uniform free
    stream plus N(0, noise) in u, v, w."""
    W = _classes(api)
    Block, Mesh, WallModel, EquilibriumWallModel = W.Block, W.Mesh, W.WallModel, W.EquilibriumWallModel
    CharacteristicFarfield, Hybrid, KEP = W.CharacteristicFarfield, W.Hybrid, W.KEP
    nodes = naca_cgrid_nodes(scale)
    gas = W.Gas(gamma=1.4, R=1.0 / (1.4 * Ma ** 2), mu_ref=1.0 / Re_c, T_ref=1.0, S_suth=110.4 / 300.0)
    blk = {name: Block(name, x) for name, x in nodes.items()}
    mesh = Mesh(list(blk.values()))
    wl, sec, aft, wu = blk["wake_lower"], blk["section"], blk["section_aft"], blk["wake_upper"]
    mesh.connect(wl, "imin", sec, "imin")          # trailing edge, lower side: i and j reversed
    mesh.connect(sec, "imax", aft, "jmax")         # upper surface: transposed
    mesh.connect(aft, "jmin", wu, "imin")          # trailing edge, upper side
    mesh.connect(wl, "jmax", wu, "jmin")           # wake cut
    for b in blk.values():
        mesh.connect(b, "kmin", b, "kmax", shift=(0.0, 0.0, -NACA_SPAN))
    a = np.deg2rad(alpha_deg)
    prim_inf = np.array([1.0, np.cos(a), np.sin(a), 0.0, gas.R])
    m = min(n_match, min(b.n[1] for b in blk.values()))
    wm = EquilibriumWallModel()
    sec.set_bc("jmin", WallModel(wm, T_wall=None, n_match=m))
    aft.set_bc("imin", WallModel(wm, T_wall=None, n_match=m))
    for b, f in ((sec, "jmax"), (wl, "jmin"), (wl, "imax"), (wu, "jmax"), (wu, "imax"), (aft, "imax")):
        b.set_bc(f, CharacteristicFarfield(prim_inf))
    mesh.finalize(device=True) if device else mesh.finalize()
    kw = dict(scheme=Hybrid(KEP(4)), sgs="vreman", cfl=0.5)
    rng = np.random.default_rng(seed)

    def prim(xc):
        one = np.ones_like(xc[0])
        pert = rng.normal(0.0, noise, size=(3,) + one.shape)
        return np.stack([one, np.cos(a) + pert[0], np.sin(a) + pert[1], pert[2], gas.R * one])
    return mesh, gas, kw, prim


# algorithmic HBM bytes per interior cell (FP64 / mixed metrics), per stage-kernel launch
# stage 1: Q read + Q1 write + metrics; stages 2, 3: + Q0 read; CFL/constraint pass: Q + S, V
STAGE_BYTES = {"fp64": (184, 224, 224), "mixed": (132, 172, 172)}
STEP_BYTES = {"fp64": 752, "mixed": 556}
CMF_BYTES = 80


# ---------------------------------------------------------------------------- serving mix
SERVING_GRIDS = ((48, 48, 48), (64, 48, 48), (96, 64, 64), (128, 96, 64), (192, 96, 96))


def re_bulk_from_re_tau(re_tau):
    """Half-height bulk Reynolds number for a friction Reynolds number, from Dean's
    correlation Re_tau = 0.09 Re_m^0.88 with Re_m = U_b (2h) / nu on the full height."""
    return 0.5 * (np.asarray(re_tau, dtype=float) / 0.09) ** (1.0 / 0.88)


@functools.lru_cache(maxsize=16)
def serving_mesh(grid):
    """Finalized channel mesh of one serving grid, built once (metrics on the GPU) and shared
    by every request on that grid (the geometry does not depend on Re_tau or Ma_b); its packed
    metrics stay on the device."""
    from .lowering import share_metrics
    mesh = channel_mesh(grid, blocks=1, beta=2.5, device=True)
    share_metrics(mesh)
    return mesh


def serving_case(re_tau, ma_b, grid, seed=0):
    """(mesh, gas, solver kwargs, prim_fn) of one serving request: the config-2 channel
    (tanh stretching beta = 2.5, KEP4 + WALE 0.5, wall model at the 3rd cell, constant
    mass flux, CFL 0.5) at the given Re_tau, bulk Mach number and grid, log-law IC with
    seeded noise."""
    gas = channel_gas(Ma_b=float(ma_b), Re_b=float(re_bulk_from_re_tau(re_tau)))
    mesh = serving_mesh(tuple(int(n) for n in grid))
    kw = dict(scheme=KEP(4), sgs="wale", sgs_kwargs=dict(Cw=0.5), cfl=0.5,
              constraints=[ConstantMassFlux(0, 1.0)])
    return mesh, gas, kw, loglaw_prim(gas, mesh, seed=seed)


def serving_requests(n=64, rate=20.0, steps=2000, seed=0, grids=SERVING_GRIDS):
    """Seeded request mix: Poisson arrivals at `rate` per second, Re_tau ~ U[550, 5200],
    Ma_b ~ U[0.1, 0.5], grid drawn uniformly from `grids`; request r's IC noise uses seed r."""
    from .serving import Request
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n))
    re_tau = rng.uniform(550.0, 5200.0, n)
    ma_b = rng.uniform(0.1, 0.5, n)
    gidx = rng.integers(0, len(grids), n)
    out = []
    for r in range(n):
        grid, rt, ma = grids[gidx[r]], float(re_tau[r]), float(ma_b[r])
        out.append(Request(rid=r, build=(lambda rt=rt, ma=ma, grid=grid, r=r: serving_case(rt, ma, grid, seed=r)),
                           steps=int(steps), arrival=float(arrivals[r]), dims=(tuple(grid),),
                           meta=dict(re_tau=rt, ma_b=ma, grid=tuple(grid))))
    return out
