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


def channel_mesh(n, blocks=1, beta=2.0, n_match=3, T_wall=1.0, Lx=2 * np.pi, Lz=np.pi):
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
    return mesh.finalize()


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
        ys, yi = np.unique(y, return_inverse=True)
        u = (ut * spalding_uplus(np.clip(np.minimum(ys, 2.0 - ys), 0.0, None) * ut / nu))[yi.reshape(y.shape)]
        # noise of std `noise` U_b in the core, scaled by the mean-velocity shape towards the
        # walls: grid-scale noise at y+ ~ 1 gives an SGS viscosity far above the molecular
        # one, which the reference's CFL estimate (molecular viscosity only) does not cover
        pert = rng.normal(0.0, 1.0, size=(3,) + y.shape) * (noise * np.clip(u / u_core, 0.0, 1.0))
        one = np.ones_like(y)
        return np.stack([one, u + pert[0], pert[1], pert[2], gas.R * one])
    return prim


def channel_case(config=2, n=None, blocks=None):
    """(mesh, gas, solver kwargs, prim_fn) of channel config 1 or 2 (optionally resized)."""
    gas = channel_gas()
    if config == 1:
        mesh = channel_mesh(n or (32, 32, 16), blocks=blocks or 2, beta=2.0)
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
    mesh = channel_mesh(n or (256, 128, 128), blocks=blocks or 1, beta=2.5)
    kw = dict(scheme=KEP(4), sgs="wale", sgs_kwargs=dict(Cw=0.5), cfl=0.5,
              constraints=[ConstantMassFlux(0, 1.0)])
    return mesh, gas, kw, loglaw_prim(gas, mesh)


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
    """Finalized channel mesh of one serving grid, built once and shared by every request on
    that grid (the geometry does not depend on Re_tau or Ma_b); its packed metrics are kept."""
    from .lowering import share_metrics
    mesh = channel_mesh(grid, blocks=1, beta=2.5)
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
