"""CPU oracle for the wmles explicit RHS + SSP-RK3 step.  TEST INFRASTRUCTURE ONLY.

This module restates, in NumPy float64, the reference algorithm of the hot path
(EduardoMolina/wmles_jax, ``wmles/solver.py`` and the physics modules it calls).  It is
the checker for the CUDA backend: only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import it, and never as the thing measured or
shipped.  The product path (``wmles_jax_b200``) never imports it.

Parity pin: ``tests/golden/make_golden.py`` runs the reference itself (its NumPy
float64 fallback, ``wmles/backend.py:36-41``) on the cases in ``tests/golden/cases.py``
and stores its outputs; ``tests/test_oracle_golden.py`` checks this module against them.

The oracle consumes a mesh, BCs and solver options built with ``wmles_jax_b200``'s
descriptor classes (same constructors as the reference).  Each function cites the
reference file:line it follows.  Elementwise operations keep the reference's order of
evaluation, so the ghost fills are bit-identical to the reference.
"""
import numpy as np

from wmles_jax_b200.bc import (SlipWall, NoSlipWall, Dirichlet, CharacteristicFarfield,
                               Extrapolate, WallModel)
from wmles_jax_b200.mesh import Interface, interface_index_map, sl
from wmles_jax_b200.schemes import KEP, MUSCLHLLC, Hybrid
from wmles_jax_b200.sgs import make_sgs
from wmles_jax_b200.smooth_ramp import SmoothRampInflow, SmoothRampSponge


# ----------------------------------------------------------------------------- gas
def sum3(a):
    """Sum over a leading axis of length 3 in the order NumPy reduces it: (a0+a1)+a2."""
    return a[0] + a[1] + a[2]


def cons_to_prim(gas, q):
    """wmles/gas.py:28-33"""
    rho = q[0]
    u = q[1:4] / rho
    p = (gas.gamma - 1.0) * (q[4] - 0.5 * rho * sum3(u * u))
    return np.concatenate([rho[None], u, p[None]], axis=0), p / (rho * gas.R)


def prim_to_cons(gas, w):
    """wmles/gas.py:35-38"""
    rho, u, p = w[0], w[1:4], w[4]
    E = p / (gas.gamma - 1.0) + 0.5 * rho * sum3(u * u)
    return np.concatenate([rho[None], rho * u, E[None]], axis=0)


def viscosity(gas, T):
    """Sutherland, wmles/gas.py:24-26"""
    return gas.mu_ref * (T / gas.T_ref) ** 1.5 * (gas.T_ref + gas.S_suth) / (T + gas.S_suth)


def sound_speed(gas, T):
    return np.sqrt(gas.gamma * gas.R * T)


# ----------------------------------------------------------------------------- ghost-cell maps
def slip_map(gas, src, nrm):
    """wmles/bc.py:41-47"""
    w, _ = cons_to_prim(gas, src)
    u = w[1:4]
    un = sum3(u * nrm)
    return prim_to_cons(gas, np.concatenate([w[:1], u - 2.0 * un * nrm, w[4:5]], axis=0))


def noslip_map(gas, src, T_wall):
    """wmles/bc.py:56-64"""
    w, T = cons_to_prim(gas, src)
    Tg = T if T_wall is None else np.maximum(2.0 * T_wall - T, 0.1 * T_wall)
    rho = w[4] / (gas.R * Tg)
    return prim_to_cons(gas, np.concatenate([rho[None], -w[1:4], w[4:5]], axis=0))


def dirichlet_map(gas, src, prim):
    """wmles/bc.py:73-77"""
    w = prim.reshape((5,) + (1,) * (src.ndim - 1)) * np.ones_like(src[:1])
    return prim_to_cons(gas, w)


def farfield_map(gas, src, nrm, prim, side):
    """Linearised characteristic far field, wmles/bc.py:86-115"""
    w, T = cons_to_prim(gas, src)
    winf = prim.reshape((5,) + (1,) * (src.ndim - 1)) * np.ones_like(src[:1])
    rho_i, u_i, p_i = winf[0], winf[1:4], winf[4]
    c_i = np.sqrt(gas.gamma * p_i / rho_i)
    n_out = nrm if side == 1 else -nrm
    un = sum3(w[1:4] * n_out)
    un_i = sum3(u_i * n_out)
    c = sound_speed(gas, T)
    drho, dp = w[0] - rho_i, w[4] - p_i
    dun = un - un_i
    a_plus = np.where(un + c > 0.0, dp + rho_i * c_i * dun, 0.0)
    a_minus = np.where(un - c > 0.0, dp - rho_i * c_i * dun, 0.0)
    dp_bc = 0.5 * (a_plus + a_minus)
    dun_bc = (a_plus - a_minus) / (2.0 * rho_i * c_i)
    out = un > 0.0
    entropy = np.where(out, drho - dp / c_i ** 2, 0.0)
    du_t = w[1:4] - u_i - dun * n_out
    du_t = np.where(out[None], du_t, 0.0)
    rho_bc = rho_i + dp_bc / c_i ** 2 + entropy
    u_bc = u_i + dun_bc * n_out + du_t
    p_bc = p_i + dp_bc
    return prim_to_cons(gas, np.concatenate([rho_bc[None], u_bc, p_bc[None]], axis=0))


# ----------------------------------------------------------------------------- inflow
def inflow_noise(modes, props, y_l, z_l, time, span_cells, ng):
    """Three normalised Fourier fields, wmles/smooth_ramp.py:179-197"""
    X = props["U_inf"] * time / props["L"]
    zi = slice(ng, ng + span_cells)
    out = []
    for comp, (kx, ky, kz, ph) in enumerate(modes):
        arg = (kx[:, None, None] * X + ky[:, None, None] * y_l[None]
               + kz[:, None, None] * z_l[None] + ph[:, None, None])
        f = np.sum(np.cos(arg), axis=0)
        f = f - np.mean(f[:, zi], axis=1, keepdims=True)
        if comp == 1:
            cov = np.mean(f[:, zi] * out[0][:, zi], axis=1, keepdims=True)
            f = f - cov * out[0]
        var = np.mean(f[:, zi] ** 2, axis=1, keepdims=True)
        out.append(f / np.sqrt(np.maximum(var, 1e-20)))
    return np.stack(out)


def inflow_fill(bc, gas, q, blk, geom, time):
    """wmles/smooth_ramp.py:150-177 (i-min face only)"""
    ng = blk.ng
    props, tab = bc.props, bc.profile
    q = q.copy()
    for m in range(ng):
        gi = ng - 1 - m
        xc = geom.xc[:, gi:gi + 1]
        y_l, z_l = xc[1, 0] / props["L"], xc[2, 0] / props["L"]
        noise = inflow_noise(bc._modes, props, y_l, z_l, time, blk.n[2], ng)
        col = lambda c: np.interp(y_l, tab[:, 0], tab[:, c])
        U = props["U_inf"]
        uu = np.maximum(col(3), 0.0) * U ** 2
        vv = np.maximum(col(4), 0.0) * U ** 2
        ww = np.maximum(col(5), 0.0) * U ** 2
        uv = col(6) * U ** 2
        su = np.sqrt(uu)
        l10 = np.where(su > 1e-14, uv / np.maximum(su, 1e-14), 0.0)
        l11 = np.sqrt(np.maximum(vv - l10 ** 2, 0.0))
        u = U * col(1) + su * noise[0]
        v = U * col(2) + l10 * noise[0] + l11 * noise[1]
        w = np.sqrt(ww) * noise[2]
        z = np.zeros_like(u)
        prim = np.stack([props["rho_inf"] + z, u, v, w, props["p_inf"] + z])[:, None]
        q[:, gi:gi + 1] = prim_to_cons(gas, prim)
    return q


# ----------------------------------------------------------------------------- schemes
def kg_flux(wa, wb, S, g):
    """Kennedy-Gruber two-point flux, wmles/schemes.py:15-23"""
    rho = 0.5 * (wa[0] + wb[0])
    u = 0.5 * (wa[1:4] + wb[1:4])
    p = 0.5 * (wa[4] + wb[4])
    ea = 0.5 * (wa[4] / ((g - 1.0) * wa[0]) + 0.5 * sum3(wa[1:4] ** 2)
                + wb[4] / ((g - 1.0) * wb[0]) + 0.5 * sum3(wb[1:4] ** 2))
    un = sum3(u * S)
    m = rho * un
    return np.concatenate([m[None], m * u + p * S, (m * ea + p * un)[None]], axis=0)


def kep_flux(order, blk, geom, w, gas, d):
    """wmles/schemes.py:57-70"""
    S = blk.slab(geom.S[d], d, 0, 1)
    L, R = blk.slab(w, d, -1, 0), blk.slab(w, d, 0, 1)
    F = kg_flux(L, R, S, gas.gamma)
    if order == 2:
        return F
    L2, R2 = blk.slab(w, d, -2, -1), blk.slab(w, d, 1, 2)
    return 2.0 * ((2.0 / 3.0) * F - (1.0 / 12.0) * (kg_flux(L, R2, S, gas.gamma)
                                                     + kg_flux(L2, R, S, gas.gamma)))


def albada(a, b, eps=1e-12):
    """wmles/schemes.py:100-101"""
    return (a * (b * b + eps) + b * (a * a + eps)) / (a * a + b * b + 2.0 * eps)


def minmod(a, b):
    """wmles/schemes.py:104-105"""
    return 0.5 * (np.sign(a) + np.sign(b)) * np.minimum(np.abs(a), np.abs(b))


def hllc(wl, wr, S, g):
    """wmles/schemes.py:108-137"""
    Sm = np.sqrt(sum3(S * S))
    n = S / Sm
    rl, ul, pl = wl[0], wl[1:4], wl[4]
    rr, ur, pr = wr[0], wr[1:4], wr[4]
    unl, unr = sum3(ul * n), sum3(ur * n)
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    sL, sR = np.minimum(unl - cl, unr - cr), np.maximum(unl + cl, unr + cr)
    ss = ((pr - pl + rl * unl * (sL - unl) - rr * unr * (sR - unr))
          / (rl * (sL - unl) - rr * (sR - unr)))
    El = pl / (g - 1.0) + 0.5 * rl * sum3(ul * ul)
    Er = pr / (g - 1.0) + 0.5 * rr * sum3(ur * ur)

    def phys(r, u, p, un, E):
        return np.concatenate([(r * un)[None], r * un * u + p * n, ((E + p) * un)[None]], axis=0)

    def cons(r, u, E):
        return np.concatenate([r[None], r * u, E[None]], axis=0)

    def star(r, u, p, un, E, s):
        f = r * (s - un) / (s - ss)
        e = E / r + (ss - un) * (ss + p / (r * (s - un)))
        return np.concatenate([f[None], f * (u + (ss - un) * n), (f * e)[None]], axis=0)

    with np.errstate(divide="ignore", invalid="ignore"):
        Fl, Fr = phys(rl, ul, pl, unl, El), phys(rr, ur, pr, unr, Er)
        Ul, Ur = cons(rl, ul, El), cons(rr, ur, Er)
        Fsl = Fl + sL * (star(rl, ul, pl, unl, El, sL) - Ul)
        Fsr = Fr + sR * (star(rr, ur, pr, unr, Er, sR) - Ur)
    F = np.where(sL >= 0, Fl, np.where(ss >= 0, Fsl, np.where(sR > 0, Fsr, Fr)))
    return F * Sm


def muscl_hllc_flux(limiter, blk, geom, w, gas, d):
    """wmles/schemes.py:140-152"""
    lim = albada if limiter == "albada" else minmod
    S = blk.slab(geom.S[d], d, 0, 1)
    L2, L = blk.slab(w, d, -2, -1), blk.slab(w, d, -1, 0)
    R, R2 = blk.slab(w, d, 0, 1), blk.slab(w, d, 1, 2)
    wl = L + 0.5 * lim(L - L2, R - L)
    wr = R - 0.5 * lim(R - L, R2 - R)
    bad = (wl[0] <= 0) | (wl[4] <= 0) | (wr[0] <= 0) | (wr[4] <= 0)
    wl, wr = np.where(bad, L, wl), np.where(bad, R, wr)
    return hllc(wl, wr, S, gas.gamma)


def inviscid_flux(scheme, blk, geom, w, gas, d, theta):
    if isinstance(scheme, KEP):
        return kep_flux(scheme.order, blk, geom, w, gas, d)
    if isinstance(scheme, MUSCLHLLC):
        return muscl_hllc_flux(scheme.limiter, blk, geom, w, gas, d)
    if isinstance(scheme, Hybrid):
        # wmles/schemes.py:163-166
        th = np.maximum(blk.slab(theta, d, -1, 0), blk.slab(theta, d, 0, 1))
        s = np.clip((th - scheme.th0) / (scheme.th1 - scheme.th0), 0.0, 1.0)
        return ((1.0 - s) * inviscid_flux(scheme.c, blk, geom, w, gas, d, theta)
                + s * inviscid_flux(scheme.u, blk, geom, w, gas, d, theta))
    raise NotImplementedError(type(scheme).__name__)


# ----------------------------------------------------------------------------- viscous
def green_gauss(phi, geom):
    """(nv, Ni, Nj, Nk) -> (nv, 3, Ni, Nj, Nk), outermost layer 0; wmles/viscous.py:6-19"""
    nd = phi.ndim
    acc = 0.0
    for d in range(3):
        Nd = phi.shape[1 + d]
        pf = 0.5 * (phi[sl(nd, d, slice(None, -1))] + phi[sl(nd, d, slice(1, None))])
        flux = pf[:, None] * geom.S[d][sl(4, d, slice(1, Nd))][None]
        inner = slice(1, -1)
        acc = acc + (flux[sl(nd + 1, d, slice(1, None), inner)]
                     - flux[sl(nd + 1, d, slice(None, -1), inner)])
    g = acc / geom.vol[1:-1, 1:-1, 1:-1]
    return np.pad(g, [(0, 0), (0, 0), (1, 1), (1, 1), (1, 1)])


def ducros(gu):
    """wmles/viscous.py:22-25"""
    div = gu[0, 0] + gu[1, 1] + gu[2, 2]
    w2 = (gu[2, 1] - gu[1, 2]) ** 2 + (gu[0, 2] - gu[2, 0]) ** 2 + (gu[1, 0] - gu[0, 1]) ** 2
    return div ** 2 / (div ** 2 + w2 + 1e-30)


def viscous_flux(blk, geom, d, phi, g, mu_eff, k_eff):
    """Face flux with the compact two-cell gradient correction; wmles/viscous.py:28-51"""
    Lf = lambda a: blk.slab(a, d, -1, 0)
    Rf = lambda a: blk.slab(a, d, 0, 1)
    gbar = 0.5 * (Lf(g) + Rf(g))
    dx = Rf(geom.xc) - Lf(geom.xc)
    dist = np.sqrt(sum3(dx * dx))
    e = dx / dist
    corr = (Rf(phi) - Lf(phi)) / dist - (gbar[:, 0] * e[0] + gbar[:, 1] * e[1] + gbar[:, 2] * e[2])
    gf = gbar + corr[:, None] * e[None]
    uf = 0.5 * (Lf(phi[:3]) + Rf(phi[:3]))
    muf = 0.5 * (Lf(mu_eff) + Rf(mu_eff))
    kf = 0.5 * (Lf(k_eff) + Rf(k_eff))
    S = blk.slab(geom.S[d], d, 0, 1)
    gu = gf[:3]
    div = gu[0, 0] + gu[1, 1] + gu[2, 2]
    eye = np.eye(3).reshape(3, 3, 1, 1, 1)
    tau = muf * (gu + np.swapaxes(gu, 0, 1) - (2.0 / 3.0) * eye * div)
    tauS = tau[:, 0] * S[0] + tau[:, 1] * S[1] + tau[:, 2] * S[2]
    dTdn = gf[3, 0] * S[0] + gf[3, 1] * S[1] + gf[3, 2] * S[2]
    return np.concatenate([np.zeros_like(div)[None], -tauS,
                           (-sum3(uf * tauS) - kf * dTdn)[None]], axis=0)


# ----------------------------------------------------------------------------- SGS
def sgs_nut(model, g, delta):
    """nu_t of wmles/sgs.py:14-42 from g[i, j] = du_i/dx_j (3, 3, ...)."""
    name, c = model.name, model.coeff
    if name == "smagorinsky":
        S = 0.5 * (g + np.swapaxes(g, 0, 1))
        return (c * delta) ** 2 * np.sqrt(2.0 * np.sum(S * S, axis=(0, 1)))
    if name == "wale":
        S = 0.5 * (g + np.swapaxes(g, 0, 1))
        SS = np.sum(S * S, axis=(0, 1))
        g2 = np.einsum('ik...,kj...->ij...', g, g)
        tr = g2[0, 0] + g2[1, 1] + g2[2, 2]
        Sd = 0.5 * (g2 + np.swapaxes(g2, 0, 1)) - np.eye(3).reshape(3, 3, 1, 1, 1) * tr / 3.0
        SdSd = np.sum(Sd * Sd, axis=(0, 1))
        return (c * delta) ** 2 * SdSd ** 1.5 / (SS ** 2.5 + SdSd ** 1.25 + 1e-30)
    if name == "vreman":
        beta = delta ** 2 * np.einsum('im...,jm...->ij...', g, g)
        B = (beta[0, 0] * beta[1, 1] - beta[0, 1] ** 2 + beta[0, 0] * beta[2, 2]
             - beta[0, 2] ** 2 + beta[1, 1] * beta[2, 2] - beta[1, 2] ** 2)
        aa = np.sum(g * g, axis=(0, 1))
        return 2.5 * c ** 2 * np.sqrt(np.maximum(B, 0.0) / (aa + 1e-30))
    raise KeyError(name)


# ----------------------------------------------------------------------------- wall model
def spalding_utau(wm, h, U, rho_w, mu_w):
    """Safeguarded Newton on Spalding's law, wmles/wall_model.py:19-40"""
    k = wm.kappa
    ekb = np.exp(-k * wm.B)
    Reh = h * U * rho_w / mu_w
    up = np.clip(np.sqrt(Reh), 1.0, 25.0)
    for _ in range(wm.n_iter):
        ku = k * up
        F = up + ekb * (np.exp(ku) - 1.0 - ku - 0.5 * ku ** 2 - ku ** 3 / 6.0) - Reh / up
        dF = 1.0 + ekb * k * (np.exp(ku) - 1.0 - ku - 0.5 * ku ** 2) + Reh / up ** 2
        up = np.minimum(np.maximum(up - F / dF, 0.5 * up), 100.0)
    return U / up


def equilibrium_wall(wm, gas, h, U, T_h, p_h, T_wall):
    """(tau_w, q_w) of wmles/wall_model.py:42-61"""
    Pr = gas.Pr
    U = np.maximum(U, 1e-8)
    if T_wall is None:
        T_w = T_h + Pr ** (1.0 / 3.0) * U ** 2 / (2.0 * gas.cp)
    else:
        T_w = T_wall + 0.0 * T_h
    rho_w = p_h / (gas.R * T_w)
    mu_w = viscosity(gas, T_w)
    ut = spalding_utau(wm, h, U, rho_w, mu_w)
    tau_w = rho_w * ut ** 2
    if T_wall is None:
        return tau_w, 0.0 * tau_w
    yp = np.maximum(h * ut * rho_w / mu_w, 1e-6)
    Gam = np.maximum(0.01 * (Pr * yp) ** 4 / (1.0 + 5.0 * Pr ** 3 * yp), 1e-20)
    beta = (3.85 * Pr ** (1 / 3) - 1.3) ** 2 + 2.12 * np.log(Pr)
    Tp = Pr * yp * np.exp(-Gam) + (2.12 * np.log(1.0 + yp) + beta) * np.exp(-1.0 / Gam)
    return tau_w, rho_w * gas.cp * ut * (T_w - T_h) / Tp


def wall_face_flux(bc, w, T, blk, geom, gas, axis, side):
    """Wall-face flux override and (tau_w, q_w); wmles/bc.py:145-166"""
    ng, n = blk.ng, blk.n[axis]
    fb = ng if side == 0 else ng + n
    mi = ng + bc.n_match - 1 if side == 0 else ng + n - bc.n_match
    ci = ng if side == 0 else ng + n - 1
    S = blk.take(geom.S[axis], axis, fb)
    Sm = np.sqrt(sum3(S * S))
    n_out = S / Sm if side == 1 else -S / Sm
    h = sum3((blk.take(geom.xc, axis, mi) - blk.take(geom.xf[axis], axis, fb)) * (-n_out))
    u = blk.take(w[1:4], axis, mi)
    u_par = u - sum3(u * n_out) * n_out
    U = np.sqrt(sum3(u_par * u_par) + 1e-20)
    T_h, p_h = blk.take(T, axis, mi), blk.take(w[4], axis, mi)
    p_b = blk.take(w[4], axis, ci)
    tau, qw = equilibrium_wall(bc.model, gas, h, U, T_h, p_h, bc.T_wall)
    t = u_par / U
    F = np.concatenate([np.zeros_like(tau)[None], (p_b * n_out + tau * t) * Sm, (-qw * Sm)[None]], axis=0)
    return (F if side == 1 else -F), tau, qw


# ----------------------------------------------------------------------------- solver
class OracleSolver:
    """NumPy float64 restatement of ``wmles.solver.Solver`` (wmles/solver.py:39-232)."""

    def __init__(self, mesh, gas, scheme, sgs="vreman", cfl=0.8, sgs_kwargs=None,
                 constraints=(), sources=(), bc_passes=2):
        self.mesh, self.blocks, self.gas = mesh, mesh.blocks, gas
        self.geoms = mesh.geoms
        self.scheme, self.cfl = scheme, cfl
        self.sgs = make_sgs(sgs, **(sgs_kwargs or {}))
        self.constraints, self.sources, self.bc_passes = tuple(constraints), tuple(sources), bc_passes
        self._xmaps = {}

    # ---- ghost cells: wmles/solver.py:59-73
    def _exchange(self, q, src, ib, face, itf):
        key = (ib, face)
        if key not in self._xmaps:
            blk, nb = self.blocks[ib], self.blocks[itf.nb]
            self._xmaps[key] = interface_index_map(blk.N, nb.N, blk.ng, blk.n[face[0]],
                                                   nb.n[itf.src_face[0]], face, itf, "cell")
        dst_flat, src_flat = self._xmaps[key]
        out = q.copy()
        out.reshape(5, -1)[:, dst_flat] = src.reshape(5, -1)[:, src_flat]
        return out

    def _mirror(self, q, blk, geom, axis, side, fn):
        """ghost layer m <- fn(interior layer m, unit normal); wmles/bc.py:14-25"""
        ng, n = blk.ng, blk.n[axis]
        fb = ng if side == 0 else ng + n
        S = geom.S[axis][sl(4, axis, slice(fb, fb + 1))]
        nrm = S / np.sqrt(sum3(S * S))
        q = q.copy()
        for m in range(ng):
            gi = ng - 1 - m if side == 0 else ng + n + m
            ii = ng + m if side == 0 else ng + n - 1 - m
            q[sl(4, axis, slice(gi, gi + 1))] = fn(q[sl(4, axis, slice(ii, ii + 1))], nrm)
        return q

    def _fill(self, bc, q, blk, geom, axis, side, time):
        gas = self.gas
        if isinstance(bc, (SlipWall, WallModel)):
            return self._mirror(q, blk, geom, axis, side, lambda s, n: slip_map(gas, s, n))
        if isinstance(bc, NoSlipWall):
            return self._mirror(q, blk, geom, axis, side, lambda s, n: noslip_map(gas, s, bc.T_wall))
        if isinstance(bc, Dirichlet):
            return self._mirror(q, blk, geom, axis, side, lambda s, n: dirichlet_map(gas, s, bc.prim))
        if isinstance(bc, CharacteristicFarfield):
            return self._mirror(q, blk, geom, axis, side,
                                lambda s, n: farfield_map(gas, s, n, bc.prim, side))
        if isinstance(bc, Extrapolate):
            ng, n = blk.ng, blk.n[axis]
            ii = ng if side == 0 else ng + n - 1
            edge = q[sl(4, axis, slice(ii, ii + 1))].copy()
            return self._mirror(q, blk, geom, axis, side, lambda s, nrm: edge)
        if isinstance(bc, SmoothRampInflow):
            if axis != 0 or side != 0:
                raise ValueError("SmoothRampInflow is only valid on the i-min face")
            return inflow_fill(bc, gas, q, blk, geom, time)
        raise NotImplementedError(type(bc).__name__)

    def apply_bcs(self, Q, time=0.0):
        Q = [np.asarray(q, float) for q in Q]
        for _ in range(self.bc_passes):
            for a in range(3):
                for ib, blk in enumerate(self.blocks):
                    q = Q[ib]
                    for s in (0, 1):
                        f = blk.faces[(a, s)]
                        if isinstance(f, Interface):
                            src = q if f.nb == ib else Q[f.nb]
                            q = self._exchange(q, src, ib, (a, s), f)
                        else:
                            q = self._fill(f, q, blk, self.geoms[ib], a, s, time)
                    Q[ib] = q
        return tuple(Q)

    # ---- RHS: wmles/solver.py:76-106
    def block_rhs(self, ib, q, geom):
        blk, gas = self.blocks[ib], self.gas
        w, T = cons_to_prim(gas, q)
        mu = viscosity(gas, T)
        phi = np.concatenate([w[1:4], T[None]], axis=0)
        g = green_gauss(phi, geom)
        if self.sgs.name == "none":
            mut = 0.0 * w[0]
        else:
            mut = w[0] * sgs_nut(self.sgs, g[:3], geom.vol ** (1.0 / 3.0))
        mu_eff = mu + mut
        k_eff = gas.cp * (mu / gas.Pr + mut / gas.Pr_t)
        theta = ducros(g[:3])
        rhs = 0.0
        for d in range(3):
            F = (inviscid_flux(self.scheme, blk, geom, w, gas, d, theta)
                 + viscous_flux(blk, geom, d, phi, g, mu_eff, k_eff))
            for s in (0, 1):
                bc = blk.faces[(d, s)]
                if getattr(bc, "flux_override", False):
                    Fw, _, _ = wall_face_flux(bc, w, T, blk, geom, gas, d, s)
                    F = F.copy()
                    F[sl(F.ndim, d, 0 if s == 0 else blk.n[d])] = Fw
            rhs = rhs - (F[sl(F.ndim, d, slice(1, None))] - F[sl(F.ndim, d, slice(None, -1))])
        return rhs / blk.interior(geom.vol)

    def rhs(self, Q, time=0.0):
        Q = self.apply_bcs(Q, time)
        ng = self.mesh.ng
        out = []
        for ib, (q, g) in enumerate(zip(Q, self.geoms)):
            r = self.block_rhs(ib, q, g)
            for src in self.sources:
                r = r + sponge_source(src, self.blocks[ib], q, g)
            out.append(np.pad(r, [(0, 0)] + [(ng, ng)] * 3))
        return tuple(out)

    # ---- time stepping: wmles/solver.py:110-133
    def advance(self, Q, dt, time=0.0):
        R0 = self.rhs(Q, time)
        Q1 = tuple(q + dt * r for q, r in zip(Q, R0))
        R1 = self.rhs(Q1, time + dt)
        Q2 = tuple(0.75 * q0 + 0.25 * (q1 + dt * r1) for q0, q1, r1 in zip(Q, Q1, R1))
        R2 = self.rhs(Q2, time + 0.5 * dt)
        Q3 = tuple((1.0 / 3.0) * q0 + (2.0 / 3.0) * (q2 + dt * r2) for q0, q2, r2 in zip(Q, Q2, R2))
        for c in self.constraints:
            Q3 = constant_mass_flux(c, Q3, self.geoms, self.blocks)
        return Q3

    def max_dt(self, Q, time=0.0):
        """CFL time step, wmles/solver.py:135-151"""
        gas = self.gas
        Q = self.apply_bcs(Q, time)
        dts = []
        for blk, q, g in zip(self.blocks, Q, self.geoms):
            w, T = cons_to_prim(gas, q)
            c = sound_speed(gas, T)
            nu = max(4.0 / 3.0, gas.gamma / gas.Pr) * viscosity(gas, T) / w[0]
            lam, lamv = 0.0, 0.0
            for d in range(3):
                Sd = g.S[d]
                Sb = 0.5 * (Sd[sl(4, d, slice(0, -1))] + Sd[sl(4, d, slice(1, None))])
                Sm = np.sqrt(sum3(Sb * Sb))
                lam = lam + np.abs(sum3(w[1:4] * Sb)) + c * Sm
                lamv = lamv + nu * Sm ** 2 / g.vol
            dts.append(np.min(blk.interior(self.cfl / ((lam + 4.0 * lamv) / g.vol))))
        return np.min(np.stack(dts))

    # ---- diagnostics: wmles/solver.py:163-232
    def wall_stats(self, Q):
        Q = self.apply_bcs(Q)
        out = {}
        for blk, q, g in zip(self.blocks, Q, self.geoms):
            w, T = cons_to_prim(self.gas, q)
            for (a, s), bc in blk.faces.items():
                if isinstance(bc, WallModel):
                    _, tau, qw = wall_face_flux(bc, w, T, blk, g, self.gas, a, s)
                    out[(blk.name, "ijk"[a] + ("min", "max")[s])] = (tau, qw)
        return out

    def wall_loads(self, Q, moment_center=(0.0, 0.0, 0.0)):
        center = np.asarray(moment_center, float)
        Q = self.apply_bcs(Q)
        out = {}
        for blk, q, g in zip(self.blocks, Q, self.geoms):
            w, T = cons_to_prim(self.gas, q)
            for (a, s), bc in blk.faces.items():
                if not isinstance(bc, WallModel):
                    continue
                ng, n = blk.ng, blk.n[a]
                fb = ng if s == 0 else ng + n
                mi = ng + bc.n_match - 1 if s == 0 else ng + n - bc.n_match
                ci = ng if s == 0 else ng + n - 1
                Sv = blk.take(g.S[a], a, fb)
                area = np.sqrt(sum3(Sv * Sv))
                nrm = Sv / area
                if s == 0:
                    nrm = -nrm
                vel = blk.take(w[1:4], a, mi)
                vt = vel - sum3(vel * nrm)[None] * nrm
                speed = np.sqrt(sum3(vt ** 2) + 1e-20)
                tang = vt / speed
                _, tau, _ = wall_face_flux(bc, w, T, blk, g, self.gas, a, s)
                pw = blk.take(w[4], a, ci)
                trac = (pw[None] * nrm + tau[None] * tang) * area[None]
                arm = blk.take(g.xf[a], a, fb) - center.reshape(3, 1, 1)
                mom = np.stack([arm[1] * trac[2] - arm[2] * trac[1],
                                arm[2] * trac[0] - arm[0] * trac[2],
                                arm[0] * trac[1] - arm[1] * trac[0]])
                out[(blk.name, "ijk"[a] + ("min", "max")[s])] = (
                    np.sum(trac, axis=(1, 2)), np.sum(mom, axis=(1, 2)))
        return out


def constant_mass_flux(c, Q, geoms, blocks):
    """wmles/solver.py:16-36"""
    num, den = 0.0, 0.0
    for q, g, b in zip(Q, geoms, blocks):
        vol = b.interior(g.vol)
        num = num + np.sum(b.interior(q[1 + c.dir]) * vol)
        den = den + np.sum(vol)
    delta = c.target - num / den
    out = []
    for q in Q:
        z = np.zeros_like(q[0])
        mom = [z, z, z]
        mom[c.dir] = z + delta
        dE = (2.0 * q[1 + c.dir] * delta + delta ** 2) / (2.0 * q[0])
        out.append(q + np.stack([z] + mom + [dE]))
    return tuple(out)


def sponge_source(src, blk, q, geom):
    """wmles/smooth_ramp.py:212-221"""
    if not isinstance(src, SmoothRampSponge):
        raise NotImplementedError(type(src).__name__)
    q_int = blk.interior(q)
    vol = blk.interior(geom.vol)
    mean = np.sum(q_int * vol[None], axis=3, keepdims=True) / np.sum(vol, axis=2, keepdims=True)[None]
    x_l = blk.interior(geom.xc[0]) / src.props["L"]
    eta = np.clip((x_l - src.x_start_l) / (src.x_end_l - src.x_start_l), 0.0, 1.0)
    ramp = eta ** 3 * (10.0 + eta * (-15.0 + 6.0 * eta))
    sigma = src.strength * src.props["U_inf"] / src.props["L"] * ramp
    return -sigma[None] * (q_int - mean)


def init_state(solver, prim_fn):
    """wmles/solver.py:54-56 (host arrays)."""
    return tuple(prim_to_cons(solver.gas, np.asarray(prim_fn(g.xc), float)) for g in solver.geoms)


def plane_means(gas, blk, q):
    """Per interior j-plane means over interior (i, k) of rho, u, v, w, uu, vv, ww, uv, uw,
    vw, T, p for one sample of one block; PlaneStats.accumulate, wmles/channel5200.py:135-151."""
    w, T = cons_to_prim(gas, q)
    u, v, wc = (blk.interior(c) for c in w[1:4])
    rho, Ta, p = blk.interior(w[0]), blk.interior(T), blk.interior(w[4])
    ax = (0, 2)
    return {"rho": rho.mean(axis=ax), "u": u.mean(axis=ax), "v": v.mean(axis=ax), "w": wc.mean(axis=ax),
            "uu": (u * u).mean(axis=ax), "vv": (v * v).mean(axis=ax), "ww": (wc * wc).mean(axis=ax),
            "uv": (u * v).mean(axis=ax), "uw": (u * wc).mean(axis=ax), "vw": (v * wc).mean(axis=ax),
            "T": Ta.mean(axis=ax), "p": p.mean(axis=ax)}


def derived_fields(solver, Q):
    """{block: {name: interior array}} of rho, velocity, pressure, temperature, Mach, mu_t,
    mu, |omega| and Q-criterion; wmles/io_vtk.py:269-293 (ghost cells filled first)."""
    gas = solver.gas
    Q = solver.apply_bcs(Q)
    out = {}
    for ib, (blk, q, geom) in enumerate(zip(solver.blocks, Q, solver.geoms)):
        w, T = cons_to_prim(gas, q)
        mu = viscosity(gas, T)
        g = green_gauss(w[1:4], geom)
        mut = 0.0 * w[0] if solver.sgs.name == "none" else w[0] * sgs_nut(solver.sgs, g, geom.vol ** (1.0 / 3.0))
        wxy, wxz, wyz = g[1, 0] - g[0, 1], g[2, 0] - g[0, 2], g[2, 1] - g[1, 2]
        omega = np.sqrt(wxy ** 2 + wxz ** 2 + wyz ** 2)
        S = 0.5 * (g + np.swapaxes(g, 0, 1))
        Om = 0.5 * (g - np.swapaxes(g, 0, 1))
        qcrit = 0.5 * (np.sum(Om ** 2, axis=(0, 1)) - np.sum(S ** 2, axis=(0, 1)))
        mach = np.sqrt(np.sum(w[1:4] ** 2, axis=0)) / sound_speed(gas, T)
        out[ib] = {"rho": blk.interior(w[0]), "velocity": blk.interior(w[1:4]), "pressure": blk.interior(w[4]),
                   "temperature": blk.interior(T), "mach": blk.interior(mach), "mu_t": blk.interior(mut),
                   "mu": blk.interior(mu), "vorticity_mag": blk.interior(omega), "q_criterion": blk.interior(qcrit)}
    return out
