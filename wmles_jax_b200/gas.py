"""Calorically perfect gas with Sutherland viscosity (host-side parameters).

Mirrors the constructor and formulas of the reference ``Gas`` (wmles/gas.py:10-41):
conservative layout q = [rho, rho u, rho v, rho w, rho E], primitive layout
w = [rho, u, v, w, p].  On the cuda backend the per-cell conversions run inside the
CUDA kernels; the methods here serve initial conditions, set-up and driver diagnostics,
on host NumPy arrays (the same operation order as the reference, so host results are
bit-identical) or on device tensors (through ``xp``, e.g. ``gas.cons_to_prim(Q[0])`` on a
state, as tests/test_sod.py:25 does).
"""
from dataclasses import dataclass

from .arrays import xp


@dataclass(frozen=True)
class Gas:
    gamma: float = 1.4
    R: float = 287.05
    Pr: float = 0.72
    Pr_t: float = 0.9
    mu_ref: float = 1.716e-5
    T_ref: float = 273.15
    S_suth: float = 110.4

    @property
    def cp(self):
        return self.gamma * self.R / (self.gamma - 1.0)

    def mu(self, T):
        """Sutherland law, wmles/gas.py:24-26."""
        return (self.mu_ref * (T / self.T_ref) ** 1.5
                * (self.T_ref + self.S_suth) / (T + self.S_suth))

    def cons_to_prim(self, q):
        """(5, ...) conservative -> ((5, ...) primitive, T); wmles/gas.py:28-33."""
        q = xp.asarray(q)
        rho = q[0]
        vel = q[1:4] / rho
        ke = vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]
        p = (self.gamma - 1.0) * (q[4] - 0.5 * rho * ke)
        T = p / (rho * self.R)
        return xp.concatenate([rho[None], vel, p[None]], axis=0), T

    def prim_to_cons(self, w):
        """(5, ...) primitive -> conservative; wmles/gas.py:35-38."""
        w = xp.asarray(w)
        rho, vel, p = w[0], w[1:4], w[4]
        ke = vel[0] * vel[0] + vel[1] * vel[1] + vel[2] * vel[2]
        E = p / (self.gamma - 1.0) + 0.5 * rho * ke
        return xp.concatenate([rho[None], rho * vel, E[None]], axis=0)

    def sound_speed(self, T):
        return xp.sqrt(self.gamma * self.R * xp.asarray(T))
