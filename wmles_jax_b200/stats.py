"""Plane statistics of a channel on the device (PlaneStats, wmles/channel5200.py:121-199).

``PlaneStats(mesh, solver)`` keeps the reference's interface: ``accumulate(Q)`` adds one
sample, ``result()`` returns ``(y, averages)``, ``mean_tau_w`` and ``wall_units(...)``
give the inner-scaled profiles.  The per-plane means of block 0 (rho, u, v, w, uu, vv, ww,
uv, uw, vw, T, p over interior (i, k)) are summed on the device by ``wm_plane_stats``, and
the wall shear stress of every wall-modelled face by ``wm_wall_stats``, so sampling costs
two small launches and no host copy; only ``result()`` copies the 12 x nj sums.  As in the
reference, block 0 must have one y per j-plane (an unskewed channel block).
"""
import numpy as np
import torch

from . import _native as N

KEYS = ("rho", "u", "v", "w", "uu", "vv", "ww", "uv", "uw", "vw", "T", "p")


class PlaneStats:
    def __init__(self, mesh, solver):
        self.mesh, self.solver = mesh, solver
        blk, geom = mesh.blocks[0], solver.host_geoms[0]
        self.y = np.asarray(blk.interior(geom.xc[1]))[0, :, 0]
        self.n = 0
        self._sum = torch.zeros((len(KEYS), blk.n[1]), dtype=torch.float64, device=solver.device)
        self._tau = torch.zeros((), dtype=torch.float64, device=solver.device)

    def accumulate(self, Q):
        """Add the plane means and the mean wall shear stress of state Q (device work only)."""
        s = self.solver
        s._check_state(Q)
        N.check(s._lib.wm_plane_stats(s._case, 0, N.ptr_array([Q[0].data_ptr()])[0],
                                      N.ptr_array([self._sum.data_ptr()])[0], s._stream()), "wm_plane_stats")
        walls = s.wall_stats_device(Q)
        if walls:
            # mean over walls of each wall's mean tau_w (the reference's sampling)
            self._tau += torch.stack([buf[0].mean() for buf in walls.values()]).mean()
        self.n += 1

    def result(self):
        """(y, {quantity: profile}) with the second moments turned into covariances."""
        if self.n == 0:
            raise RuntimeError("call accumulate() at least once before result()")
        avg = {k: v / self.n for k, v in zip(KEYS, self._sum.cpu().numpy())}
        for a, b in (("u", "u"), ("v", "v"), ("w", "w"), ("u", "v"), ("u", "w"), ("v", "w")):
            key = a + b
            avg[key] = avg[key] - avg[a] * avg[b]
        return self.y, avg

    @property
    def mean_tau_w(self):
        if self.n == 0:
            raise RuntimeError("call accumulate() at least once before mean_tau_w")
        return float(self._tau) / self.n

    def wall_units(self, tau_w, rho_w, mu_w, h):
        """(u_tau, inner-scaled profiles of the lower half y < h): y/delta, y+, U+, dU/dy+
        (second-order differences in y+), W+, P+ (pressure above the wall value, linearly
        extrapolated from the first two planes), the six Reynolds stresses over u_tau^2 and
        k+ = (uu+ + vv+ + ww+) / 2."""
        y, avg = self.result()
        u_tau = np.sqrt(tau_w / rho_w)
        lower = y < h
        yl = y[lower]
        yp = yl * u_tau / (mu_w / rho_w)
        up = avg["u"][lower] / u_tau
        p = avg["p"][lower]
        p_wall = p[0] - yl[0] * (p[1] - p[0]) / (yl[1] - yl[0])
        stress = u_tau ** 2
        out = {"y/delta": yl / h, "y+": yp, "U+": up, "dU/dy+": np.gradient(up, yp),
               "W+": avg["w"][lower] / u_tau, "P+": (p - p_wall) / (rho_w * stress)}
        for key in ("uu", "vv", "ww", "uv", "uw", "vw"):
            out[key + "+"] = avg[key][lower] / stress
        out["k+"] = 0.5 * (out["uu+"] + out["vv+"] + out["ww+"])
        return u_tau, out
