"""Boundary conditions (descriptors lowered to the CUDA ghost-gather program).

Same classes and constructor arguments as the reference (wmles/bc.py:28-166).  On the
cuda backend a BC is not called per array: ``wmles_jax_b200.lowering`` traces the
reference's ghost-fill order symbolically and turns every ghost cell into a chain of
the per-cell maps below, which the ghost kernel replays on the device.

Ghost-cell maps (ghost layer m <- f(cell state, unit +axis normal n of the boundary face)):

* ``SlipWall``        reflect the normal velocity (wmles/bc.py:38-47)
* ``NoSlipWall``      negate velocity; T_g = max(2 T_w - T, 0.1 T_w) if isothermal
                      (wmles/bc.py:50-64)
* ``Dirichlet``       fixed primitive state (wmles/bc.py:67-77)
* ``CharacteristicFarfield`` linearised characteristics (wmles/bc.py:80-115)
* ``Extrapolate``     copy of the first interior layer (wmles/bc.py:118-125)
* ``WallModel``       slip ghosts + wall-face flux override from the wall model
                      (wmles/bc.py:128-166)
"""
import numpy as np


class BC:
    """Base class.  ``flux_override`` marks a BC whose wall-face flux replaces the
    numerical flux (wmles/bc.py:28-35)."""
    flux_override = False


class SlipWall(BC):
    pass


class NoSlipWall(BC):
    def __init__(self, T_wall=None):
        self.T_wall = T_wall


class Dirichlet(BC):
    def __init__(self, prim):
        self.prim = np.asarray(prim, float)


class CharacteristicFarfield(BC):
    def __init__(self, prim):
        self.prim = np.asarray(prim, float)


class Extrapolate(BC):
    pass


class WallModel(BC):
    """Wall-modelled LES wall: slip ghosts for the numerics, wall-face flux
    [0, p n + tau_w t, -q_w] |S| from ``model`` sampled ``n_match`` cells off the wall.
    ``T_wall=None`` means adiabatic."""
    flux_override = True

    def __init__(self, model, T_wall=None, n_match=1):
        self.model, self.T_wall, self.n_match = model, T_wall, n_match
        self._slip = SlipWall()
