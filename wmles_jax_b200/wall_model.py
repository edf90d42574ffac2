"""Equilibrium wall model descriptor (wmles/wall_model.py:15-61).

Spalding's law F(u+) = u+ + e^{-kB}(e^{k u+} - 1 - k u+ - (k u+)^2/2 - (k u+)^3/6) - Re_h/u+
is solved for u+ by ``n_iter`` safeguarded Newton steps (clipped to [0.5 u+, 100],
start clip(sqrt(Re_h), 1, 25)); the wall heat flux uses Kader's temperature law for an
isothermal wall, or the recovery temperature with q_w = 0 for an adiabatic wall.
The solve runs per wall face in FP64 in the CUDA wall kernel (``wall_face`` in csrc/surface.cu).
"""


class EquilibriumWallModel:
    def __init__(self, kappa=0.41, B=5.2, n_iter=30):
        self.kappa, self.B, self.n_iter = kappa, B, n_iter
