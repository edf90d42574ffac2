"""Post-step constraints (descriptors).

``ConstantMassFlux(direction, target)`` (wmles/solver.py:16-36): after each step the
volume-averaged rho u_dir over all block interiors is shifted to ``target`` by adding
delta = target - sum(rho u_dir V) / sum(V) to the momentum component and
(2 rho u_dir delta + delta^2) / (2 rho) to the energy, in every cell.  On the cuda
backend the sum is a fixed-order FP64 device reduction fused into the last RK stage.
"""


class ConstantMassFlux:
    def __init__(self, direction, target):
        if direction not in (0, 1, 2):
            raise ValueError("direction must be 0, 1 or 2")
        self.dir, self.target = direction, target
