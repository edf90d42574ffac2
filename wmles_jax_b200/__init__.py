"""B200-native backend of wmles (WMLES_BACKEND=cuda).

Public API of the reference package (wmles/__init__.py:1-9) for the explicit RHS +
SSP-RK3 hot path: the same classes and constructors, with the time step executed by
hand-written sm_100a CUDA kernels in ``libwmles_cuda.so`` (see ``include/wmles_cuda.h``).
State arrays are torch CUDA float64 tensors of shape (5, Ni, Nj, Nk), ghosts included.
"""
from .backend import HAS_JAX, device_info
from .gas import Gas
from .mesh import Block, Mesh
from .bc import SlipWall, NoSlipWall, Dirichlet, CharacteristicFarfield, Extrapolate, WallModel
from .wall_model import EquilibriumWallModel
from .schemes import KEP, MUSCLHLLC, Hybrid
from .sgs import make_sgs
from .constraints import ConstantMassFlux
from .smooth_ramp import SmoothRampInflow, SmoothRampSponge


def __getattr__(name):
    # the solver loads the CUDA library; import it lazily so that mesh set-up and the
    # descriptor classes stay usable on hosts without a GPU
    if name == "Solver":
        from .solver import Solver
        return Solver
    raise AttributeError(name)


__all__ = ["HAS_JAX", "device_info", "Gas", "Block", "Mesh", "SlipWall", "NoSlipWall", "Dirichlet",
           "CharacteristicFarfield", "Extrapolate", "WallModel", "EquilibriumWallModel", "KEP",
           "MUSCLHLLC", "Hybrid", "make_sgs", "ConstantMassFlux", "SmoothRampInflow",
           "SmoothRampSponge", "Solver"]
