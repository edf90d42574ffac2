"""A ``wmles`` package that resolves to the cuda backend: the import binding a maintainer
adds to the reference's ``wmles/__init__.py`` for ``WMLES_BACKEND=cuda`` (the names of
wmles/__init__.py:1-7), packaged on its own so that driver code written against the
reference's public API runs here unmodified.  Only tests put it on ``sys.path``."""
from wmles_jax_b200 import (HAS_JAX, Gas, Block, Mesh, SlipWall, NoSlipWall, Dirichlet,  # noqa: F401
                            CharacteristicFarfield, Extrapolate, WallModel, EquilibriumWallModel,
                            KEP, MUSCLHLLC, Hybrid, Solver, ConstantMassFlux)
