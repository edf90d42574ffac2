"""Inviscid face-flux schemes (descriptors; the flux arithmetic lives in the CUDA stage
kernel, wmles_jax_b200/csrc/physics.cuh).

* ``KEP(order)``  Kennedy-Gruber split-form central flux, order 2 or 4
  (wmles/schemes.py:15-23,57-70).
* ``MUSCLHLLC(limiter)``  MUSCL reconstruction of primitives (van Albada or minmod) with a
  positivity fallback, then HLLC (wmles/schemes.py:100-152).
* ``Hybrid(central, upwind, th0, th1)``  F = (1-s) F_central + s F_upwind with
  s = clip((max(theta_L, theta_R) - th0) / (th1 - th0), 0, 1) (wmles/schemes.py:155-166).
"""


class KEP:
    def __init__(self, order=4):
        if order not in (2, 4):
            raise ValueError("KEP order must be 2 or 4")
        self.order = order


class MUSCLHLLC:
    LIMITERS = ("albada", "minmod")

    def __init__(self, limiter="albada"):
        if limiter not in self.LIMITERS:
            raise KeyError(limiter)
        self.limiter = limiter


class Hybrid:
    def __init__(self, central=None, upwind=None, th0=0.6, th1=0.9):
        self.c = central or KEP(4)
        self.u = upwind or MUSCLHLLC()
        self.th0, self.th1 = th0, th1
        if not isinstance(self.c, KEP) or not isinstance(self.u, MUSCLHLLC):
            raise NotImplementedError("Hybrid blends a KEP central flux with a MUSCLHLLC upwind flux")
