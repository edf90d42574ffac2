"""Smooth-ramp boundary physics that runs every RK stage: synthetic-turbulence inflow
and the spanwise-mean sponge (descriptors; device code in csrc/inflow.cu and the stage
kernel's source term).

``SmoothRampInflow`` (wmles/smooth_ramp.py:116-197): per i-min ghost layer, three
unit-variance Fourier fields (``n_modes`` cosines in (U t / L, y / L, z / L)) are made
zero-mean over the interior span, the second is decorrelated from the first, each is
normalised by its span variance, and the velocity is the profile-table mean plus a
Cholesky-style mix of the fields by the table's Reynolds stresses.  The mode table is
drawn here, once, with NumPy's ``default_rng(seed + component)`` in the reference's
draw order (normal kx, normal ky, weighted choice of kz, uniform phase) so that the
modes are identical to the reference's.

``SmoothRampSponge`` (wmles/smooth_ramp.py:200-221): r += -sigma(x) (q - <q>_z) with a
quintic ramp sigma over [x_start, x_end] and a volume-weighted spanwise mean.
"""
import numpy as np

from .bc import BC

SPAN_L = 0.288


class SmoothRampInflow(BC):
    def __init__(self, props, profile, length_scales=(0.1, 0.02, 0.03),
                 seed=0, n_modes=64, span_cells=16):
        length_scales = np.asarray(length_scales, dtype=float)
        if (length_scales.shape != (3,) or not np.all(np.isfinite(length_scales))
                or np.any(length_scales <= 0.0)):
            raise ValueError("inflow length_scales must contain three positive finite values")
        if seed < 0:
            raise ValueError("inflow seed must be non-negative")
        if n_modes < 4 or span_cells < 3:
            raise ValueError("inflow synthesis needs at least four modes and three spanwise cells")
        self.props, self.profile = props, np.asarray(profile, dtype=float)
        self.length_scales = tuple(length_scales)
        self.seed, self.n_modes = int(seed), int(n_modes)
        half = max(1, span_cells // 2)
        wavenumbers = np.array([m for m in range(-half, half + 1) if m != 0])
        kz_choices = 2.0 * np.pi * wavenumbers / SPAN_L
        weights = np.exp(-0.5 * (kz_choices * length_scales[2]) ** 2)
        weights /= np.sum(weights)
        self._modes = []
        for comp in range(3):
            gen = np.random.default_rng(self.seed + comp)
            kx = gen.normal(0.0, 1.0 / length_scales[0], n_modes)
            ky = gen.normal(0.0, 1.0 / length_scales[1], n_modes)
            kz = gen.choice(kz_choices, size=n_modes, p=weights)
            ph = gen.uniform(0.0, 2.0 * np.pi, n_modes)
            self._modes.append((kx, ky, kz, ph))

    def mode_table(self):
        """(3, 4, n_modes) float64: [component][kx, ky, kz, phase][mode]."""
        return np.array([[np.asarray(v, float) for v in m] for m in self._modes])


class SmoothRampSponge:
    def __init__(self, props, x_start_l, x_end_l, strength=1.0):
        if not np.isfinite(strength) or strength < 0.0:
            raise ValueError("sponge strength must be finite and non-negative")
        if not np.isfinite(x_start_l + x_end_l) or x_start_l >= x_end_l:
            raise ValueError("sponge start must be finite and upstream of its end")
        self.props = props
        self.x_start_l, self.x_end_l = float(x_start_l), float(x_end_l)
        self.strength = float(strength)
