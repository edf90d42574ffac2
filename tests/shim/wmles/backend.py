"""``wmles.backend`` of the cuda binding: the names drivers import from it
(examples/channel_wmles.py:15, tests/test_multiblock.py:7)."""
from wmles_jax_b200.backend import (DEVICE, HAS_JAX, asarray, device_info, fori_loop, jit,  # noqa: F401
                                    set_at, xp)
