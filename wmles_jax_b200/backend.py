"""Backend selection for the B200 build (cf. wmles/backend.py:18-56).

``WMLES_BACKEND=cuda`` selects this package's CUDA path.  There is no fallback: the
solver raises if the CUDA library cannot be loaded or no GPU is visible.
``WMLES_DEVICE`` keeps the reference's accepted values (auto, cpu, gpu, cuda); ``cpu`` is
rejected for the cuda backend because this path has no CPU implementation.
Host-side set-up (meshes, initial conditions) uses NumPy, exposed as ``xp``.
"""
import os

import numpy as xp  # noqa: F401  (host-side array namespace for set-up code)

BACKEND = os.environ.get("WMLES_BACKEND", "cuda").strip().lower() or "cuda"
DEVICE_REQUEST = os.environ.get("WMLES_DEVICE", "auto").strip().lower()
if DEVICE_REQUEST not in {"auto", "cpu", "gpu", "cuda"}:
    raise ValueError("WMLES_DEVICE must be one of: auto, cpu, gpu, cuda")
HAS_JAX = False


def require_gpu():
    """Raise unless a CUDA device is usable; returns the torch device."""
    if DEVICE_REQUEST == "cpu":
        raise RuntimeError("WMLES_DEVICE=cpu: the cuda backend has no CPU path")
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("WMLES_BACKEND=cuda needs a visible CUDA device (none found)")
    return torch.device("cuda", torch.cuda.current_device())


def device_info():
    try:
        import torch
        if torch.cuda.is_available():
            i = torch.cuda.current_device()
            return f"cuda:{i}:{torch.cuda.get_device_name(i)}"
    except Exception:  # pragma: no cover - torch import failure is reported by the solver
        pass
    return "cuda:unavailable"


def asarray(value, dtype=None):
    """``value`` as a tensor on the selected CUDA device (cf. wmles/backend.py:51-54, which
    places arrays on the JAX device); NumPy dtype semantics for ``dtype``."""
    import torch
    return torch.from_numpy(xp.ascontiguousarray(xp.asarray(value, dtype=dtype))).to(require_gpu())


def __getattr__(name):
    # DEVICE (wmles/backend.py:32): the torch device of the cuda path, None without a GPU;
    # resolved on access so that importing the package needs no GPU
    if name == "DEVICE":
        try:
            return require_gpu()
        except RuntimeError:
            return None
    raise AttributeError(name)
