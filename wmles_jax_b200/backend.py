"""Backend module of the B200 build (cf. wmles/backend.py:1-76).

This package is the ``WMLES_BACKEND=cuda`` path.  The variable is read at import, like the
reference reads it (wmles/backend.py:10): unset, empty or ``cuda`` select this path; any
other value (``numpy``, ``jax``) asks for one of the reference's own paths, which this
package does not implement, so constructing a ``Solver`` then raises instead of running on
the GPU.  There is no fallback either way: the solver raises if the CUDA library cannot be
loaded or no GPU is visible.  ``WMLES_DEVICE`` keeps the reference's accepted values (auto,
cpu, gpu, cuda); ``cpu`` is rejected because this path has no CPU implementation.

``xp`` works on host arrays (NumPy, bit for bit) and on device states (torch), see
``arrays.py``; ``set_at``, ``jit`` and ``fori_loop`` keep the reference's helpers for case
code that calls them (wmles/backend.py:57-76).
"""
import os

from .arrays import xp  # noqa: F401

BACKEND = os.environ.get("WMLES_BACKEND", "cuda").strip().lower() or "cuda"
DEVICE_REQUEST = os.environ.get("WMLES_DEVICE", "auto").strip().lower()
if DEVICE_REQUEST not in {"auto", "cpu", "gpu", "cuda"}:
    raise ValueError("WMLES_DEVICE must be one of: auto, cpu, gpu, cuda")
HAS_JAX = False


def require_gpu():
    """Raise unless this path is selected and a CUDA device is usable; returns the torch
    device."""
    if BACKEND != "cuda":
        raise RuntimeError(f"WMLES_BACKEND={BACKEND} selects the reference's own array path; "
                           "wmles_jax_b200 implements WMLES_BACKEND=cuda only")
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


def set_at(a, idx, v):
    """Functional ``a[idx] = v`` (a new array, wmles/backend.py:57-63) for NumPy arrays and
    torch tensors."""
    a = a.clone() if hasattr(a, "clone") else a.copy()
    a[idx] = v
    return a


def jit(fn, **kw):
    """No tracing compiler on this path: the step runs as CUDA kernels (wmles/backend.py:66)."""
    return fn


def fori_loop(lo, hi, body, init):
    """wmles/backend.py:70-76 without JAX: a plain loop."""
    x = init
    for i in range(lo, hi):
        x = body(i, x)
    return x


def __getattr__(name):
    # DEVICE (wmles/backend.py:32): the torch device of the cuda path, None without a GPU;
    # resolved on access so that importing the package needs no GPU
    if name == "DEVICE":
        try:
            return require_gpu()
        except RuntimeError:
            return None
    raise AttributeError(name)
