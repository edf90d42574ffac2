"""The ``xp`` array namespace of the cuda backend (cf. wmles/backend.py:18-41).

The reference's drivers and case modules call ``xp`` both on host set-up arrays (cell
centres handed to an initial-condition function) and on device states (``xp.min`` of the
density, ``xp.sum`` of the kinetic energy, examples/channel_wmles.py:53-59,141-143).  In
this backend set-up arrays are NumPy and states are torch CUDA tensors, so ``xp`` picks the
implementation from its arguments: any torch tensor among them (also inside a list or
tuple, as ``stack`` takes them) selects torch on that tensor's device, otherwise NumPy runs
unchanged, bit for bit, as the reference's NumPy path.  NumPy's ``axis`` / ``keepdims`` /
``dtype`` keywords are translated for torch; scalars and NumPy arrays mixed with a tensor
are moved to the tensor's device.  Non-callable attributes (``xp.pi``, ``xp.float64``,
``xp.newaxis``) are NumPy's.
"""
import sys

import numpy as np


def _t():
    import torch
    return torch


def _is_tensor(x):
    # a tensor exists only once torch is imported: never import it just to look
    torch = sys.modules.get("torch")
    return torch is not None and isinstance(x, torch.Tensor)


def _find_tensor(args, kwargs):
    for a in list(args) + list(kwargs.values()):
        if _is_tensor(a):
            return a
        if isinstance(a, (list, tuple)):
            for b in a:
                if _is_tensor(b):
                    return b
    return None


_DTYPES = {np.dtype("float64"): "float64", np.dtype("float32"): "float32", np.dtype("int64"): "int64",
           np.dtype("int32"): "int32", np.dtype("bool"): "bool"}


def _torch_dtype(dtype):
    if dtype is None or isinstance(dtype, _t().dtype):
        return dtype
    return getattr(_t(), _DTYPES[np.dtype(dtype)])


def _as_tensor(x, like):
    """x on the device of ``like`` (tensors pass through; NumPy arrays and scalars are
    converted, floating values in ``like``'s floating dtype)."""
    torch = _t()
    if isinstance(x, torch.Tensor):
        return x
    if isinstance(x, (list, tuple)):
        return [_as_tensor(v, like) for v in x]
    a = np.asarray(x)
    dt = like.dtype if (a.dtype.kind == "f" and like.dtype.is_floating_point) else None
    return torch.as_tensor(a, device=like.device, dtype=dt)


def _kw(kwargs):
    """NumPy reduction keywords -> torch."""
    out = dict(kwargs)
    if "axis" in out:
        ax = out.pop("axis")
        if ax is not None:
            out["dim"] = tuple(ax) if isinstance(ax, (list, tuple)) else ax
    if "keepdims" in out:
        out["keepdim"] = out.pop("keepdims")
    if "dtype" in out:
        out["dtype"] = _torch_dtype(out["dtype"])
    return out


def _reduce(name):
    def fn(a, axis=None, **kwargs):
        torch = _t()
        kw = _kw(kwargs)
        if axis is None:
            return getattr(torch, name)(a) if not kw else getattr(torch, name)(a, **kw)
        return getattr(torch, {"min": "amin", "max": "amax"}.get(name, name))(
            a, dim=tuple(axis) if isinstance(axis, (list, tuple)) else axis, **kw)
    return fn


def _binary(name):
    def fn(a, b, *rest, **kwargs):
        like = a if _is_tensor(a) else b
        return getattr(_t(), name)(_as_tensor(a, like), _as_tensor(b, like), *rest, **kwargs)
    return fn


def _clip(a, a_min=None, a_max=None, **kwargs):
    torch = _t()
    lo = a_min if (a_min is None or np.isscalar(a_min)) else _as_tensor(a_min, a)
    hi = a_max if (a_max is None or np.isscalar(a_max)) else _as_tensor(a_max, a)
    return torch.clamp(_as_tensor(a, lo if _is_tensor(lo) else hi), min=lo, max=hi)


def _join(name):
    def fn(arrays, axis=0, **kwargs):
        like = next(x for x in arrays if _is_tensor(x))
        return getattr(_t(), name)([_as_tensor(x, like) for x in arrays], dim=axis)
    return fn


def _where(cond, a=None, b=None):
    torch = _t()
    if a is None and b is None:
        return torch.where(cond)
    like = next(x for x in (cond, a, b) if _is_tensor(x))
    cond = _as_tensor(cond, like)
    a = a if np.isscalar(a) else _as_tensor(a, like)
    b = b if np.isscalar(b) else _as_tensor(b, like)
    return torch.where(cond, a, b)


def _asarray(a, dtype=None, **kwargs):
    return a if dtype is None else a.to(_torch_dtype(dtype))


def _array(a, dtype=None, copy=True, **kwargs):
    out = _asarray(a, dtype)
    return out.clone() if (copy and out is a) else out


_TORCH = {
    "sum": _reduce("sum"), "mean": _reduce("mean"), "min": _reduce("min"), "max": _reduce("max"),
    "amin": _reduce("min"), "amax": _reduce("max"), "prod": _reduce("prod"),
    "minimum": _binary("minimum"), "maximum": _binary("maximum"), "hypot": _binary("hypot"),
    "arctan2": _binary("atan2"), "power": _binary("pow"),
    "clip": _clip, "stack": _join("stack"), "concatenate": _join("cat"), "where": _where,
    "asarray": _asarray, "array": _array,
}


def _renamed(name):
    return lambda a, **kwargs: getattr(_t(), name)(a)


for _np_name, _th_name in (("arcsin", "asin"), ("arccos", "acos"), ("arctan", "atan")):
    _TORCH[_np_name] = _renamed(_th_name)


class ArrayNamespace:
    """``xp``: NumPy for host arrays, torch for device tensors (see the module docstring)."""

    def __getattr__(self, name):
        np_attr = getattr(np, name)
        if not callable(np_attr) or isinstance(np_attr, type):
            return np_attr

        def dispatch(*args, **kwargs):
            like = _find_tensor(args, kwargs)
            if like is None:
                return np_attr(*args, **kwargs)
            if name in _TORCH:
                return _TORCH[name](*args, **kwargs)
            fn = getattr(_t(), name, None)
            if fn is None:
                raise NotImplementedError(f"xp.{name} on device tensors")
            args = [_as_tensor(a, like) if isinstance(a, np.ndarray) else a for a in args]
            return fn(*args, **_kw(kwargs))
        dispatch.__name__ = name
        return dispatch

    def __repr__(self):
        return "<xp: numpy for host arrays, torch for device tensors>"


xp = ArrayNamespace()
