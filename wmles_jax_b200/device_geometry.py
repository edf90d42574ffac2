"""Block geometry on the device for ``Mesh.finalize(device=True)`` (wm_block_geometry).

The metrics of wmles/mesh.py:53-73 and the packed table the stage kernels read are
computed on the GPU from the node array extended by the ghost nodes, with the host path's
arithmetic: the ``Geom`` arrays returned to the host are bit-identical to
``mesh.compute_geometry``'s, the packed table to ``lowering.block_metrics``' except the
filter width V^(1/3) (device pow, a few ulp).  For a 192 x 96 x 96 channel block this
replaces about 2.2 s of host NumPy (geometry and packing) by a copy of the nodes up, three
memory-bound kernels and one copy of the geometry down, and the case built from it copies
the packed table on the device instead of uploading it.
"""
import ctypes as C

import numpy as np
import torch

from . import _native as N
from .backend import require_gpu

NMET = 27


def block_geometry(X):
    """``(vol, xc, S, xf)`` on the host and the packed metric table (device tensor of
    NMET x N0 x N1 x N2 float64) of one block from its extended node array X
    (3, N0+1, N1+1, N2+1).  Runs on a private stream and waits for it, so it can run
    beside other device work (e.g. a server's steps on other streams)."""
    X = np.asarray(X)
    Nc = tuple(int(s) - 1 for s in X.shape[1:])
    if X.ndim != 4 or X.shape[0] != 3 or min(Nc) < 1:
        raise ValueError(f"node array of shape {X.shape}: expected (3, N0+1, N1+1, N2+1)")
    dev = require_gpu()
    lib = N.load()
    n = int(np.prod(Nc))
    fext = [tuple(Nc[a] + (a == d) for a in range(3)) for d in range(3)]
    sizes = [n, 3 * n] + [3 * int(np.prod(e)) for e in fext] * 2
    offs = np.cumsum([0] + sizes)
    stream = torch.cuda.Stream(device=dev)
    with torch.cuda.stream(stream):
        Xd = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float64)).to(dev)
        buf = torch.empty(int(offs[-1]), dtype=torch.float64, device=dev)
        met = torch.empty((NMET,) + Nc, dtype=torch.float64, device=dev)
        p = [buf.data_ptr() + 8 * int(o) for o in offs[:-1]]
        dp = lambda a: C.cast(C.c_void_p(int(a)), N.c_double_p)   # noqa: E731
        N.check(lib.wm_block_geometry(dp(Xd.data_ptr()), (C.c_int * 3)(*Nc), dp(p[0]), dp(p[1]),
                                      N.ptr_array(p[2:5]), N.ptr_array(p[5:8]), dp(met.data_ptr()),
                                      C.c_void_p(stream.cuda_stream)), "wm_block_geometry")
        host = buf.cpu().numpy()
    stream.synchronize()
    part = [host[offs[i]:offs[i + 1]] for i in range(len(sizes))]
    vol = part[0].reshape(Nc)
    xc = part[1].reshape((3,) + Nc)
    S = tuple(part[2 + d].reshape((3,) + fext[d]) for d in range(3))
    xf = tuple(part[5 + d].reshape((3,) + fext[d]) for d in range(3))
    return (vol, xc, S, xf), met
