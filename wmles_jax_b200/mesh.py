"""Structured multiblock mesh: blocks, interfaces, ghost nodes and metrics (host NumPy).

API of the reference (wmles/mesh.py): ``Block(name, nodes, ng=3)``, ``Block.set_bc``,
``Mesh(blocks)``, ``Mesh.connect(A, faceA, B, faceB, shift)``, ``Mesh.finalize()``, and a
``Geom(vol, xc, S, xf)`` per block.  Set-up runs once, on the host or, with
``finalize(device=True)``, with the metrics computed on the GPU (same bits); its result
feeds the device metric arrays built by ``wmles_jax_b200.lowering``.

Every block-to-block copy (ghost nodes here, ghost cells in the ghost-gather program)
is expressed as an *index map*: the flat source indices that land in each destination
ghost position.  ``interface_index_map`` derives it by pushing an array of flat indices
through the same layer selection, m-ordering, axis permutation and tangential flips that
the reference's ``exchange`` (wmles/mesh.py:125-155) applies to data.

The metric formulas (face area = half cross product of the face diagonals, face centre
= mean of its four nodes, volume by the divergence theorem, cell centre = mean of the
eight nodes) follow wmles/mesh.py:53-73 operation by operation so that the host
metrics are bit-identical to the reference's.
"""
from itertools import product
from typing import NamedTuple

import numpy as np

FACE_NAMES = {"imin": (0, 0), "imax": (0, 1),
              "jmin": (1, 0), "jmax": (1, 1),
              "kmin": (2, 0), "kmax": (2, 1)}


def sl(nd, d, s, other=slice(None)):
    """Index tuple for an nd-array whose last 3 axes are spatial: ``s`` on spatial axis d,
    ``other`` on the remaining spatial axes (wmles/mesh.py:29-35)."""
    lead = nd - 3
    t = [slice(None)] * lead + [other] * 3
    t[lead + d] = s
    return tuple(t)


class Geom(NamedTuple):
    """Static geometry of one block, wmles/mesh.py:38-43.

    vol (Ni,Nj,Nk); xc (3,Ni,Nj,Nk); S[d] (3, .., N_d+1, ..) face area vectors along +d;
    xf[d] face centres with the shape of S[d]."""
    vol: np.ndarray
    xc: np.ndarray
    S: tuple
    xf: tuple


def _cross(a, b):
    return np.stack([a[1] * b[2] - a[2] * b[1],
                     a[2] * b[0] - a[0] * b[2],
                     a[0] * b[1] - a[1] * b[0]])


def _dot3(a, b):
    p = a * b
    return p[0] + p[1] + p[2]


def compute_geometry(X):
    """Metrics from an extended node array X (3, Ni+1, Nj+1, Nk+1); wmles/mesh.py:53-73."""
    Ni, Nj, Nk = (n - 1 for n in X.shape[1:])

    def corner(d, a, b):
        # node (a, b) of the faces normal to d; tangents in cyclic order (d+1, d+2)
        t1, t2 = (d + 1) % 3, (d + 2) % 3
        idx = [slice(None)] * 4
        ext = (Ni, Nj, Nk)
        idx[1 + t1] = slice(a, ext[t1] + a)
        idx[1 + t2] = slice(b, ext[t2] + b)
        return X[tuple(idx)]

    S, xf = [], []
    for d in range(3):
        c00, c10, c01, c11 = corner(d, 0, 0), corner(d, 1, 0), corner(d, 0, 1), corner(d, 1, 1)
        S.append(0.5 * _cross(c11 - c00, c01 - c10))
        xf.append(0.25 * (c00 + c10 + c01 + c11))

    def hi(a, d):
        return a[sl(4, d, slice(1, None))]

    def lo(a, d):
        return a[sl(4, d, slice(None, -1))]

    vol = (_dot3(hi(xf[0], 0), hi(S[0], 0)) - _dot3(lo(xf[0], 0), lo(S[0], 0))
           + _dot3(hi(xf[1], 1), hi(S[1], 1)) - _dot3(lo(xf[1], 1), lo(S[1], 1))
           + _dot3(hi(xf[2], 2), hi(S[2], 2)) - _dot3(lo(xf[2], 2), lo(S[2], 2))) / 3.0
    xc = 0
    for a, b, c in product((0, 1), repeat=3):
        xc = xc + X[:, a:Ni + a, b:Nj + b, c:Nk + c]
    xc = xc / 8.0
    return vol, xc, tuple(S), tuple(xf)


class Interface:
    """Block-to-block connection seen from the destination block (wmles/mesh.py:77-85)."""

    def __init__(self, nb, src_face, mapping, flip, shift):
        self.nb = nb                  # block the ghost values are copied from
        self.src_face = src_face      # its connected face, (axis, side)
        self.mapping = mapping        # axis of that block for each axis of this one
        self.flip = flip              # per axis of this block: index runs reversed (tangential axes)
        self.shift = np.asarray(shift, float)

    def __repr__(self):
        return (f"Interface(nb={self.nb}, src_face={self.src_face}, mapping={self.mapping}, "
                f"flip={self.flip})")


class Block:
    def __init__(self, name, nodes, ng=3):
        nodes = np.asarray(nodes, float)
        if nodes.ndim != 4 or nodes.shape[0] != 3:
            raise ValueError("nodes must be (3, ni+1, nj+1, nk+1)")
        self.name, self.ng, self.x_int = name, ng, nodes
        self.n = tuple(s - 1 for s in nodes.shape[1:])
        if min(self.n) < ng:
            raise ValueError("each block needs at least ng cells per direction")
        self.N = tuple(n + 2 * ng for n in self.n)
        self.faces = {}
        self.X = None
        self.geom = None
        self.metrics_dev = None

    def set_bc(self, face, bc):
        self.faces[FACE_NAMES[face]] = bc

    # slicing helpers for any array with 3 trailing spatial axes (NumPy or torch)
    def interior(self, a):
        lead, ng = a.ndim - 3, self.ng
        return a[(slice(None),) * lead + tuple(slice(ng, ng + n) for n in self.n)]

    def take(self, a, axis, idx):
        lead, ng = a.ndim - 3, self.ng
        t = [slice(None)] * lead + [slice(ng, ng + n) for n in self.n]
        t[lead + axis] = idx
        return a[tuple(t)]

    def slab(self, a, d, lo, hi):
        lead, ng = a.ndim - 3, self.ng
        t = [slice(None)] * lead + [slice(ng, ng + n) for n in self.n]
        t[lead + d] = slice(ng + lo, ng + self.n[d] + hi)
        return a[tuple(t)]


def interface_index_map(shape_dst, shape_src, ng, n_dst_axis, n_src_axis, face_dst, itf, kind):
    """Flat-index map of one ghost exchange (wmles/mesh.py:125-155).

    Returns ``(dst_flat, src_flat)``, two int64 arrays of equal length: after the
    exchange, ``dst.flat[dst_flat] == src.flat[src_flat]`` (plus ``itf.shift`` for node
    data).  ``shape_*`` are the 3 spatial extents; ``kind`` is "cell" or "node"."""
    aA, sA = face_dst
    aB, sB = itf.src_face
    if kind == "cell":
        lo_src = ng if sB == 0 else n_src_axis
        lo_dst = ng + n_dst_axis if sA == 1 else 0
    else:
        lo_src = ng + 1 if sB == 0 else n_src_axis
        lo_dst = ng + n_dst_axis + 1 if sA == 1 else 0
    src_ids = np.arange(int(np.prod(shape_src)), dtype=np.int64).reshape(shape_src)
    layers = src_ids[sl(3, aB, slice(lo_src, lo_src + ng))]
    if sB == 1:
        layers = layers[sl(3, aB, slice(None, None, -1))]          # nearest layer first
    layers = np.transpose(layers, [itf.mapping[m] for m in range(3)])
    for t in range(3):
        if itf.flip[t]:
            layers = layers[sl(3, t, slice(None, None, -1))]
    if sA == 0:
        layers = layers[sl(3, aA, slice(None, None, -1))]          # back to array order
    dst_ids = np.arange(int(np.prod(shape_dst)), dtype=np.int64).reshape(shape_dst)
    target = dst_ids[sl(3, aA, slice(lo_dst, lo_dst + ng))]
    if target.shape != layers.shape:
        raise ValueError(f"interface extents do not conform: {target.shape} vs {layers.shape}")
    return target.ravel(), layers.ravel()


def _reflect_nodes(X, blk, axis, side):
    """Ghost nodes mirrored through the boundary node plane (wmles/mesh.py:158-166)."""
    ng, n = blk.ng, blk.n[axis]
    if side == 0:
        inner = X[sl(4, axis, slice(ng + 1, ng + 1 + ng))][sl(4, axis, slice(None, None, -1))]
        X[sl(4, axis, slice(0, ng))] = 2 * X[sl(4, axis, slice(ng, ng + 1))] - inner
    else:
        b = ng + n
        inner = X[sl(4, axis, slice(n, n + ng))][sl(4, axis, slice(None, None, -1))]
        X[sl(4, axis, slice(b + 1, b + 1 + ng))] = 2 * X[sl(4, axis, slice(b, b + 1))] - inner


def _node_plane(blk, axis, side):
    return np.take(blk.x_int, 0 if side == 0 else blk.n[axis], axis=1 + axis)


def _match_orientation(A, fa, B, fb, shift):
    """Axis mapping and tangential flips that carry B's interface node plane (+shift)
    onto A's; candidates are tried in the order of wmles/mesh.py:169-193."""
    aA, _ = fa
    aB, _ = fb
    pa = _node_plane(A, *fa)
    pb = _node_plane(B, *fb) + np.asarray(shift, float).reshape(3, 1, 1)
    tA = [m for m in range(3) if m != aA]
    tB = [m for m in range(3) if m != aB]
    tol = 1e-9 * max(np.abs(pa).max(), 1e-30)
    for order in ((0, 1), (1, 0)):
        perm = [tB[order[0]], tB[order[1]]]
        cand0 = np.transpose(pb, [0, 1 + order[0], 1 + order[1]])
        for f1, f2 in product((0, 1), repeat=2):
            cand = cand0[:, ::-1] if f1 else cand0
            cand = cand[:, :, ::-1] if f2 else cand
            if cand.shape == pa.shape and np.allclose(cand, pa, atol=tol, rtol=0):
                mapping, flip = [0] * 3, [False] * 3
                mapping[aA], mapping[tA[0]], mapping[tA[1]] = aB, perm[0], perm[1]
                flip[tA[0]], flip[tA[1]] = bool(f1), bool(f2)
                return tuple(mapping), tuple(flip)
    raise ValueError(f"interface {A.name}{fa} <-> {B.name}{fb}: no axis permutation or flip maps one "
                     f"face's nodes onto the other's (is the periodic shift right?)")


class Mesh:
    def __init__(self, blocks):
        self.blocks = list(blocks)
        if len({b.ng for b in self.blocks}) != 1:
            raise ValueError("all blocks must share ng")
        self.ng = self.blocks[0].ng
        self.geoms = None

    def index(self, blk):
        return next(i for i, b in enumerate(self.blocks) if b is blk)

    def connect(self, A, faceA, B, faceB, shift=(0.0, 0.0, 0.0)):
        """Join A.faceA to B.faceB; ``shift`` = x_A(plane) - x_B(plane) (periodic offset)."""
        fa, fb = FACE_NAMES[faceA], FACE_NAMES[faceB]
        shift = np.asarray(shift, float)
        for X, fx, Y, fy, sh in ((A, fa, B, fb, shift), (B, fb, A, fa, -shift)):
            mapping, flip = _match_orientation(X, fx, Y, fy, sh)
            X.faces[fx] = Interface(self.index(Y), fy, mapping, flip, sh)

    def finalize(self, node_passes=3, device=False):
        """Ghost nodes (node_passes sweeps of exchange / reflection) and metrics;
        wmles/mesh.py:213-242.

        device=True computes the metrics on the GPU (``device_geometry.block_geometry``):
        the ``Geom`` arrays are the same bits, and each block keeps its packed metric table
        on the device (``Block.metrics_dev``, 216 B per cell including ghosts) for the
        solvers built on this mesh; ``release_device_metrics`` frees it."""
        ng = self.ng
        for b in self.blocks:
            for f in FACE_NAMES.values():
                if f not in b.faces:
                    raise KeyError(f"block {b.name}: face {f} is neither connected nor given a boundary condition")
            X = np.zeros((3,) + tuple(n + 1 + 2 * ng for n in b.n))
            X[(slice(None),) + tuple(slice(ng, ng + n + 1) for n in b.n)] = b.x_int
            b.X = X
        maps = {}      # the index maps are the same on every pass
        for _ in range(node_passes):
            for a in range(3):
                for ib, b in enumerate(self.blocks):
                    for s in (0, 1):
                        f = b.faces[(a, s)]
                        if isinstance(f, Interface):
                            src = self.blocks[f.nb]
                            key = (ib, a, s)
                            if key not in maps:
                                maps[key] = interface_index_map(
                                    b.X.shape[1:], src.X.shape[1:], ng, b.n[a], src.n[f.src_face[0]],
                                    (a, s), f, "node")
                            dst_flat, src_flat = maps[key]
                            vals = src.X.reshape(3, -1)[:, src_flat] + f.shift.reshape(3, 1)
                            b.X.reshape(3, -1)[:, dst_flat] = vals
                        else:
                            _reflect_nodes(b.X, b, a, s)
        geoms = []
        for b in self.blocks:
            if device:
                from .device_geometry import block_geometry
                (vol, xc, S, xf), b.metrics_dev = block_geometry(b.X)
            else:
                vol, xc, S, xf = compute_geometry(b.X)
                b.metrics_dev = None
            if vol.min() <= 0:
                raise ValueError(f"block {b.name}: a cell volume is zero or negative (the node ordering is "
                                 f"left-handed, or the grid folds over itself)")
            b.geom = Geom(vol, xc, S, xf)
            geoms.append(b.geom)
        self.geoms = tuple(geoms)
        return self

    def release_device_metrics(self):
        """Free the packed metric tables kept on the device by finalize(device=True)
        (solvers already built keep their own copies)."""
        for b in self.blocks:
            b.metrics_dev = None
