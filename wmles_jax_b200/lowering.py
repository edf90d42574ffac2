"""Lowering of a mesh + solver options into the flat case descriptor of libwmles_cuda.so.

* Metrics: per block a (WM_NMET, Ni, Nj, Nk) float64 array holding, for every cell, the
  area vector of its LOWER face in each direction (the reference's S[d][:, c]), the volume,
  the centre and the SGS filter width V^(1/3) (computed with NumPy's ``**`` exactly as
  wmles/solver.py:81 does).
* Wall faces: |S|, the outward unit normal and the wall distance of the sample cell,
  evaluated with the reference's NumPy expressions (wmles/bc.py:146-155) so that the device
  wall model starts from bit-identical geometry.
* Ghost program: the reference fills ghost cells in a fixed order (wmles/solver.py:59-73:
  ``bc_passes`` x axis x block x side; block-to-block exchange copies the full tangential
  extent, so edge and corner ghosts propagate between passes).  ``trace_ghost_fill`` runs
  that order on *expression ids* instead of values: an exchange copies ids, a mirror BC
  creates an op node (slip / no-slip / far field) whose child is the id of the source cell,
  Dirichlet creates a constant leaf, the synthetic inflow creates inflow leaves.  After the
  passes every ghost cell is a chain of ops ending in one leaf, which is what the device
  gather kernel replays.
"""
from dataclasses import dataclass

import numpy as np

from .bc import SlipWall, NoSlipWall, Dirichlet, CharacteristicFarfield, Extrapolate, WallModel
from .mesh import Interface, interface_index_map, sl
from .smooth_ramp import SmoothRampInflow

NMET = 27
OP_SLIP, OP_NOSLIP, OP_FARFIELD = 1, 2, 3
SRC_CELL, SRC_INFLOW, SRC_CONST = 0, 1, 2
_K_INFLOW, _K_CONST, _K_OP = 1, 2, 3


_SHARED = {}   # id(geom) -> [geom, packed metrics or None], for geometries many cases reuse


def share_metrics(mesh):
    """Keep the packed metric arrays of `mesh` after their first use (for a mesh shared by
    many cases, e.g. a serving grid cache); the registry holds the mesh's geometries."""
    for g in mesh.geoms:
        _SHARED.setdefault(id(g), [g, None])


def block_metrics(blk, geom):
    """(NMET, Ni, Nj, Nk) float64 metric array of one block: the device table kept by
    Mesh.finalize(device=True) when the block has one for this geometry, else a host array."""
    dev = getattr(blk, "metrics_dev", None)
    if dev is not None and blk.geom is geom:
        return dev
    ent = _SHARED.get(id(geom))
    if ent is not None and ent[0] is geom:
        if ent[1] is None:
            ent[1] = _block_metrics(blk, geom)
        return ent[1]
    return _block_metrics(blk, geom)


def _block_metrics(blk, geom):
    Ni, Nj, Nk = blk.N
    M = np.empty((NMET, Ni, Nj, Nk))
    M[0:3] = geom.S[0][:, :Ni]
    M[3:6] = geom.S[1][:, :, :Nj]
    M[6:9] = geom.S[2][:, :, :, :Nk]
    M[9] = geom.vol
    M[10:13] = geom.xc
    M[13] = geom.vol ** (1.0 / 3.0)
    M[14] = 1.0 / geom.vol
    # viscous correction geometry of each cell's lower face: e = dx / |dx|, 1 / |dx| with
    # dx = xc[c] - xc[c - 1] along d (wmles/viscous.py:35-37); zero on the first layer
    for d in range(3):
        base = 15 + 4 * d
        M[base:base + 4] = 0.0
        dx = geom.xc[sl(4, d, slice(1, None))] - geom.xc[sl(4, d, slice(None, -1))]
        dist = np.sqrt(np.sum(dx * dx, axis=0))
        M[(slice(base, base + 3),) + sl(3, d, slice(1, None))] = dx / dist
        M[(base + 3,) + sl(3, d, slice(1, None))] = 1.0 / dist
    return M


def wall_geometry(blk, geom, axis, side, n_match):
    """(5, nt1, nt2): |S|, n_out (3), h of a wall-modelled face; wmles/bc.py:146-155."""
    ng, n = blk.ng, blk.n[axis]
    fb = ng if side == 0 else ng + n
    mi = ng + n_match - 1 if side == 0 else ng + n - n_match
    S = blk.take(geom.S[axis], axis, fb)
    Sm = np.sqrt(np.sum(S * S, axis=0))
    n_out = S / Sm if side == 1 else -S / Sm
    xf = blk.take(geom.xf[axis], axis, fb)
    xcm = blk.take(geom.xc, axis, mi)
    h = np.sum((xcm - xf) * (-n_out), axis=0)
    return np.ascontiguousarray(np.concatenate([Sm[None], n_out, h[None]], axis=0))


@dataclass
class GhostProgram:
    dst: np.ndarray       # (count, 2) int32: block, flat cell
    src: np.ndarray       # (count, 2) int32: kind << 24 | block (bc id for CONST), flat cell
    ops: np.ndarray       # (count, 2) int32: first op, op count
    op_code: np.ndarray   # (nops,) int32
    op_nrm: np.ndarray    # (nops, 3) float64

    @property
    def count(self):
        return len(self.dst)


class _Nodes:
    """Growable node table of the ghost-fill trace."""

    def __init__(self):
        self.kind, self.a, self.code, self.nrm = [], [], [], []
        self.n = 0

    def add(self, kind, a, code, nrm):
        m = len(a)
        ids = np.arange(self.n, self.n + m, dtype=np.int64)
        self.kind.append(np.full(m, kind, np.int8))
        self.a.append(np.asarray(a, np.int64))
        self.code.append(np.full(m, code, np.int64) if np.isscalar(code) else np.asarray(code, np.int64))
        self.nrm.append(np.zeros((m, 3)) if nrm is None else np.asarray(nrm, float).reshape(m, 3))
        self.n += m
        return ids

    def freeze(self):
        cat = lambda L, dt, shape: np.concatenate(L) if L else np.zeros(shape, dt)
        return (cat(self.kind, np.int8, 0), cat(self.a, np.int64, 0), cat(self.code, np.int64, 0),
                cat(self.nrm, float, (0, 3)))


class BCTable:
    """Per-BC constants referenced by op codes and constant leaves (8 doubles each)."""

    def __init__(self, gas):
        self.gas, self.rows, self._ids = gas, [], {}

    def id_of(self, bc):
        key = id(bc)
        if key in self._ids:
            return self._ids[key]
        row = np.zeros(8)
        if isinstance(bc, Dirichlet):
            prim = np.asarray(bc.prim, float).reshape(5, 1)
            row[:5] = self.gas.prim_to_cons(prim * np.ones((1, 1)))[:, 0]
        elif isinstance(bc, CharacteristicFarfield):
            row[:5] = bc.prim
        elif isinstance(bc, NoSlipWall):
            row[5] = 0.0 if bc.T_wall is None else float(bc.T_wall)
            row[6] = 0.0 if bc.T_wall is None else 1.0
        self.rows.append(row)
        self._ids[key] = len(self.rows) - 1
        if len(self.rows) > 255:
            raise NotImplementedError("more than 255 distinct boundary conditions")
        return self._ids[key]

    def array(self):
        return np.array(self.rows) if self.rows else np.zeros((1, 8))


def trace_ghost_fill(blocks, geoms, bc_passes, bctab):
    """Symbolic run of Solver.apply_bcs (wmles/solver.py:59-73) on expression ids.

    Returns (E, nodes, offsets): E[b] is an int64 array with the blocks' ghosted shape;
    a value < 0 encodes "the value cell g had before the fill" with g = -1 - value (a global
    cell id, block offsets in ``offsets``); a value >= 0 is a node of ``nodes``."""
    offsets = np.cumsum([0] + [int(np.prod(b.N)) for b in blocks])
    E = [-1 - (offsets[ib] + np.arange(int(np.prod(b.N)), dtype=np.int64)).reshape(b.N)
         for ib, b in enumerate(blocks)]
    nodes = _Nodes()
    maps = {}
    for _ in range(bc_passes):
        for a in range(3):
            for ib, blk in enumerate(blocks):
                for s in (0, 1):
                    f = blk.faces[(a, s)]
                    if isinstance(f, Interface):
                        key = (ib, a, s)
                        if key not in maps:
                            nb = blocks[f.nb]
                            maps[key] = interface_index_map(blk.N, nb.N, blk.ng, blk.n[a], nb.n[f.src_face[0]],
                                                            (a, s), f, "cell")
                        dflat, sflat = maps[key]
                        src_ids = E[f.nb].ravel()[sflat]          # read before the write (self-links)
                        E[ib].ravel()[dflat] = src_ids
                    else:
                        _trace_fill(f, E, ib, blk, geoms[ib], a, s, nodes, bctab, offsets)
    return E, nodes.freeze(), offsets


def _trace_fill(bc, E, ib, blk, geom, axis, side, nodes, bctab, offsets):
    ng, n = blk.ng, blk.n[axis]
    Eb = E[ib]
    if isinstance(bc, SmoothRampInflow):
        if axis != 0 or side != 0:
            raise ValueError("SmoothRampInflow is only valid on the i-min face")
        for m in range(ng):
            gi = ng - 1 - m
            cells = np.arange(int(np.prod(blk.N)), dtype=np.int64).reshape(blk.N)[gi]
            Eb[gi] = nodes.add(_K_INFLOW, offsets[ib] + cells.ravel(), 0, None).reshape(cells.shape)
        return
    fb = ng if side == 0 else ng + n
    S = geom.S[axis][sl(4, axis, slice(fb, fb + 1))]
    nrm = S / np.sqrt(np.sum(S * S, axis=0))                     # wmles/bc.py:18-19
    nrm_cells = np.moveaxis(nrm, 0, -1)                           # (.., 3) over the layer
    for m in range(ng):
        gi = ng - 1 - m if side == 0 else ng + n + m
        ii = ng + m if side == 0 else ng + n - 1 - m
        dst = sl(3, axis, slice(gi, gi + 1))
        if isinstance(bc, Extrapolate):
            edge = ng if side == 0 else ng + n - 1
            Eb[dst] = Eb[sl(3, axis, slice(edge, edge + 1))]
            continue
        child = Eb[sl(3, axis, slice(ii, ii + 1))]
        shape = child.shape
        if isinstance(bc, (SlipWall, WallModel)):
            ids = nodes.add(_K_OP, child.ravel(), OP_SLIP, nrm_cells.reshape(-1, 3))
        elif isinstance(bc, NoSlipWall):
            ids = nodes.add(_K_OP, child.ravel(), OP_NOSLIP | (bctab.id_of(bc) << 8), None)
        elif isinstance(bc, CharacteristicFarfield):
            ids = nodes.add(_K_OP, child.ravel(), OP_FARFIELD | (bctab.id_of(bc) << 8) | (side << 16),
                            nrm_cells.reshape(-1, 3))
        elif isinstance(bc, Dirichlet):
            ids = nodes.add(_K_CONST, np.full(child.size, bctab.id_of(bc)), 0, None)
        else:
            raise NotImplementedError(f"cuda backend: unsupported boundary condition {type(bc).__name__}")
        Eb[dst] = ids.reshape(shape)


def _depths(blk):
    """Per-axis ghost depth (0 = interior) of every cell of the block."""
    out = []
    for a in range(3):
        x = np.arange(blk.N[a])
        d = np.where(x < blk.ng, blk.ng - x, np.where(x >= blk.ng + blk.n[a], x - blk.ng - blk.n[a] + 1, 0))
        shape = [1, 1, 1]
        shape[a] = blk.N[a]
        out.append(d.reshape(shape))
    return np.broadcast_arrays(*out)


def rhs_ghost_mask(blk):
    """Ghost cells the fused stage kernel reads: face ghosts of depth 1-2 and edge ghosts
    of depth (1, 1), the third index interior."""
    di, dj, dk = _depths(blk)
    nz = (di > 0).astype(int) + (dj > 0) + (dk > 0)
    face = (nz == 1) & (np.maximum(np.maximum(di, dj), dk) <= 2)
    edge = (nz == 2) & (np.maximum(np.maximum(di, dj), dk) == 1)
    return face | edge


def all_ghost_mask(blk):
    """Every ghost cell of the block."""
    m = np.ones(blk.N, bool)
    m[tuple(slice(blk.ng, blk.ng + n) for n in blk.n)] = False
    return m


def build_program(blocks, E, nodes, offsets, select, allow_stale):
    """Resolve the traced ids of the selected ghost cells into a GhostProgram."""
    kind, a, code, nrm = nodes
    dst_b, dst_c, vals = [], [], []
    for ib, blk in enumerate(blocks):
        mask = select(ib, blk)
        flat = np.flatnonzero(mask.ravel())
        ev = E[ib].ravel()[flat]
        if allow_stale:
            keep = ev != (-1 - (offsets[ib] + flat))                # untouched cells need no entry
            flat, ev = flat[keep], ev[keep]
        dst_b.append(np.full(len(flat), ib, np.int64))
        dst_c.append(flat)
        vals.append(ev)
    dst_b, dst_c, cur = np.concatenate(dst_b), np.concatenate(dst_c), np.concatenate(vals)
    count = len(cur)
    chain = []                                                    # op node ids, outermost first
    while True:
        is_op = cur >= 0
        is_op[is_op] = kind[cur[is_op]] == _K_OP
        if not is_op.any():
            break
        col = np.full(count, -1, np.int64)
        col[is_op] = cur[is_op]
        chain.append(col)
        cur = np.where(is_op, a[np.where(is_op, cur, 0)], cur)
    # leaves
    src = np.zeros((count, 2), np.int64)
    leaf_cell = cur < 0
    g = -1 - cur[leaf_cell]
    gb = np.searchsorted(offsets, g, side="right") - 1
    gc = g - offsets[gb]
    if not allow_stale:
        interior = np.ones(len(g), bool)
        for ib, blk in enumerate(blocks):
            sel = gb == ib
            idx = np.unravel_index(gc[sel], blk.N)
            ok = np.ones(sel.sum(), bool)
            for ax in range(3):
                ok &= (idx[ax] >= blk.ng) & (idx[ax] < blk.ng + blk.n[ax])
            interior[sel] = ok
        if not interior.all():
            raise NotImplementedError("cuda backend: a ghost cell read by the RHS depends on an unfilled "
                                      "ghost value (unsupported topology)")
    src[leaf_cell, 0] = (SRC_CELL << 24) | gb
    src[leaf_cell, 1] = gc
    nl = ~leaf_cell
    lk = kind[cur[nl]]
    la = a[cur[nl]]
    infl = lk == _K_INFLOW
    gbi = np.searchsorted(offsets, la[infl], side="right") - 1
    src_nl = np.zeros((nl.sum(), 2), np.int64)
    src_nl[infl, 0] = (SRC_INFLOW << 24) | gbi
    src_nl[infl, 1] = la[infl] - offsets[gbi]
    cst = lk == _K_CONST
    src_nl[cst, 0] = (SRC_CONST << 24) | la[cst]
    src_nl[cst, 1] = 0
    src[nl] = src_nl
    # ops in application order (innermost first)
    depth = np.zeros(count, np.int64)
    for col in chain:
        depth += col >= 0
    starts = np.concatenate([[0], np.cumsum(depth)[:-1]]) if count else np.zeros(0, np.int64)
    nops = int(depth.sum())
    op_code = np.zeros(nops, np.int64)
    op_nrm = np.zeros((nops, 3))
    for level, col in enumerate(chain):
        has = col >= 0
        pos = starts[has] + (depth[has] - 1 - level)
        op_code[pos] = code[col[has]]
        op_nrm[pos] = nrm[col[has]]
    i32 = lambda x: np.ascontiguousarray(x, np.int32)
    return GhostProgram(dst=i32(np.stack([dst_b, dst_c], 1)), src=i32(src),
                        ops=i32(np.stack([starts, depth], 1)), op_code=i32(op_code),
                        op_nrm=np.ascontiguousarray(op_nrm))


def lower_ghost_programs(blocks, geoms, gas, bc_passes):
    """(program for the RHS, program for apply_bcs, BC table) of a finalized mesh."""
    bctab = BCTable(gas)
    E, nodes, offsets = trace_ghost_fill(blocks, geoms, bc_passes, bctab)
    prog_rhs = build_program(blocks, E, nodes, offsets, lambda ib, b: rhs_ghost_mask(b), False)
    prog_all = build_program(blocks, E, nodes, offsets, lambda ib, b: all_ghost_mask(b), True)
    return prog_rhs, prog_all, bctab.array()
