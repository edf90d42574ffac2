"""Multiblock explicit finite-volume solver on the B200 (WMLES_BACKEND=cuda).

Same constructor and methods as the reference ``Solver`` (wmles/solver.py:39-232):
``init_state``, ``apply_bcs``, ``rhs``, ``max_dt``, ``advance``, ``wall_stats``,
``wall_loads``, plus ``step`` (max_dt + advance in one call, the drivers' loop body).
The state is a tuple of torch CUDA float64 tensors (5, Ni, Nj, Nk), ghosts included, and
every call returns new tensors as the reference's functional API does.  ``solver.geoms``
holds the block geometry on the device (torch tensors), as the reference's does (JAX device
arrays placed by Mesh.finalize), so driver arithmetic such as ``q[1:4] ** 2 / q[0] * g.vol``
runs on the device; ``solver.host_geoms`` (= ``mesh.geoms``) is the host NumPy copy the
set-up uses.

Built-in BCs, schemes, SGS models, ``ConstantMassFlux`` and ``SmoothRampSponge`` are
recognised by class and lowered into one ``wm_case`` of libwmles_cuda.so; anything else
raises NotImplementedError (there is no CPU fallback).
"""
import ctypes as C
import weakref

import numpy as np
import torch

from . import _native as N
from .backend import require_gpu
from .bc import WallModel
from .constraints import ConstantMassFlux
from .lowering import block_metrics, lower_ghost_programs, wall_geometry
from .schemes import KEP, MUSCLHLLC, Hybrid
from .sgs import make_sgs, SGS_IDS
from .smooth_ramp import SmoothRampInflow, SmoothRampSponge

PRECISIONS = {"fp64": 0, "mixed": 1}
SCHEME_KEP, SCHEME_MUSCL, SCHEME_HYBRID = 0, 1, 2


def _scheme_fields(scheme):
    if isinstance(scheme, KEP):
        return SCHEME_KEP, scheme.order, 0, 0.6, 0.9
    if isinstance(scheme, MUSCLHLLC):
        return SCHEME_MUSCL, 4, MUSCLHLLC.LIMITERS.index(scheme.limiter), 0.6, 0.9
    if isinstance(scheme, Hybrid):
        return SCHEME_HYBRID, scheme.c.order, MUSCLHLLC.LIMITERS.index(scheme.u.limiter), scheme.th0, scheme.th1
    raise NotImplementedError(f"cuda backend: unsupported scheme {type(scheme).__name__}")


class Solver:
    def __init__(self, mesh, gas, scheme, sgs="vreman", cfl=0.8, sgs_kwargs=None, constraints=(),
                 sources=(), bc_passes=2, *, precision="fp64", tile=None, chunk=None):
        if tile == "auto":           # measured once per workload and machine, then cached
            from .autotune import tune
            kw = dict(scheme=scheme, sgs=sgs, cfl=cfl, sgs_kwargs=sgs_kwargs, constraints=constraints,
                      sources=sources, bc_passes=bc_passes)
            tile, _ = tune([(mesh, gas, kw, None)], precision=precision)
        self._prepare(mesh, gas, scheme, sgs, cfl, sgs_kwargs, constraints, sources, bc_passes,
                      precision=precision, tile=tile, chunk=chunk)
        self._create()

    def _prepare(self, mesh, gas, scheme, sgs="vreman", cfl=0.8, sgs_kwargs=None, constraints=(),
                 sources=(), bc_passes=2, *, precision="fp64", tile=None, chunk=None):
        """Host half of construction: validation and lowering into a case descriptor (no
        device call; a server runs it on a worker thread)."""
        self.device = require_gpu()
        self.mesh, self.blocks, self.gas = mesh, mesh.blocks, gas
        self.host_geoms = mesh.geoms
        if self.host_geoms is None:
            raise ValueError("call mesh.finalize() before building the solver")
        self.scheme, self.cfl = scheme, cfl
        self.sgs = make_sgs(sgs, **(sgs_kwargs or {}))
        self.constraints, self.sources, self.bc_passes = tuple(constraints), tuple(sources), bc_passes
        if precision not in PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
        self.precision = precision
        if len(self.blocks) > N.MAX_BLOCKS:
            raise NotImplementedError(f"cuda backend: more than {N.MAX_BLOCKS} blocks")
        self._lib = N.load()
        self._keep = []
        self._desc = self._lower(tile, chunk)

    def _create(self, release=True):
        """Device half of construction: wm_case_create uploads the descriptor's arrays (kept
        with release=False, e.g. to create the case again with another tile shape)."""
        handle = C.c_void_p()
        N.check(self._lib.wm_case_create(C.byref(self._desc), C.byref(handle)), "wm_case_create")
        self._case = handle
        if release:
            self._keep = self._desc = None         # host arrays were copied to the device

    @property
    def geoms(self):
        """Block geometry (Geom of vol, xc, S, xf) as float64 tensors on the solver's device,
        copied from the host geometry on first use."""
        dev = getattr(self, "_dev_geoms", None)
        if dev is None:
            from .mesh import Geom

            def t(a):
                return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(self.device)
            dev = self._dev_geoms = tuple(Geom(t(g.vol), t(g.xc), tuple(t(x) for x in g.S), tuple(t(x) for x in g.xf))
                                          for g in self.host_geoms)
        return dev

    def __del__(self):
        h = getattr(self, "_case", None)
        if h is not None and h.value:
            try:
                self._lib.wm_case_destroy(h)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self._case = None

    # ------------------------------------------------------------------ lowering
    def _arr(self, a, dtype):
        a = np.ascontiguousarray(a, dtype=dtype)
        self._keep.append(a)
        return a

    def _program(self, prog):
        p = N.WmGhostProgram()
        p.count = prog.count
        p.dst = N.as_int_p(self._arr(prog.dst, np.int32))
        p.src = N.as_int_p(self._arr(prog.src, np.int32))
        p.ops = N.as_int_p(self._arr(prog.ops, np.int32))
        p.nops = len(prog.op_code)
        p.op_code = N.as_int_p(self._arr(prog.op_code if len(prog.op_code) else np.zeros(1), np.int32))
        p.op_nrm = N.as_double_p(self._arr(prog.op_nrm if len(prog.op_nrm) else np.zeros((1, 3)), np.float64))
        return p

    def _lower(self, tile, chunk):
        g = self.gas
        d = N.WmCaseDesc()
        d.gas = N.WmGas(g.gamma, g.R, g.Pr, g.Pr_t, g.mu_ref, g.T_ref, g.S_suth)
        d.scheme, d.kep_order, d.limiter, d.th0, d.th1 = _scheme_fields(self.scheme)
        d.sgs, d.sgs_coeff = SGS_IDS[self.sgs.name], self.sgs.coeff
        d.cfl = float(self.cfl)
        d.precision = PRECISIONS[self.precision]
        # constraint
        d.cmf_dir = -1
        for c in self.constraints:
            if not isinstance(c, ConstantMassFlux) or d.cmf_dir >= 0:
                raise NotImplementedError("cuda backend: supports one ConstantMassFlux constraint")
            den = 0.0
            for b, geo in zip(self.blocks, self.host_geoms):
                den = den + np.sum(b.interior(geo.vol))        # wmles/solver.py:26-27
            d.cmf_dir, d.cmf_target, d.cmf_volume = int(c.dir), float(c.target), float(den)
        # blocks
        nb = len(self.blocks)
        blocks = (N.WmBlock * nb)()
        for ib, (b, geo) in enumerate(zip(self.blocks, self.host_geoms)):
            blocks[ib].n = (C.c_int * 3)(*b.n)
            blocks[ib].ng = b.ng
            met = block_metrics(b, geo)
            if isinstance(met, torch.Tensor):                 # device table (finalize(device=True))
                if met.device != self.device or met.dtype != torch.float64 or not met.is_contiguous():
                    raise ValueError(f"block {b.name}: device metric table on {met.device}, {met.dtype}")
                self._keep.append(met)
                blocks[ib].metrics = C.cast(C.c_void_p(met.data_ptr()), N.c_double_p)
            else:
                blocks[ib].metrics = N.as_double_p(self._arr(met, np.float64))
        self._keep.append(blocks)
        d.nblocks, d.blocks = nb, blocks
        # wall-modelled faces
        self.walls = []
        for ib, (b, geo) in enumerate(zip(self.blocks, self.host_geoms)):
            for (a, s), bc in sorted(b.faces.items()):
                if isinstance(bc, WallModel):
                    self.walls.append((ib, a, s, bc))
        walls = (N.WmWall * max(1, len(self.walls)))()
        for w, (ib, a, s, bc) in enumerate(self.walls):
            m = bc.model
            walls[w].block, walls[w].axis, walls[w].side, walls[w].n_match = ib, a, s, int(bc.n_match)
            walls[w].isothermal = 0 if bc.T_wall is None else 1
            walls[w].T_wall = 0.0 if bc.T_wall is None else float(bc.T_wall)
            walls[w].kappa, walls[w].B, walls[w].n_iter = float(m.kappa), float(m.B), int(m.n_iter)
            blk = self.blocks[ib]
            geo = wall_geometry(blk, self.host_geoms[ib], a, s, bc.n_match)
            nt = [blk.n[t] for t in range(3) if t != a]
            if geo.shape != (5, nt[0], nt[1]):
                raise RuntimeError(f"wall geometry of block {blk.name}: shape {geo.shape}, expected {(5, *nt)}")
            walls[w].geom = N.as_double_p(self._arr(geo, np.float64))
        self._keep.append(walls)
        d.nwalls, d.walls = len(self.walls), walls
        # ghost programs
        prog_rhs, prog_all, table = lower_ghost_programs(self.blocks, self.host_geoms, g, self.bc_passes)
        self.ghost_programs = (prog_rhs, prog_all)
        d.ghost_rhs, d.ghost_all = self._program(prog_rhs), self._program(prog_all)
        d.nbc, d.bc_table = len(table), N.as_double_p(self._arr(table, np.float64))
        # synthetic inflow
        d.inflow = None
        for ib, b in enumerate(self.blocks):
            for (a, s), bc in b.faces.items():
                if isinstance(bc, SmoothRampInflow):
                    if d.inflow:
                        raise NotImplementedError("cuda backend: one SmoothRampInflow face per case")
                    inf = N.WmInflow()
                    inf.block, inf.n_modes, inf.n_tab = ib, bc.n_modes, len(bc.profile)
                    inf.modes = N.as_double_p(self._arr(bc.mode_table(), np.float64))
                    inf.table = N.as_double_p(self._arr(bc.profile, np.float64))
                    p = bc.props
                    inf.U_inf, inf.L, inf.rho_inf, inf.p_inf = p["U_inf"], p["L"], p["rho_inf"], p["p_inf"]
                    self._keep.append(inf)
                    d.inflow = C.pointer(inf)
        self.has_inflow = bool(d.inflow)
        # sources
        d.sponge.enabled = 0
        for src in self.sources:
            if not isinstance(src, SmoothRampSponge) or d.sponge.enabled:
                raise NotImplementedError("cuda backend: supports one SmoothRampSponge source")
            d.sponge = N.WmSponge(1, src.x_start_l, src.x_end_l, src.strength, src.props["U_inf"], src.props["L"])
        d.tile = -1 if tile is None else int(tile)
        d.chunk = 0 if chunk is None else int(chunk)
        self._keep.append(d)
        return d

    # ------------------------------------------------------------------ state helpers
    def _check_state(self, Q):
        if len(Q) != len(self.blocks):
            raise ValueError(f"state has {len(Q)} blocks, mesh has {len(self.blocks)}")
        for q, b in zip(Q, self.blocks):
            if not isinstance(q, torch.Tensor) or q.device.type != "cuda":
                raise TypeError("cuda backend state must be torch CUDA tensors")
            if q.dtype != torch.float64 or tuple(q.shape) != (5,) + tuple(b.N) or not q.is_contiguous():
                raise ValueError(f"block {b.name}: expected contiguous float64 (5, {b.N}), got "
                                 f"{q.dtype} {tuple(q.shape)}")

    def _ptrs(self, Q):
        return N.ptr_array([q.data_ptr() for q in Q])

    def _stream(self):
        return C.c_void_p(torch.cuda.current_stream(self.device).cuda_stream)

    def _dt_tensor(self, dt):
        if isinstance(dt, torch.Tensor):
            t = dt.to(device=self.device, dtype=torch.float64).reshape(())
            return t.contiguous()
        return torch.full((), float(dt), dtype=torch.float64, device=self.device)

    # ------------------------------------------------------------------ API
    def init_state(self, prim_fn):
        """prim_fn(xc) -> primitives [rho, u, v, w, p] at the ghosted cell centres
        (wmles/solver.py:54-56); evaluated with NumPy on the host, then uploaded."""
        out = []
        for geo in self.host_geoms:
            w = np.asarray(prim_fn(geo.xc), float)
            out.append(torch.from_numpy(np.ascontiguousarray(self.gas.prim_to_cons(w))).to(self.device))
        return tuple(out)

    def apply_bcs(self, Q, geoms=None, time=0.0):
        """New state with every ghost cell filled (wmles/solver.py:59-73).  Accepts the
        reference's (Q, geoms, time) call as well as (Q, time=...)."""
        if not isinstance(geoms, (tuple, list)) and geoms is not None:
            time = geoms
        self._check_state(Q)
        out = tuple(q.clone() for q in Q)
        N.check(self._lib.wm_apply_bcs(self._case, self._ptrs(out), float(time), self._stream()), "wm_apply_bcs")
        return out

    def rhs(self, Q, time=0.0):
        """RHS on the interior, zero on the ghosts (wmles/solver.py:97-106)."""
        self._check_state(Q)
        R = tuple(torch.zeros_like(q) for q in Q)
        N.check(self._lib.wm_rhs(self._case, self._ptrs(Q), self._ptrs(R), float(time), self._stream()), "wm_rhs")
        return R

    def max_dt(self, Q, time=0.0):
        """CFL time step as a 0-d CUDA tensor (``float(dt)`` synchronises)."""
        self._check_state(Q)
        dt = torch.empty((), dtype=torch.float64, device=self.device)
        N.check(self._lib.wm_max_dt(self._case, self._ptrs(Q), N.ptr_array([dt.data_ptr()])[0], self._stream()),
                "wm_max_dt")
        return dt

    def advance(self, Q, dt, time=0.0):
        """One SSP-RK3 step plus constraints (wmles/solver.py:123-133).  The interior is the
        result; the ghost cells of the returned state are those of Q after the step's
        boundary fill (which refreshes Q's ghost cells in place) plus the constraint's shift,
        as in the reference, where the RK stages combine ghost values the RHS leaves at
        zero and the constraint shifts every cell."""
        self._check_state(Q)
        dtt = self._dt_tensor(dt)
        out = tuple(torch.empty_like(q) for q in Q)
        N.check(self._lib.wm_advance(self._case, self._ptrs(Q), self._ptrs(out), N.ptr_array([dtt.data_ptr()])[0],
                                     float(time), self._stream()), "wm_advance")
        return out

    def step(self, Q, time=0.0):
        """dt = max_dt(Q); Q' = advance(Q, dt); returns (Q', dt).

        The CFL reduction of Q' is fused into the step's last pass; when the next call is
        handed exactly the returned state (same tensors, not modified in place since),
        that dt is reused instead of reducing Q' again."""
        self._check_state(Q)
        chain = getattr(self, "_chain", None)
        if (chain is not None and len(chain[0]) == len(Q)
                and all(r() is q and q._version == v for (r, v), q in zip(chain[0], Q))):
            dt = chain[1]
        else:
            dt = self.max_dt(Q)
        dt_next = torch.empty((), dtype=torch.float64, device=self.device)
        out = tuple(torch.empty_like(q) for q in Q)
        N.check(self._lib.wm_step_fused(self._case, self._ptrs(Q), self._ptrs(out),
                                        N.ptr_array([dt.data_ptr()])[0], N.ptr_array([dt_next.data_ptr()])[0],
                                        float(time), self._stream()), "wm_step_fused")
        self._chain = (tuple((weakref.ref(q), q._version) for q in out), dt_next)
        return out, dt

    # ------------------------------------------------------------------ failure detection
    def status(self, clear=False):
        """The case's status word (bits _native.ST_*: non-finite state, non-positive density
        or pressure, bad time step, unsettled wall-model Newton), accumulated by the kernels
        since the last clear; synchronises the current stream."""
        st = C.c_uint()
        N.check(self._lib.wm_case_status(self._case, C.byref(st), 1 if clear else 0, self._stream()),
                "wm_case_status")
        return st.value

    def check(self):
        """Raise _native.NonFiniteStateError if a step or CFL pass since the last check saw a
        state that is no longer a flow state (NaN / Inf, density or pressure <= 0, a time step
        that is not finite and positive); clears the word.  Synchronises the current stream."""
        N.check(self._lib.wm_check(self._case, self._stream()), "wm_check")

    # ------------------------------------------------------------------ measurement
    def profile(self, enable=True):
        """Reset launch counters; with ``enable`` also time every launch with CUDA events."""
        N.check(self._lib.wm_profile_enable(self._case, 1 if enable else 0), "wm_profile_enable")

    def profile_read(self, kind=-1):
        """(device ms summed over recorded launches, launch count) of one kernel kind
        (_native.KIND_*; -1 = all)."""
        ms, n = C.c_double(), C.c_longlong()
        N.check(self._lib.wm_profile_read(self._case, int(kind), C.byref(ms), C.byref(n)), "wm_profile_read")
        return ms.value, n.value

    def wall_stats(self, Q):
        """{(block, face): (tau_w, q_w)} host arrays for every wall-modelled face
        (wmles/solver.py:163-179)."""
        out = {}
        for key, buf in self.wall_stats_device(Q).items():
            h = buf.cpu().numpy()
            out[key] = (h[0], h[1])
        return out

    def wall_stats_device(self, Q):
        """{(block, face): tensor (2, nt1, nt2) of (tau_w, q_w)} on the device, no host copy."""
        self._check_state(Q)
        bufs = []
        for ib, a, s, bc in self.walls:
            b = self.blocks[ib]
            t = [x for x in range(3) if x != a]
            bufs.append(torch.empty((2, b.n[t[0]], b.n[t[1]]), dtype=torch.float64, device=self.device))
        if not bufs:
            return {}
        N.check(self._lib.wm_wall_stats(self._case, self._ptrs(Q), self._ptrs(bufs), self._stream()), "wm_wall_stats")
        return {(self.blocks[ib].name, "ijk"[a] + ("min", "max")[s]): buf
                for (ib, a, s, bc), buf in zip(self.walls, bufs)}

    def wall_loads(self, Q, moment_center=(0.0, 0.0, 0.0)):
        """Integrated fluid-on-wall force and moment per wall-modelled face
        (wmles/solver.py:181-232); tau_w from the device wall model, the surface
        integration on the host in FP64."""
        center = np.asarray(moment_center, dtype=float)
        if center.shape != (3,) or not np.all(np.isfinite(center)):
            raise ValueError("moment_center must contain three finite coordinates")
        stats = self.wall_stats(Q)
        out = {}
        for ib, a, s, bc in self.walls:
            blk, geo = self.blocks[ib], self.host_geoms[ib]
            ng, n = blk.ng, blk.n[a]
            fb = ng if s == 0 else ng + n
            mi = ng + bc.n_match - 1 if s == 0 else ng + n - bc.n_match
            ci = ng if s == 0 else ng + n - 1
            q = Q[ib]
            qm = blk.take(q, a, mi).cpu().numpy()
            qc = blk.take(q, a, ci).cpu().numpy()
            wm, _ = self.gas.cons_to_prim(qm)
            wc, _ = self.gas.cons_to_prim(qc)
            Sv = blk.take(geo.S[a], a, fb)
            area = np.sqrt(np.sum(Sv * Sv, axis=0))
            nrm = Sv / area
            if s == 0:
                nrm = -nrm
            vel = wm[1:4]
            vt = vel - np.sum(vel * nrm, axis=0)[None] * nrm
            tang = vt / np.sqrt(np.sum(vt ** 2, axis=0) + 1e-20)
            name = (blk.name, "ijk"[a] + ("min", "max")[s])
            tau = stats[name][0]
            trac = (wc[4][None] * nrm + tau[None] * tang) * area[None]
            arm = blk.take(geo.xf[a], a, fb) - center.reshape(3, 1, 1)
            mom = np.stack([arm[1] * trac[2] - arm[2] * trac[1], arm[2] * trac[0] - arm[0] * trac[2],
                            arm[0] * trac[1] - arm[1] * trac[0]])
            out[name] = (np.sum(trac, axis=(1, 2)), np.sum(mom, axis=(1, 2)))
        return out
