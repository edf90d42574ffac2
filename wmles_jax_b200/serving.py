"""Continuous batching of many independent cases on one GPU.

A *request* is one case (mesh, gas, solver options, initial condition) to be advanced a
fixed number of steps; its result is the final state.  Requests arrive at any time.  The
server keeps every admitted case resident in HBM (metrics, ghost programs, two state
buffers used in ping-pong, two device time steps) and advances ALL resident cases together:
one ``wm_batch_step`` per step, i.e. one launch per kernel per RK stage over the
concatenated block / tile work list of every case (libwmles_cuda.so, wm_batch_*).  While the
set of resident cases stays the same, each step is replayed from a CUDA graph (two graphs,
one per ping-pong parity).  Between steps the server retires finished cases and admits
waiting ones, so requests that arrive while others run join the next step.

* Admission: a request is admitted when its estimated device bytes fit in the free HBM
  (device free memory plus what PyTorch's allocator holds unused) minus a reserve, and the
  batch has block slots left (at most ``WM_MAX_BLOCKS`` blocks per batch).
* Scheduling: every resident case is a candidate each time the set changes (an arrival or
  a completion); the cases with the least remaining work (cells x steps left) are stepped,
  up to a cell budget that fills the GPU, and the others stay paused on the device, so
  short requests do not wait behind long ones while the GPU stays full (FIFO available).
* Host preparation (lowering, ghost programs, initial state) runs on builder threads,
  overlapping the GPU steps; graph captures and device-side case construction exclude each
  other.
* Results do not depend on the mix: per-case reductions run over that case's own cells in
  a fixed order and its stage tiles are fixed at construction, so a case advanced in any
  batch is bit-identical to the same case advanced alone with ``Solver.step``.
* Time-to-result is measured from the request's arrival to the moment the host sees the
  device finish the request's last step (an event per step, at most six steps in flight).
* Failure: every step also copies the members' status words (non-finite state, density or
  pressure <= 0, bad time step) to page-locked host memory; when the host sees a fatal bit
  it evicts that case between steps (its result is an error, its memory is freed) while the
  others go on unchanged (their reductions never mix with another case's).

No reference counterpart: the reference advances one case per ``Solver`` in a Python loop
(examples/channel_wmles.py:121-152).
"""
import ctypes as C
import queue
import sys
import threading
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as N
from .lowering import NMET


# ---------------------------------------------------------------------------- batch handle
class Batch:
    """A wm_batch over solvers that share precision, scheme, SGS model and tile shape."""

    def __init__(self, solvers):
        self.solvers = list(solvers)
        if not self.solvers:
            raise ValueError("a batch needs at least one solver")
        self._lib = N.load()
        arr = (C.c_void_p * len(self.solvers))(*[s._case.value for s in self.solvers])
        h = C.c_void_p()
        N.check(self._lib.wm_batch_create(len(self.solvers), arr, C.byref(h)), "wm_batch_create")
        self._h = h
        nb, nt, nl = C.c_int(), C.c_int(), C.c_longlong()
        N.check(self._lib.wm_batch_info(h, C.byref(nb), C.byref(nt), C.byref(nl)), "wm_batch_info")
        self.nblocks, self.ntiles, self.launches_per_step = nb.value, nt.value, nl.value

    def args(self, q_in, q_out, dt_in, dt_next, times=None):
        """Pointer arrays of one step: q_in/q_out are per-solver state tuples, dt_* per-solver
        0-d float64 tensors.  Built once per membership and parity, replayed many times."""
        flat = lambda qs: N.ptr_array([q.data_ptr() for Q in qs for q in Q])  # noqa: E731
        t = np.zeros(len(self.solvers)) if times is None else np.asarray(times, dtype=np.float64)
        return (flat(q_in), flat(q_out), N.ptr_array([d.data_ptr() for d in dt_in]),
                N.ptr_array([d.data_ptr() for d in dt_next]), np.ascontiguousarray(t))

    def step_args(self, args, stream=None):
        qi, qo, di, dn, t = args
        s = C.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)
        N.check(self._lib.wm_batch_step(self._h, qi, qo, di, dn, N.as_double_p(t), s), "wm_batch_step")

    def step(self, q_in, q_out, dt_in, dt_next, times=None, stream=None):
        self.step_args(self.args(q_in, q_out, dt_in, dt_next, times), stream)

    def status_async(self, stream=None):
        """Enqueue a copy of the member cases' status words (bits _native.ST_*, member order)
        into a page-locked host array, returned; read it once an event recorded after this
        call has completed.  The words only accumulate bits, so a read that races a later
        copy still sees every fault up to the event."""
        if getattr(self, "_status", None) is None:
            self._status = torch.zeros(len(self.solvers), dtype=torch.int32).pin_memory()
        s = C.c_void_p((stream or torch.cuda.current_stream()).cuda_stream)
        N.check(self._lib.wm_batch_status(self._h, C.c_void_p(self._status.data_ptr()), s), "wm_batch_status")
        return self._status

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            self._lib.wm_batch_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # pragma: no cover - interpreter shutdown
            pass


# ---------------------------------------------------------------------------- requests
@dataclass
class Request:
    """One case to advance ``steps`` steps.  ``build()`` returns (mesh, gas, solver kwargs,
    prim_fn) like workloads.channel_case; ``dims`` are the interior extents of its blocks
    (known before building, used for admission)."""
    rid: int
    build: object
    steps: int
    arrival: float = 0.0                  # seconds after the server starts
    dims: tuple = ()
    meta: dict = field(default_factory=dict)

    @property
    def cells(self):
        return int(sum(np.prod(d) for d in self.dims))


def estimate_bytes(dims, precision, ng=3):
    """Device bytes of a resident case: FP64 metrics (+ FP32 copy for the mixed form), two
    work states of the RK stages, two ping-pong states, plus 10 % for wall faces, ghost
    programs and tables."""
    met = NMET * (8 + (4 if precision == "mixed" else 0))
    per_cell = met + 2 * 40 + 2 * 40
    cells = sum(int(np.prod([n + 2 * ng for n in d])) for d in dims)
    return int(1.1 * per_cell * cells) + (1 << 20)


def free_device_bytes(device=None):
    free, _ = torch.cuda.mem_get_info(device)
    return free + torch.cuda.memory_reserved(device) - torch.cuda.memory_allocated(device)


class Admission:
    """Admission bookkeeping.  Bytes, blocks and interior cells of admitted cases (resident,
    or admitted and still being built) are charged against limits fixed at start: a byte
    budget (device free bytes minus a reserve), the batch's block slots, and a cell budget
    that keeps one batch step large enough to fill the GPU without making every resident
    case wait for all the others (None: no cell limit).  A case is always admitted into an
    empty server if its bytes fit."""

    def __init__(self, budget_bytes, max_blocks=N.MAX_BLOCKS, max_cases=N.MAX_BLOCKS, max_cells=None):
        self.budget, self.max_blocks, self.max_cases = int(budget_bytes), max_blocks, max_cases
        self.max_cells = max_cells
        self.used = 0
        self.blocks = 0
        self.cases = 0
        self.cells = 0
        self.peak = 0             # most bytes ever charged at once

    def never_fits(self, nbytes, nblocks):
        """True for a request that exceeds the limits even with nothing else admitted."""
        return nbytes > self.budget or nblocks > self.max_blocks

    def fits(self, nbytes, nblocks, ncells=0):
        if nbytes > self.budget or nblocks > self.max_blocks:
            raise ValueError(f"request needs {nbytes} bytes / {nblocks} blocks: it can never be admitted "
                             f"(budget {self.budget} bytes, {self.max_blocks} blocks)")
        cells_ok = self.max_cells is None or self.cases == 0 or self.cells + ncells <= self.max_cells
        return (self.used + nbytes <= self.budget and self.blocks + nblocks <= self.max_blocks
                and self.cases + 1 <= self.max_cases and cells_ok)

    def take(self, nbytes, nblocks, ncells=0):
        self.used += nbytes
        self.peak = max(self.peak, self.used)
        self.blocks += nblocks
        self.cases += 1
        self.cells += ncells

    def give(self, nbytes, nblocks, ncells=0):
        self.used -= nbytes
        self.blocks -= nblocks
        self.cases -= 1
        self.cells -= ncells


def order_key(policy):
    """Admission order among arrived requests: "sjf" = least work (cells x steps) first, ties
    by arrival; "fifo" = arrival order."""
    if policy == "sjf":
        return lambda r: (r.cells * r.steps, r.arrival, r.rid)
    if policy == "fifo":
        return lambda r: (r.arrival, r.rid)
    raise ValueError(f"unknown admission policy {policy!r}")


def pick_next(waiting, admission, precision, policy):
    """The first arrived request, in policy order, that the admission limits accept (None if
    none fits now).  Under "fifo" a request that does not fit blocks the ones behind it."""
    for r in sorted(waiting, key=order_key(policy)):
        if admission.fits(estimate_bytes(r.dims, precision), len(r.dims), r.cells):
            return r
        if policy == "fifo":
            return None
    return None


@dataclass
class _Resident:
    req: Request
    solver: object
    bufs: list            # [state A, state B], tuples of per-block tensors
    dts: list             # [dt A, dt B], 0-d float64 tensors
    nbytes: int
    parity: int = 0       # bufs[parity] holds the current state
    done: int = 0         # steps completed
    admitted: float = 0.0
    fault: str = None     # set once the case's status word shows a fatal fault


@dataclass
class Result:
    rid: int
    state: tuple          # final state (device tensors); None if the request failed
    dt: torch.Tensor      # CFL time step of the final state (device); NaN if the state is not finite
    steps: int
    cells: int
    arrival: float
    admitted: float
    finished: float
    error: str = None     # why the request could not be served (its case could not be built,
                          # or its state stopped being a flow state and it was evicted)

    @property
    def ok(self):
        return self.error is None

    @property
    def time_to_result(self):
        return self.finished - self.arrival


def select_active(resident, policy, max_cells, max_blocks=N.MAX_BLOCKS):
    """Resident cases to step next: in policy order ("srpt": least remaining work, cells x
    steps left, first; "fifo": arrival order), taken greedily while the batch stays within
    `max_cells` interior cells (None: no limit) and `max_blocks` blocks and cases (the first
    case always).  The others stay resident and paused.  Items need ``.req`` (a Request)
    and ``.done`` (steps taken)."""
    if policy == "fifo":
        order = sorted(resident, key=lambda r: (r.req.arrival, r.req.rid))
    else:
        order = sorted(resident, key=lambda r: (r.req.cells * (r.req.steps - r.done), r.req.arrival, r.req.rid))
    chosen, cells, blocks = [], 0, 0
    for r in order:
        nb = len(r.req.dims)
        if chosen and (blocks + nb > max_blocks or len(chosen) + 1 > max_blocks
                       or (max_cells is not None and cells + r.req.cells > max_cells)):
            continue
        chosen.append(r)
        cells += r.req.cells
        blocks += nb
    return chosen


# ---------------------------------------------------------------------------- server
class Server:
    """Continuous-batching server (see the module docstring).

    precision / tile / chunk: solver options shared by every case (one batch; tile="auto" tunes
    the tile shape over the grids of the requests before serving); graphs: replay
    steps from CUDA graphs once a membership has run ``graph_after`` steps eagerly;
    reserve_bytes: HBM left free; budget_bytes: override of the memory budget of built cases;
    max_cells: interior cells stepped together (None: all resident cases); policy: which
    resident cases are stepped ("srpt": least remaining work first, the others paused on the
    device until they are among the least again; "fifo": arrival order); builders: host
    threads preparing cases (smallest first, or in arrival order under "fifo")."""

    def __init__(self, precision="mixed", tile=None, chunk=None, graphs=True, graph_after=2,
                 reserve_bytes=4 << 30, budget_bytes=None, max_cells=8 << 20, policy="srpt", builders=2,
                 device=None):
        from .backend import require_gpu
        self.device = device or require_gpu()
        self.precision, self.tile, self.chunk = precision, tile, chunk
        self.tuned = None
        self.graphs, self.graph_after = graphs, graph_after
        self.in_flight = 6          # steps queued ahead: slack against host-side stalls
        if policy not in ("srpt", "fifo"):
            raise ValueError(f"unknown scheduling policy {policy!r}")
        self.policy, self.builders = policy, max(1, int(builders))
        self.max_cells = max_cells
        budget = budget_bytes if budget_bytes is not None else free_device_bytes(self.device) - reserve_bytes
        # building is bounded by memory and by a lookahead of twice the cell budget (built,
        # unfinished cases); the cell budget bounds the cases stepped together
        self.admission = Admission(max(0, budget), max_blocks=1 << 30, max_cases=1 << 30,
                                   max_cells=None if max_cells is None else 2 * max_cells)
        self.stream = torch.cuda.Stream(self.device)
        self._lock = threading.Lock()             # case construction vs graph capture
        self._cond = threading.Condition()        # admission waits for retirements
        self.stats = {}

    # ------------------------------------------------------------------ building
    def _build(self, req, bstream):
        """Host work (lowering, initial state) unlocked; device work under the lock that keeps
        it out of graph captures."""
        from .solver import Solver
        mesh, gas, kw, prim = req.build()
        solver = Solver.__new__(Solver)
        solver._prepare(mesh, gas, precision=self.precision, tile=self.tile, chunk=self.chunk, **kw)
        if solver.has_inflow:
            raise NotImplementedError("the server advances cases without a synthetic inflow only")
        # the initial state exactly as Solver.init_state builds it
        q0 = [np.ascontiguousarray(gas.prim_to_cons(np.asarray(prim(g.xc), float))) for g in solver.host_geoms]
        with self._lock, torch.cuda.stream(bstream):
            solver._create()
            qa = tuple(torch.from_numpy(q).to(self.device) for q in q0)
            qb = tuple(torch.empty_like(q) for q in qa)
            da = solver.max_dt(qa)
            db = torch.empty_like(da)
            bstream.synchronize()
        return solver, [qa, qb], [da, db]

    def _builder(self, todo, t0, ready, errors, left):
        bstream = torch.cuda.Stream(self.device)
        try:
            while True:
                with self._cond:
                    while True:
                        if errors:
                            return
                        if not todo:
                            return
                        now = time.perf_counter() - t0
                        waiting = [r for r in todo if r.arrival <= now]
                        for r in [r for r in waiting if self.admission.never_fits(
                                estimate_bytes(r.dims, self.precision), len(r.dims))]:
                            todo.remove(r)     # larger than the whole budget: fails alone
                            waiting.remove(r)
                            ready.put(Result(r.rid, None, None, 0, r.cells, r.arrival, now, now,
                                             error="MemoryError: larger than the device memory budget"))
                        req = pick_next(waiting, self.admission, self.precision,
                                        "fifo" if self.policy == "fifo" else "sjf")
                        if req is not None:
                            break
                        nxt = min(r.arrival for r in todo) - now
                        self._cond.wait(timeout=min(0.05, nxt) if nxt > 0 else 0.05)
                    todo.remove(req)
                    nbytes = estimate_bytes(req.dims, self.precision)
                    self.admission.take(nbytes, len(req.dims), req.cells)
                try:
                    solver, bufs, dts = self._build(req, bstream)
                except Exception as e:      # this request fails; the server goes on
                    with self._cond:
                        self.admission.give(nbytes, len(req.dims), req.cells)
                        self._cond.notify_all()
                    ready.put(Result(req.rid, None, None, 0, req.cells, req.arrival, time.perf_counter() - t0,
                                     time.perf_counter() - t0, error=f"{type(e).__name__}: {e}"))
                    continue
                ready.put(_Resident(req, solver, bufs, dts, nbytes, admitted=time.perf_counter() - t0))
        except BaseException as e:   # surfaced by run()
            errors.append(e)
        finally:
            with self._cond:
                left[0] -= 1
                last = left[0] == 0
                self._cond.notify_all()
            if last:
                ready.put(None)

    def tune(self, requests):
        """Tile shape for this server's cases: one case of each distinct grid of ``requests``,
        advanced together under each candidate tile (autotune.tune, cached)."""
        from .autotune import tune
        seen, cases = set(), []
        for r in requests:
            if r.dims not in seen:
                seen.add(r.dims)
                cases.append(r.build())
        return tune(cases, precision=self.precision)

    # ------------------------------------------------------------------ stepping
    def _capture(self, batch, args):
        """CUDA graph of one batch step, or None while the builder thread holds the device
        (case construction allocates and synchronises, which a capture must not see)."""
        if not self._lock.acquire(blocking=False):
            return None
        try:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.stream(self.stream):
                g.capture_begin(capture_error_mode="thread_local")
                try:
                    batch.step_args(args, self.stream)
                finally:
                    g.capture_end()
            return g
        finally:
            self._lock.release()

    def _select(self, resident):
        return select_active(resident, self.policy, self.max_cells)

    def run(self, requests, timeout=None):
        """Serve ``requests`` (arrival times relative to now); returns {rid: Result}."""
        if self.tile == "auto":
            self.tuned = self.tune(requests)
            self.tile = self.tuned[0]
        todo = sorted(requests, key=lambda r: r.arrival)
        ready, errors, left = queue.Queue(), [], [self.builders]
        # hand the interpreter lock over often: the builder threads run Python-heavy host
        # preparation while this thread must keep the device queue fed
        switch = sys.getswitchinterval()
        sys.setswitchinterval(5e-4)
        try:
            return self._run(todo, ready, errors, left, timeout)
        finally:
            sys.setswitchinterval(switch)

    def _run(self, todo, ready, errors, left, timeout):
        t0 = time.perf_counter()
        workers = [threading.Thread(target=self._builder, args=(todo, t0, ready, errors, left), daemon=True)
                   for _ in range(self.builders)]
        for w in workers:
            w.start()
        resident, active, joined, results = [], [], [], {}
        pending = []               # (event, [residents finished by that step]) of steps in flight
        batch, args, graphs, run_len = None, {}, {}, 0
        builder_done = False
        n = dict(batch_steps=0, graph_steps=0, captures=0, memberships=0, kernel_launches=0, cell_steps=0,
                 pauses=0, evicted=0)
        seg, busy_ms = None, 0.0    # device time of the batch steps, per membership segment

        def close_segment():
            nonlocal seg, busy_ms
            if seg is not None:
                end = torch.cuda.Event(enable_timing=True)
                end.record(self.stream)
                end.synchronize()
                busy_ms += seg.elapsed_time(end)
                seg = None

        def clock():
            return time.perf_counter() - t0

        def take(item):
            nonlocal builder_done
            if item is None:
                builder_done = True
            elif isinstance(item, Result):      # a request that failed to build
                results[item.rid] = item
            else:
                joined.append(item)

        def stamp(upto):
            while len(pending) > upto:
                ev, fin, status, members = pending.pop(0)
                ev.synchronize()
                now = clock()
                # status words of that step's members (bits only accumulate, so a copy enqueued
                # by a later step and landing meanwhile only adds faults)
                for r, bits in zip(members, status.tolist()):
                    if bits & N.ST_FATAL and r.fault is None:
                        r.fault = (f"NonFiniteStateError: {', '.join(N.status_names(bits & N.ST_FATAL))} "
                                   f"within the first {r.done} steps")
                        n["evicted"] += 1
                for r in fin:
                    if r.fault is None:
                        results[r.req.rid] = Result(r.req.rid, r.bufs[r.parity], r.dts[r.parity], r.done,
                                                    r.req.cells, r.req.arrival, r.admitted, now)

        def evict(rs):
            now = clock()
            for r in rs:
                results[r.req.rid] = Result(r.req.rid, None, None, r.done, r.req.cells, r.req.arrival,
                                            r.admitted, now, error=r.fault)

        def release(rs):
            with self._cond:
                for r in rs:
                    r.bufs[1 - r.parity] = None
                    r.dts[1 - r.parity] = None
                    r.solver = None
                    self.admission.give(r.nbytes, len(r.req.dims), r.req.cells)
                self._cond.notify_all()

        with torch.cuda.stream(self.stream):
            while True:
                if errors:
                    raise errors[0]
                if timeout is not None and clock() > timeout:
                    raise TimeoutError("serving did not finish in time")
                if not resident and not joined and not builder_done:
                    try:                       # idle: wait for the next admitted case
                        take(ready.get(timeout=0.05))
                    except queue.Empty:
                        continue
                while True:                    # every case admitted since the last step
                    try:
                        take(ready.get_nowait())
                    except queue.Empty:
                        break
                leaving = [r for r in active if r.done >= r.req.steps or r.fault]
                if joined or leaving or (batch is None and resident):
                    for r in joined:
                        if r.req.steps <= 0:
                            results[r.req.rid] = Result(r.req.rid, r.bufs[0], r.dts[0], 0, r.req.cells,
                                                        r.req.arrival, r.admitted, clock())
                            release([r])
                        else:
                            resident.append(r)
                    joined = []
                    resident = [r for r in resident if r.done < r.req.steps and not r.fault]
                    chosen = self._select(resident)
                    if leaving or [id(r) for r in chosen] != [id(r) for r in active]:
                        # membership change: drain the steps in flight, free the leavers, rebuild
                        close_segment()
                        self.stream.synchronize()
                        stamp(0)
                        # the drained steps may show more faulted cases: they leave now too
                        late = [r for r in resident if r.fault]
                        if late:
                            resident = [r for r in resident if not r.fault]
                            chosen = self._select(resident)
                            leaving += [r for r in late if r not in leaving]
                        evict([r for r in leaving if r.fault])
                        graphs.clear()
                        args = {}
                        if batch is not None:
                            batch.close()
                            batch = None
                        release(leaving)
                        n["pauses"] += sum(1 for r in active if r.done < r.req.steps and r not in chosen)
                        active = chosen
                        if active:
                            batch = Batch([r.solver for r in active])
                            n["memberships"] += 1
                            run_len = 0
                            seg = torch.cuda.Event(enable_timing=True)
                            seg.record(self.stream)
                if not active:
                    if builder_done and ready.empty() and not resident:
                        break
                    continue
                key = tuple(r.parity for r in active)
                if key not in args:
                    args[key] = batch.args([r.bufs[r.parity] for r in active],
                                           [r.bufs[1 - r.parity] for r in active],
                                           [r.dts[r.parity] for r in active],
                                           [r.dts[1 - r.parity] for r in active])
                g = graphs.get(key)
                if g is None and self.graphs and run_len >= self.graph_after:
                    g = self._capture(batch, args[key])
                    if g is not None:
                        graphs[key] = g
                        n["captures"] += 1
                if g is not None:
                    g.replay()
                    n["graph_steps"] += 1
                else:
                    batch.step_args(args[key], self.stream)
                status = batch.status_async(self.stream)
                run_len += 1
                n["batch_steps"] += 1
                n["kernel_launches"] += batch.launches_per_step
                fin = []
                for r in active:
                    r.parity ^= 1
                    r.done += 1
                    n["cell_steps"] += r.req.cells
                    if r.done >= r.req.steps:
                        fin.append(r)
                ev = torch.cuda.Event()
                ev.record(self.stream)
                pending.append((ev, fin, status, list(active)))
                stamp(self.in_flight)          # bounded number of steps in flight
            close_segment()
            self.stream.synchronize()
            stamp(0)
            if batch is not None:
                batch.close()
        for w in workers:
            w.join()
        if errors:
            raise errors[0]
        # faults seen only in the last drain: those cases finished their steps, but their
        # results are not flow states
        for r in list(active) + list(resident):
            if r.fault and results.get(r.req.rid) is not None and results[r.req.rid].ok:
                evict([r])
        served = [r for r in results.values() if r.ok]
        wall = max((r.finished for r in served), default=0.0)
        ttr = np.array([r.time_to_result for r in served])
        nonfinite = sum(1 for r in served if not np.isfinite(float(r.dt)))
        self.stats = dict(n, requests=len(results), failed=len(results) - len(served), nonfinite=nonfinite,
                          wall_s=wall, peak_admitted_bytes=self.admission.peak,
                          mcell_steps_per_s=n["cell_steps"] / wall / 1e6 if wall > 0 else 0.0,
                          device_busy_s=busy_ms * 1e-3,
                          device_mcell_steps_per_s=n["cell_steps"] / (busy_ms * 1e-3) / 1e6 if busy_ms > 0 else 0.0,
                          p50_s=float(np.percentile(ttr, 50)) if len(ttr) else None,
                          p99_s=float(np.percentile(ttr, 99)) if len(ttr) else None)
        return results


# ---------------------------------------------------------------------------- helpers
def serve_alone(req, precision="mixed", tile=None, chunk=None):
    """The request advanced by itself through Solver.step (the reference loop); returns
    (state, dt of the final state)."""
    from .solver import Solver
    mesh, gas, kw, prim = req.build()
    s = Solver(mesh, gas, precision=precision, tile=tile, chunk=chunk, **kw)
    Q = s.init_state(prim)
    for _ in range(req.steps):
        Q, _ = s.step(Q)
    return Q, s.max_dt(Q)
