"""Batched stepping (wm_batch_step) and the continuous-batching server.

Each case's result must be the same alone (Solver.step, one case per call) and in any mix:
in a batch with other cases, with staggered arrivals and departures, replayed from CUDA
graphs, and under an admission budget that keeps only some cases resident.  The per-case
reductions and stage tiles do not depend on the mix, so the tolerance is zero: interior
states and time steps are compared bit for bit."""
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

# (Re_tau, Ma_b, grid): uneven grids, Reynolds and Mach numbers
MIX = [(600.0, 0.3, (16, 16, 16)), (2000.0, 0.15, (24, 16, 16)), (5000.0, 0.45, (16, 24, 16)),
       (1200.0, 0.2, (32, 16, 24))]


def _requests(steps, arrivals):
    from wmles_jax_b200.serving import Request
    from wmles_jax_b200.workloads import serving_case
    out = []
    for r, ((rt, ma, grid), n, t) in enumerate(zip(MIX, steps, arrivals)):
        out.append(Request(rid=r, build=(lambda rt=rt, ma=ma, grid=grid, r=r: serving_case(rt, ma, grid, seed=r)),
                           steps=n, arrival=t, dims=(grid,)))
    return out


def _interior(q):
    return q[:, 3:-3, 3:-3, 3:-3]


def _same(Qa, Qb):
    return all(torch.equal(_interior(a), _interior(b)) for a, b in zip(Qa, Qb))


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_batch_step_matches_alone(precision):
    from wmles_jax_b200 import Solver
    from wmles_jax_b200.serving import Batch, serve_alone
    steps = 6
    reqs = _requests([steps] * len(MIX), [0.0] * len(MIX))
    alone = [serve_alone(r, precision=precision) for r in reqs]
    solvers, bufs, dts = [], [], []
    for r in reqs:
        mesh, gas, kw, prim = r.build()
        s = Solver(mesh, gas, precision=precision, **kw)
        q = s.init_state(prim)
        solvers.append(s)
        bufs.append([q, tuple(torch.empty_like(x) for x in q)])
        d = s.max_dt(q)
        dts.append([d, torch.empty_like(d)])
    batch = Batch(solvers)
    assert batch.nblocks == len(MIX)
    for k in range(steps):
        p = k % 2
        batch.step([b[p] for b in bufs], [b[1 - p] for b in bufs], [d[p] for d in dts], [d[1 - p] for d in dts])
    torch.cuda.synchronize()
    batch.close()
    for i, (Q, dt) in enumerate(alone):
        assert _same(bufs[i][steps % 2], Q), f"case {i}: state differs from the case run alone"
        assert torch.equal(dts[i][steps % 2], dt), f"case {i}: dt differs"


def _check_server(results, reqs, alone):
    assert sorted(results) == [r.rid for r in reqs]
    for r, (Q, dt) in zip(reqs, alone):
        res = results[r.rid]
        assert res.steps == r.steps
        assert _same(res.state, Q), f"request {r.rid}: served state differs from the case run alone"
        assert torch.equal(res.dt, dt)
        assert res.finished >= res.arrival


def test_server_same_alone_and_in_the_mix():
    from wmles_jax_b200.serving import Server, serve_alone
    reqs = _requests([12, 20, 7, 15], [0.0, 0.0, 0.3, 0.6])
    alone = [serve_alone(r) for r in reqs]
    srv = Server(precision="mixed", graphs=True, graph_after=1)
    results = srv.run(reqs, timeout=300)
    _check_server(results, reqs, alone)
    st = srv.stats
    assert st["memberships"] >= 2          # cases joined and left while others ran
    assert st["graph_steps"] > 0 and st["captures"] > 0
    assert st["p50_s"] is not None and st["p99_s"] >= st["p50_s"]


def test_server_admission_budget():
    from wmles_jax_b200.serving import Server, estimate_bytes, serve_alone
    reqs = _requests([5, 9, 4, 6], [0.0] * 4)
    alone = [serve_alone(r) for r in reqs]
    sizes = sorted(estimate_bytes(r.dims, "mixed") for r in reqs)
    budget = sizes[-1] + sizes[0]           # never room for more than two of them
    srv = Server(precision="mixed", graphs=False, budget_bytes=budget)
    results = srv.run(reqs, timeout=300)
    _check_server(results, reqs, alone)
    assert srv.stats["peak_admitted_bytes"] <= budget
    assert srv.stats["memberships"] >= 3


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_results_do_not_depend_on_chunk(precision):
    """The stage work list may be cut into any chunk length along i (a batch picks its own):
    the constant-mass-flux partials are per column and plane, so results are bit-identical.
    Chunks of one and two planes make every segment a prologue, one or two marching steps and
    the segment's closing epilogue."""
    from wmles_jax_b200 import Solver
    from wmles_jax_b200.workloads import serving_case
    outs = []
    for chunk in (None, 1, 2, 4, 7, 24):
        # a fresh builder per run: prim_fn draws its noise from a generator it owns
        mesh, gas, kw, prim = serving_case(1500.0, 0.3, (24, 16, 16), seed=5)
        s = Solver(mesh, gas, precision=precision, chunk=chunk, **kw)
        Q = s.init_state(prim)
        for _ in range(4):
            Q, dt = s.step(Q)
        outs.append((Q, s.max_dt(Q)))
    for Q, dt in outs[1:]:
        assert _same(Q, outs[0][0]) and torch.equal(dt, outs[0][1])


def test_autotune_picks_a_measured_tile(tmp_path, monkeypatch):
    from wmles_jax_b200 import autotune
    from wmles_jax_b200.workloads import serving_case
    monkeypatch.setenv("WMLES_TUNE_CACHE", str(tmp_path / "tiles.json"))
    cases = [serving_case(800.0, 0.3, g, seed=1) for g in ((16, 16, 16), (24, 16, 16))]
    tile, ms = autotune.tune(cases, precision="mixed", steps=4, warmup=3)
    assert set(ms) == set(autotune.CANDIDATES["mixed"]) and tile == autotune.pick(ms)
    assert all(v > 0 for v in ms.values())
    tile2, ms2 = autotune.tune(cases, precision="mixed")     # served from the cache
    assert tile2 == tile and ms2 == ms


def test_server_survives_a_failing_request():
    """A request whose case cannot be built fails alone; the others are served unchanged."""
    from wmles_jax_b200.serving import Request, Server, serve_alone

    def bad():
        raise ValueError("no such grid")
    reqs = _requests([6, 4], [0.0, 0.1])
    reqs.append(Request(rid=99, build=bad, steps=5, arrival=0.05, dims=((8, 8, 8),)))
    reqs.append(Request(rid=98, build=bad, steps=5, arrival=0.0, dims=((4096, 4096, 4096),)))
    alone = [serve_alone(r) for r in reqs[:2]]
    srv = Server(precision="mixed", graphs=False)
    results = srv.run(reqs, timeout=300)
    assert not results[99].ok and "no such grid" in results[99].error
    assert not results[98].ok and "memory" in results[98].error
    _check_server({k: v for k, v in results.items() if k not in (98, 99)}, reqs[:2], alone)
    assert srv.stats["failed"] == 2 and srv.stats["nonfinite"] == 0


def _poisoned(req, value, var):
    """The request with one interior cell of its initial condition replaced by ``value``
    in primitive variable ``var`` (a host-side fault: NaN, or a negative pressure)."""
    from wmles_jax_b200.serving import Request
    build = req.build

    def poisoned():
        mesh, gas, kw, prim = build()

        def prim2(xc):
            w = prim(xc)
            c = tuple(s // 2 for s in w.shape[1:])
            w[(var,) + c] = value
            return w
        return mesh, gas, kw, prim2
    return Request(rid=req.rid, build=poisoned, steps=req.steps, arrival=req.arrival, dims=req.dims)


@pytest.mark.parametrize("value,var,bit", [(float("nan"), 1, 1), (-5.0e3, 4, 4)])
def test_server_evicts_a_faulted_case(value, var, bit):
    """A request whose initial state holds a NaN velocity or a negative pressure is evicted
    with an error naming the fault; the other requests finish bit-identical to running alone;
    Solver.check raises on the same case run alone."""
    from wmles_jax_b200 import Solver, _native as N
    from wmles_jax_b200.serving import Server, serve_alone
    reqs = _requests([12, 20, 7, 15], [0.0, 0.0, 0.2, 0.4])
    bad = 1
    reqs[bad] = _poisoned(reqs[bad], value, var)
    alone = {r.rid: serve_alone(r) for r in reqs if r.rid != bad}
    srv = Server(precision="mixed", graphs=True, graph_after=1)
    results = srv.run(reqs, timeout=300)
    assert sorted(results) == [r.rid for r in reqs]
    res = results[bad]
    assert not res.ok and res.state is None and "NonFiniteStateError" in res.error, res.error
    assert N.ST_NAMES[bit] in res.error
    assert srv.stats["evicted"] == 1 and srv.stats["failed"] == 1
    for r in reqs:
        if r.rid == bad:
            continue
        Q, dt = alone[r.rid]
        assert results[r.rid].ok and _same(results[r.rid].state, Q) and torch.equal(results[r.rid].dt, dt)
    mesh, gas, kw, prim = reqs[bad].build()
    s = Solver(mesh, gas, precision="mixed", **kw)
    Q, _ = s.step(s.init_state(prim))
    assert s.status() & bit
    with pytest.raises(N.NonFiniteStateError):
        s.check()
    assert s.status() == 0                      # check() cleared the word


def test_status_clean_on_a_healthy_case():
    from wmles_jax_b200 import Solver, _native as N
    reqs = _requests([3], [0.0])
    mesh, gas, kw, prim = reqs[0].build()
    s = Solver(mesh, gas, **kw)
    Q = s.init_state(prim)
    for _ in range(3):
        Q, _ = s.step(Q)
    assert s.status() & N.ST_FATAL == 0
    s.check()
