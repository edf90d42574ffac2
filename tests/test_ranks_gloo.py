"""Multi-rank plumbing of bench.py on CPU: two gloo ranks agree on the slowest rank's time,
pass the barrier, and the reference arm runs on rank 0 only (the other ranks print nothing)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        bench.rank_barrier(dist)
        ms = 3.0 + rank                                  # rank 1 is the slower one
        got = bench.reduce_max(ms, dist, "cpu")
        value = bench.whole_job_value(1000, world, got)
        ref = bench.run_reference(None, rank, world) if rank != 0 else "rank0"
        out.put((rank, got, value, ref))
        bench.rank_barrier(dist)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [4.0, 4.0]            # both ranks report the slowest time
    assert all(abs(r[2] - 1000 * 2 / 4e-3 / 1e6) < 1e-12 for r in res)
    assert res[1][3] is None                             # the reference arm is rank 0's alone


def test_single_process_identity():
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    assert bench.reduce_max(2.5, None) == 2.5
    bench.rank_barrier(None)
    assert bench.whole_job_value(4_194_304, 1, 2.0) == pytest.approx(2097.152)
