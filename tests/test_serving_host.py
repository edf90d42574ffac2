"""Host logic of the serving layer that needs no GPU: admission accounting, the device-byte
estimate, the seeded request mix and the Re_tau -> Re_b mapping."""
import numpy as np
import pytest

from wmles_jax_b200.serving import Admission, Request, estimate_bytes, pick_next, select_active
from wmles_jax_b200.workloads import SERVING_GRIDS, re_bulk_from_re_tau, serving_requests


def test_admission_accounting():
    a = Admission(1000, max_blocks=3, max_cases=2)
    assert a.fits(600, 1)
    a.take(600, 1)
    assert not a.fits(500, 1)          # bytes
    assert a.fits(400, 2)
    a.take(400, 2)
    assert not a.fits(0, 1)            # blocks and cases
    a.give(600, 1)
    assert a.fits(500, 1) and a.peak == 1000 and a.used == 400
    assert a.never_fits(2000, 1) and not a.never_fits(1000, 1)
    with pytest.raises(ValueError):
        a.fits(2000, 1)                # can never be admitted
    with pytest.raises(ValueError):
        a.fits(10, 4)


def test_admission_cell_budget():
    a = Admission(1 << 40, max_cells=100)
    assert a.fits(1, 1, 500)             # an empty server admits any case whose bytes fit
    a.take(1, 1, 500)
    assert not a.fits(1, 1, 1)
    a.give(1, 1, 500)
    a.take(1, 1, 60)
    assert a.fits(1, 1, 40) and not a.fits(1, 1, 41)


def _req(rid, dims, steps, arrival):
    return Request(rid=rid, build=None, steps=steps, arrival=arrival, dims=(dims,))


def test_pick_next_policies():
    big, small, mid = _req(0, (40, 40, 40), 10, 0.0), _req(1, (8, 8, 8), 10, 0.5), _req(2, (20, 20, 20), 10, 0.2)
    waiting = [big, small, mid]
    a = Admission(1 << 40)
    assert pick_next(waiting, a, "mixed", "sjf") is small
    assert pick_next(waiting, a, "mixed", "fifo") is big
    # sjf backfills with whatever fits; fifo does not skip the head of the queue
    a = Admission(1 << 40, max_cells=9000)
    a.take(1, 1, 1)
    assert pick_next([big, mid], a, "mixed", "sjf") is mid
    assert pick_next([big, mid], a, "mixed", "fifo") is None
    with pytest.raises(ValueError):
        pick_next(waiting, a, "mixed", "lifo")


def test_estimate_bytes():
    small, big = estimate_bytes([(48, 48, 48)], "mixed"), estimate_bytes([(192, 96, 96)], "mixed")
    assert big > small > 0
    assert estimate_bytes([(48, 48, 48)], "fp64") < small          # no FP32 metric copy
    # at least the two ping-pong and two work states of 5 float64 per ghosted cell
    assert small >= 4 * 40 * 54 ** 3


def test_re_mapping_inverts_dean():
    re_tau = np.array([550.0, 1000.0, 5200.0])
    re_m = 2.0 * re_bulk_from_re_tau(re_tau)
    np.testing.assert_allclose(0.09 * re_m ** 0.88, re_tau, rtol=1e-12)


def test_serving_requests_seeded_mix():
    a, b = serving_requests(), serving_requests()
    assert len(a) == 64
    assert [r.arrival for r in a] == [r.arrival for r in b]
    assert [r.meta for r in a] == [r.meta for r in b]
    arr = np.array([r.arrival for r in a])
    assert np.all(np.diff(arr) > 0) and arr[0] > 0
    assert 1.0 < arr[-1] < 8.0                       # 64 arrivals at 20 per second
    for r in a:
        assert 550.0 <= r.meta["re_tau"] <= 5200.0 and 0.1 <= r.meta["ma_b"] <= 0.5
        assert r.meta["grid"] in SERVING_GRIDS and r.dims == (r.meta["grid"],) and r.steps == 2000
    assert len({r.meta["grid"] for r in a}) == len(SERVING_GRIDS)
    assert serving_requests(seed=1)[0].arrival != a[0].arrival


def test_backend_names_the_drivers_use():
    from wmles_jax_b200 import backend
    assert backend.HAS_JAX is False and hasattr(backend, "xp") and callable(backend.device_info)
    import torch
    if not torch.cuda.is_available():
        assert backend.DEVICE is None
        with pytest.raises(RuntimeError):
            backend.asarray([1.0, 2.0])


class _Res:
    def __init__(self, req, done=0):
        self.req, self.done = req, done


def test_select_active_least_remaining_work_within_budget():
    a = _Res(_req(0, (40, 40, 40), 100, 0.0))            # 64000 cells, 6.4 M cell-steps
    b = _Res(_req(1, (8, 8, 8), 100, 0.5))               # 512 cells
    c = _Res(_req(2, (20, 20, 20), 100, 0.2), done=50)   # 8000 cells, half done
    assert [r.req.rid for r in select_active([a, b, c], "srpt", None)] == [1, 2, 0]
    # a budget that does not hold the big case pauses it; the first case is always taken
    assert [r.req.rid for r in select_active([a, b, c], "srpt", 10000)] == [1, 2]
    assert [r.req.rid for r in select_active([a], "srpt", 10)] == [0]
    # remaining work, not size: the big case near its end (64000 cell-steps left) overtakes
    # the half-done medium one (400000 left)
    a.done = 99
    assert [r.req.rid for r in select_active([a, b, c], "srpt", None)] == [1, 0, 2]
    assert [r.req.rid for r in select_active([a, b, c], "fifo", None)] == [0, 2, 1]
    assert len(select_active([_Res(_req(i, (4, 4, 4), 1, 0.0)) for i in range(200)], "srpt", None)) == 96
