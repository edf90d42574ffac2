"""Autotuner bookkeeping without a GPU: cache keys, the cache file round trip, the choice."""
from wmles_jax_b200 import autotune as A


def test_workload_key_is_order_free():
    k1 = A.workload_key([(48, 48, 48), (64, 48, 48)], "mixed", "KEP4", "wale", "B200")
    k2 = A.workload_key([(64, 48, 48), (48, 48, 48)], "mixed", "KEP4", "wale", "B200")
    assert k1 == k2
    assert k1 != A.workload_key([(48, 48, 48)], "mixed", "KEP4", "wale", "B200")
    assert k1 != A.workload_key([(48, 48, 48), (64, 48, 48)], "fp64", "KEP4", "wale", "B200")


def test_cache_round_trip(tmp_path, monkeypatch):
    path = tmp_path / "sub" / "tiles.json"
    monkeypatch.setenv("WMLES_TUNE_CACHE", str(path))
    assert A.cache_path() == str(path)
    assert A.load_cache() == {}
    A.store("k", {"tile": 1, "ms_per_step": {"0": 2.0, "1": 1.5}})
    A.store("j", {"tile": 0, "ms_per_step": {"0": 1.0}})
    data = A.load_cache()
    assert data["k"]["tile"] == 1 and data["j"]["tile"] == 0
    path.write_text("not json")
    assert A.load_cache() == {}


def test_pick_fastest_lowest_id_on_ties():
    assert A.pick({0: 2.0, 1: 1.0, 3: 1.5}) == 1
    assert A.pick({2: 1.0, 0: 1.0}) == 0
    assert set(A.CANDIDATES["fp64"]) < set(A.CANDIDATES["mixed"]) == set(A.TILE_SHAPES)
