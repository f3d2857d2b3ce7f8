"""Autotuner host logic with a stand-in lattice (no GPU): the cheapest
candidate wins, the winner is applied and cached, a cached entry is reused
without timing."""
import json

from nissa_b200 import tune


class FakeLattice:
    T, LX, LY, LZ = 8, 4, 4, 4
    device = 0

    def __init__(self, best_shape=3, best_links=1, best_r=2, dims=None, best_rows=None):
        if dims:
            self.T, self.LX, self.LY, self.LZ = dims
        self.knobs = {}
        self.calls = 0
        self.best = (best_shape, best_links, best_r)
        self.best_rows = best_rows

    def set_tuning(self, k, v):
        self.knobs[k] = v

    def bench_hop(self, precision, variant=0, nrep=10, flush=True):
        self.calls += 1
        shape = self.knobs.get("hop_cfg_" + precision, 0)
        links = self.knobs.get("links_single", 0)
        ms = 1.0 + abs(shape - self.best[0]) * 0.1 + (0.0 if links == self.best[1] else 0.05)
        if shape == tune.TILED_SHAPE and self.best_rows:
            ms += 0.01 * abs(self.knobs.get("tma_rows", 0) - self.best_rows)
        return ms, 1e6

    def bench_hop_batched(self, precision, nrhs=12, nrep=5, flush=True):
        self.calls += 1
        return 1.0 + abs(self.knobs.get("mrhs_per_thread", 1) - self.best[2]), 1.0


def test_single_picks_cheapest_and_caches(tmp_path):
    cache = str(tmp_path / "t.json")
    lat = FakeLattice()
    r = tune.autotune(lat, "single", device_name="dev", cache=cache)
    assert not r["cached"]
    assert r["settings"] == {"hop_cfg_single": 3, "links_single": 1}
    assert lat.knobs["hop_cfg_single"] == 3 and lat.knobs["links_single"] == 1
    table = json.load(open(cache))
    assert list(table) == ["dev|8x4x4x4|single|1"]
    lat2 = FakeLattice()
    r2 = tune.autotune(lat2, "single", device_name="dev", cache=cache)
    assert r2["cached"] and lat2.calls == 0
    assert lat2.knobs == {"hop_cfg_single": 3, "links_single": 1}


def test_half_and_batched_keys_are_separate(tmp_path):
    cache = str(tmp_path / "t.json")
    lat = FakeLattice(best_shape=0, best_r=4)
    assert tune.autotune(lat, "half", device_name="dev", cache=cache)["settings"] == {"hop_cfg_half": 0}
    assert tune.autotune(lat, "half", nrhs=48, device_name="dev", cache=cache)["settings"] == {"mrhs_per_thread": 4}
    assert tune.autotune(lat, "double", nrhs=48, device_name="dev", cache=cache)["settings"]["mrhs_per_thread"] in (1, 2)
    assert len(json.load(open(cache))) == 3


def test_retune_ignores_cache(tmp_path):
    cache = str(tmp_path / "t.json")
    lat = FakeLattice(best_shape=1)
    tune.autotune(lat, "double", device_name="dev", cache=cache)
    lat.best = (2, 0, 1)
    r = tune.autotune(lat, "double", device_name="dev", cache=cache, retune=True)
    assert r["settings"] == {"hop_cfg_double": 2}


def test_tile_rows_choices_follow_the_tile_rules():
    # R divides LY, R*LZ/2 <= 128, a partial plane keeps two halo rows and 16 sites
    assert tune.tile_rows_choices(32, 32) == [1, 2, 4, 8]
    assert tune.tile_rows_choices(16, 16) == [2, 4, 8, 16]
    assert tune.tile_rows_choices(24, 24) == [2, 3, 4, 6, 8]
    assert tune.tile_rows_choices(8, 8) == [4, 8]
    assert tune.tile_rows_choices(4, 4) == []        # LZ not a multiple of 8
    assert tune.tile_rows_choices(32, 12) == []
    assert tune.tile_rows_choices(8, 256) == []      # rows longer than 64 sites


def test_site_tiling_is_searched_with_the_staged_shape(tmp_path):
    cache = str(tmp_path / "t.json")
    lat = FakeLattice(best_shape=tune.TILED_SHAPE, dims=(64, 32, 32, 32), best_rows=4)
    r = tune.autotune(lat, "half", device_name="dev", cache=cache)
    assert r["settings"] == {"hop_cfg_half": tune.TILED_SHAPE, "tma_rows": 4}
    assert lat.knobs["tma_rows"] == 4 and lat.knobs["hop_cfg_half"] == tune.TILED_SHAPE
    tiled = [c for c in r["candidates"] if c["hop_cfg"] == tune.TILED_SHAPE]
    assert sorted(c["tma_rows"] for c in tiled) == [1, 2, 4, 8]
    assert len(r["candidates"]) == len(tune.HOP_SHAPES["half"]) - 1 + 4
    # evidence: time and algorithmic bandwidth of each candidate (4 launches of 1e6 bytes)
    for c in r["candidates"]:
        assert abs(c["alg_gbs"] - 4e6 / (c["ms_per_iteration"] * 1e-3) / 1e9) < 1e-9
    assert r["alg_gbs"] == min(r["candidates"], key=lambda c: c["ms_per_iteration"])["alg_gbs"]


def test_untiled_winner_resets_the_tiling(tmp_path):
    cache = str(tmp_path / "t.json")
    lat = FakeLattice(best_shape=6, dims=(64, 32, 32, 32), best_rows=2)
    r = tune.autotune(lat, "half", device_name="dev", cache=cache)
    assert r["settings"] == {"hop_cfg_half": 6, "tma_rows": 0}
    assert lat.knobs["tma_rows"] == 0


def test_record_capture_keeps_ncu_evidence(tmp_path):
    cache = str(tmp_path / "t.json")
    lat = FakeLattice(best_shape=6, dims=(64, 32, 32, 32))
    tune.autotune(lat, "half", device_name="dev", cache=cache)
    e = tune.record_capture((64, 32, 32, 32), "half", 3.0e8, 80e-6, device_name="dev", cache=cache, source="x")
    assert abs(e["ncu"]["dram_gbs"] - 3.0e8 / 80e-6 / 1e9) < 1e-6
    r = tune.autotune(FakeLattice(dims=(64, 32, 32, 32)), "half", device_name="dev", cache=cache)
    assert r["cached"] and r["ncu"]["source"] == "x"
    try:
        tune.record_capture((8, 8, 8, 8), "half", 1.0, 1.0, device_name="dev", cache=cache)
    except KeyError:
        pass
    else:
        raise AssertionError("a capture without a tuned entry is refused")
