"""Autotuner host logic with a stand-in lattice (no GPU): the cheapest
candidate wins, the winner is applied and cached, a cached entry is reused
without timing."""
import json

from nissa_b200 import tune


class FakeLattice:
    T, LX, LY, LZ = 8, 4, 4, 4
    device = 0

    def __init__(self, best_shape=3, best_links=1, best_r=2):
        self.knobs = {}
        self.calls = 0
        self.best = (best_shape, best_links, best_r)

    def set_tuning(self, k, v):
        self.knobs[k] = v

    def bench_hop(self, precision, variant=0, nrep=10, flush=True):
        self.calls += 1
        shape = self.knobs.get("hop_cfg_" + precision, 0)
        links = self.knobs.get("links_single", 0)
        ms = 1.0 + abs(shape - self.best[0]) * 0.1 + (0.0 if links == self.best[1] else 0.05)
        return ms, 1.0

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
