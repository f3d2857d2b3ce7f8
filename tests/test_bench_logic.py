"""Host logic of bench.py that needs no GPU: the headline's launch choices
(command line, autotuner, the opt-in FP16-arithmetic hop) and the lookup of
the ncu traffic figure in the committed profiles."""
import argparse

import bench
from nissa_b200 import tune


class FakeLattice:
    T, LX, LY, LZ = 8, 4, 4, 4
    device = 0

    def __init__(self):
        self.knobs = {}

    def set_tuning(self, k, v):
        self.knobs[k] = v

    def get_tuning(self, k):
        return self.knobs.get(k, 0)

    def bench_hop(self, precision, variant=0, nrep=10, flush=True):
        shape = self.knobs.get("hop_cfg_" + precision, 0)
        return 1.0 + 0.1 * abs(shape - 6), 1e6


def _args(**kw):
    a = dict(precision="half", hop_cfg=-1, tma_rows=-1, half_arith=False)
    a.update(kw)
    return argparse.Namespace(**a)


def test_command_line_choices_name_only_the_given_knobs():
    lat = FakeLattice()
    r = bench.headline_tuning(lat, _args(hop_cfg=5))
    assert r == {"source": "command line", "settings": {"hop_cfg_half": 5}}
    assert lat.knobs == {"hop_cfg_half": 5}
    lat = FakeLattice()
    r = bench.headline_tuning(lat, _args(hop_cfg=7, tma_rows=4, half_arith=True))
    assert r["settings"] == {"hop_cfg_half": 7, "tma_rows": 4, "half_arith": 1, "reliable_delta_half": 0.01}
    assert lat.knobs["half_arith"] == 1 and lat.knobs["reliable_delta_half"] == 0.01


def test_autotuned_headline_then_fp16_arithmetic(tmp_path, monkeypatch):
    monkeypatch.setattr(tune, "default_cache_path", lambda: str(tmp_path / "t.json"))
    import torch
    monkeypatch.setattr(torch.cuda, "get_device_name", lambda *_: "fake", raising=False)
    lat = FakeLattice()
    r = bench.headline_tuning(lat, _args())
    assert r["source"] == "autotuner" and r["settings"]["hop_cfg_half"] == 6
    assert len(r["candidates"]) == len(tune.HOP_SHAPES["half"])
    assert "half_arith" not in lat.knobs
    lat = FakeLattice()
    r = bench.headline_tuning(lat, _args(half_arith=True))
    assert r["source"] == "autotuner (cached)"
    # the FP16-arithmetic hop is switched on after the tuner timed the FP32-arithmetic shapes
    assert r["settings"]["half_arith"] == 1 and lat.knobs["half_arith"] == 1


def test_traffic_figures_come_from_the_committed_profiles():
    t, src = bench.hop_traffic("half", 6)
    assert t and 2.5e8 < t < 3.5e8 and src.startswith("profiles/")
    t, src = bench.hop_traffic("half-fp16-arithmetic", 6)
    assert t and 2.5e8 < t < 3.5e8 and src.startswith("profiles/")
    t, why = bench.hop_traffic("half", 2)
    assert t is None and "no ncu capture" in why
