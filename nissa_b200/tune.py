"""Autotuning of the launch choices of one lattice on one GPU.

The choices (all results-neutral: every choice computes the same operator and
solver) are the tuning knobs of the C ABI (tms_set_tuning):

  hop_cfg_<precision>  launch shape of the e/o hopping kernel (one or two
                       sites per thread, register caps, packed FP32 spin rows,
                       gathers streamed through shared memory by cp.async,
                       row tiles staged by bulk copies)
  links_single         FP32 or 16-bit links under the FP32 inner solver
  mrhs_per_thread      right-hand sides per thread of the batched kernel (0:
                       one, its gathers pipelined through shared memory)

Each candidate is timed with the library's own kernel benchmarks (CUDA
events, L2 flushed between launches), weighted as one CG iteration uses the
launches: two hop + inverse-diagonal launches and two hop + Schur-combine
launches.  The winners are cached per (device, volume, precision, number of
right-hand sides) in a JSON file, so a serving process pays for tuning once
per volume.
"""
from __future__ import annotations

import json
import os
import threading

HOP_SHAPES = {"double": (0, 1, 2), "single": (0, 1, 2, 3, 4, 5, 6, 7), "half": (0, 1, 2, 3, 4, 5, 6, 7)}
MRHS_CHOICES = (0, 1, 2, 4)  # 0: one right-hand side per thread, gathers pipelined through shared memory

_lock = threading.Lock()


def default_cache_path() -> str:
    base = os.environ.get("XDG_CACHE_HOME") or os.path.join(os.path.expanduser("~"), ".cache")
    return os.path.join(base, "nissa_b200", "tune.json")


def _key(device_name: str, dims, precision: str, nrhs: int) -> str:
    return "%s|%s|%s|%d" % (device_name, "x".join(str(d) for d in dims), precision, nrhs)


def _load(path):
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(path, table):
    d = os.path.dirname(path)
    if d:
        os.makedirs(d, exist_ok=True)
    tmp = path + ".tmp%d" % os.getpid()
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def iteration_cost(bench, precision: str, nrep: int = 10) -> float:
    """Device milliseconds of the four hopping launches of one CG iteration."""
    t1, _ = bench(precision, variant=1, nrep=nrep, flush=True)
    t2, _ = bench(precision, variant=2, nrep=nrep, flush=True)
    return 2.0 * t1 + 2.0 * t2


def tune_single(lat, precision: str, nrep: int = 10) -> dict:
    """Pick the hopping launch shape (and, for FP32 spinors, the link format)
    that minimises one CG iteration; applies it and returns the settings."""
    best = None
    link_opts = (0, 1) if precision == "single" else (None,)
    for links in link_opts:
        if links is not None:
            lat.set_tuning("links_single", links)
        for shape in HOP_SHAPES[precision]:
            lat.set_tuning("hop_cfg_" + precision, shape)
            ms = iteration_cost(lat.bench_hop, precision, nrep)
            if best is None or ms < best[0]:
                best = (ms, shape, links)
    ms, shape, links = best
    settings = {"hop_cfg_" + precision: shape}
    if links is not None:
        settings["links_single"] = links
    apply(lat, settings)
    return {"settings": settings, "ms_per_iteration": ms}


def tune_batched(lat, precision: str, nrhs: int, nrep: int = 5) -> dict:
    """Pick the right-hand sides per thread of the batched kernel for nrhs."""
    best = None
    for r in MRHS_CHOICES:
        if precision == "double" and (r > 2 or r == 0):
            continue
        lat.set_tuning("mrhs_per_thread", r)
        ms, _ = lat.bench_hop_batched(precision, nrhs=nrhs, nrep=nrep, flush=True)
        if best is None or ms < best[0]:
            best = (ms, r)
    settings = {"mrhs_per_thread": best[1]}
    apply(lat, settings)
    return {"settings": settings, "ms_per_launch": best[0]}


def apply(lat, settings: dict) -> None:
    for k, v in settings.items():
        lat.set_tuning(k, v)


def autotune(lat, precision: str, nrhs: int = 1, device_name: str | None = None, cache: str | None = None,
             retune: bool = False) -> dict:
    """Tune `lat` (a Lattice with its conf uploaded) for solves in `precision`
    with `nrhs` right-hand sides per launch, through the cache."""
    if device_name is None:
        import torch
        device_name = torch.cuda.get_device_name(lat.device)
    path = cache or default_cache_path()
    key = _key(device_name, (lat.T, lat.LX, lat.LY, lat.LZ), precision, nrhs)
    with _lock:
        table = _load(path)
        if not retune and key in table:
            apply(lat, table[key]["settings"])
            return dict(table[key], cached=True)
    res = tune_batched(lat, precision, nrhs) if nrhs > 1 else tune_single(lat, precision)
    with _lock:
        table = _load(path)
        table[key] = res
        _store(path, table)
    return dict(res, cached=False)
