"""Autotuning of the launch choices of one lattice on one GPU.

The choices (all results-neutral: every choice computes the same operator and
solver) are the tuning knobs of the C ABI (tms_set_tuning):

  hop_cfg_<precision>  launch shape of the e/o hopping kernel (one or two
                       sites per thread, register caps, packed FP32 spin rows,
                       gathers streamed through shared memory by cp.async,
                       row tiles staged by bulk copies)
  tma_rows             the site tiling of the staged shape: lattice rows of
                       LZ/2 sites per CTA tile (a CTA owns R rows of one
                       (t, x) plane and stages their faces); searched with
                       that shape, on volumes where it applies
  links_single         FP32 or 16-bit links under the FP32 inner solver
  mrhs_per_thread      right-hand sides per thread of the batched kernel (0:
                       one, its gathers pipelined through shared memory)

Each candidate is timed with the library's own kernel benchmarks (CUDA
events, L2 flushed between launches), weighted as one CG iteration uses the
launches: two hop + inverse-diagonal launches and two hop + Schur-combine
launches.  The winners are cached per (device, volume, precision, number of
right-hand sides) in a JSON file, so a serving process pays for tuning once
per volume.  Beside each winner the cache keeps the evidence: every
candidate's device time and algorithmic bandwidth, and the DRAM bandwidth of
an ncu capture of the winning kernel once one is recorded (record_capture).
"""
from __future__ import annotations

import json
import os
import threading

HOP_SHAPES = {"double": (0, 1, 2), "single": (0, 1, 2, 3, 4, 5, 6, 7), "half": (0, 1, 2, 3, 4, 5, 6, 7)}
TILED_SHAPE = 7      # the shape whose CTAs own row tiles (tma_rows)
TILE_THREADS = 128   # sites a tile may hold
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


def tile_rows_choices(LY: int, LZ: int) -> list:
    """Row counts R the staged shape can tile a (t, x) plane with (tma_rows):
    R divides LY, R*LZ/2 sites fit a tile, and a partial plane leaves room for
    its two halo rows and holds at least 16 sites.  Empty when the shape does
    not apply (LZ not a multiple of 8 or above 128)."""
    h = LZ // 2
    if LZ % 8 or h > 64:
        return []
    return [R for R in range(1, LY + 1)
            if LY % R == 0 and R * h <= TILE_THREADS and (R == LY or (R + 2 <= LY and R * h >= 16))]


def iteration_cost(bench, precision: str, nrep: int = 10):
    """Device milliseconds of the four hopping launches of one CG iteration,
    and their algorithmic bytes."""
    t1, b1 = bench(precision, variant=1, nrep=nrep, flush=True)
    t2, b2 = bench(precision, variant=2, nrep=nrep, flush=True)
    return 2.0 * t1 + 2.0 * t2, 2.0 * b1 + 2.0 * b2


def _gbs(nbytes, ms):
    return nbytes / (ms * 1e-3) / 1e9 if ms > 0 else 0.0


def tune_single(lat, precision: str, nrep: int = 10) -> dict:
    """Pick the hopping launch shape (its site tiling for the staged shape and,
    for FP32 spinors, the link format) that minimises one CG iteration;
    applies it and returns the settings with every candidate's timing."""
    candidates = []
    link_opts = (0, 1) if precision == "single" else (None,)
    rows_opts = tile_rows_choices(lat.LY, lat.LZ)
    for links in link_opts:
        if links is not None:
            lat.set_tuning("links_single", links)
        for shape in HOP_SHAPES[precision]:
            lat.set_tuning("hop_cfg_" + precision, shape)
            for rows in (rows_opts if shape == TILED_SHAPE and rows_opts else [None]):
                if rows is not None:
                    lat.set_tuning("tma_rows", rows)
                ms, nbytes = iteration_cost(lat.bench_hop, precision, nrep)
                c = {"hop_cfg": shape, "ms_per_iteration": ms, "alg_gbs": _gbs(nbytes, ms)}
                if links is not None:
                    c["links_single"] = links
                if rows is not None:
                    c["tma_rows"] = rows
                candidates.append(c)
    best = min(candidates, key=lambda c: c["ms_per_iteration"])
    settings = {"hop_cfg_" + precision: best["hop_cfg"]}
    if "links_single" in best:
        settings["links_single"] = best["links_single"]
    if rows_opts and precision != "double":
        settings["tma_rows"] = best.get("tma_rows", 0)
    apply(lat, settings)
    return {"settings": settings, "ms_per_iteration": best["ms_per_iteration"], "alg_gbs": best["alg_gbs"],
            "candidates": candidates}


def tune_batched(lat, precision: str, nrhs: int, nrep: int = 5) -> dict:
    """Pick the right-hand sides per thread of the batched kernel for nrhs."""
    candidates = []
    for r in MRHS_CHOICES:
        if precision == "double" and (r > 2 or r == 0):
            continue
        lat.set_tuning("mrhs_per_thread", r)
        ms, nbytes = lat.bench_hop_batched(precision, nrhs=nrhs, nrep=nrep, flush=True)
        candidates.append({"mrhs_per_thread": r, "ms_per_launch": ms, "alg_gbs": _gbs(nbytes, ms)})
    best = min(candidates, key=lambda c: c["ms_per_launch"])
    settings = {"mrhs_per_thread": best["mrhs_per_thread"]}
    apply(lat, settings)
    return {"settings": settings, "ms_per_launch": best["ms_per_launch"], "alg_gbs": best["alg_gbs"],
            "candidates": candidates}


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


def record_capture(dims, precision: str, dram_bytes: float, seconds: float, nrhs: int = 1,
                   device_name: str | None = None, cache: str | None = None, source: str = "") -> dict:
    """Store beside a cached winner the DRAM traffic of an ncu capture of its
    hopping kernel (dram__bytes_read.sum + dram__bytes_write.sum of one launch,
    and that launch's gpu__time_duration): the entry gains
    {"ncu": {"dram_bytes", "seconds", "dram_gbs", "source"}}.  dims = (T, LX, LY, LZ)."""
    if device_name is None:
        import torch
        device_name = torch.cuda.get_device_name(0)
    path = cache or default_cache_path()
    key = _key(device_name, dims, precision, nrhs)
    with _lock:
        table = _load(path)
        if key not in table:
            raise KeyError("no tuned entry %s" % key)
        table[key]["ncu"] = {"dram_bytes": float(dram_bytes), "seconds": float(seconds),
                             "dram_gbs": _gbs(float(dram_bytes), float(seconds) * 1e3), "source": source}
        _store(path, table)
        return table[key]
