"""Benchmark: twisted-mass e/o CG solves per second on one B200 (or N replicas).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one full solve D_tm psi = eta through the e/o
preconditioned CG, the reference's inv_tmD_cg_eoprec): 32^3 x 64 lattice,
gauge links U = exp(i eps H) with eps = 0.35 (seeded), antiperiodic time,
kappa = 0.1610, mu = 0.005, point sources at the origin cycling over the 12
spin-colour columns, stopped at |r|/|b| <= 1e-10 (squared residue 1e-20), in
mixed precision: FP16 inner CG (half spinors with a per-site FP32 scale,
16-bit fixed-point 12-real links) with FP64 reliable updates, the final true
residual checked in FP64 (--precision single|double selects the others).

Printed JSON line (rank 0): value = solves/s with the inputs resident in HBM
(device timing, CUDA events, max over ranks); e2e = the same columns through
the C ABI (tms_cg_eoprec_columns) from pinned host buffers, every column's
host<->device copies inside the timed region (overlapping the neighbouring
columns' solves);
roofline = the inner solver's hopping kernel (hop + inverse diagonal, the first
half of K) timed alone with CUDA events, L2 flushed between launches; fp64 = the
plain FP64 GPU CG on the same solves and the FP64 e/o Dslash bandwidth;
variants = the other inner precisions on the same solves; cpu_baseline = one
whole solve of the reference's own OpenMP code (oracle/_ref) on the same conf,
whose solution is also the yardstick of accuracy.rel_err_vs_reference.
--impl reference times one whole reference solve per step.

The same line carries, as sub-objects (rank 0, N = 1), the other
configurations of the workload: configs_8c16 (plain FP64 CG, 8^3x16) and
configs_16c32 (12 columns, FP32 inner with 12-real links, 16^3x32), each with
the reference's own CPU solve timed and compared; batched_48 (48 right-hand
sides at 24^3x48); cgm_32c64 (8-shift multi-mass CG, 3 sources, 32^3x64); serve
(three resident volumes under Poisson load: p50/p99 latency at a stated rate).

N > 1 GPUs run independent replicas (one gauge copy per GPU, each rank solving
its own columns): the path needs no collective, scaling is weak.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(name="tm e/o CG solve, 32^3x64, mixed %s-inner/FP64-reliable, |r|/|b|<=1e-10",
                T=64, L=32, eps=0.35, seed=1, kappa=0.1610, mu=0.005, residue=1e-20, bc_t=-1.0)
PREC_NAME = {"double": "FP64", "single": "FP32", "half": "FP16"}
PREC_DTYPE = {"double": "f64", "single": "f32 inner / f64 reliable updates",
              "half": "f16 storage, f32 arithmetic inner / f64 reliable updates"}
METRIC = "CG solves/s & Dslash HBM GB/s, 32³×64 mixed vs FP64 @1e-10; p50/p99 serve"
UNIT = "solves/s"
HOP_KERNEL = {"half": "hopping kernel of the FP16 inner solver (16-bit 12-real links) + inverse diagonal, "
                      "the first half of K (the library's launch shape for FP16 spinors)",
              "single": "hopping kernel of the FP32 inner solver (16-bit 12-real links) + inverse diagonal, "
                        "the first half of K (the library's launch shape for FP32 spinors)"}
# DRAM bytes of one launch of that kernel on this workload: read from the ncu
# summary of the current kernel under profiles/ (its "dram bytes per launch" line)
# ncu captures of the inner hop on this workload, by (precision, launch shape)
HOP_PROFILE = {("half", 6): "hop_kernel_fp16_pipelined_32c64.md",
               ("half-fp16-arithmetic", 6): "hop_kernel_fp16_arith_32c64.md"}


def hop_traffic(prec, shape):
    """(bytes, source) of the ncu capture of the inner hop, or (None, why)."""
    import re
    name = HOP_PROFILE.get((prec, shape))
    if not name:
        return None, "no ncu capture of launch shape %d of this kernel" % shape
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            m = re.search(r"dram bytes per launch:\s*([0-9.e+]+)", f.read())
        return (float(m.group(1)), "profiles/" + name) if m else (None, "profiles/%s has no traffic line" % name)
    except OSError:
        return None, "profiles/%s absent" % name


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()

    def summary(self):
        try:
            rows = [l.split(",") for l in open(self.f.name).read().strip().splitlines() if l.strip()]
        except Exception:
            rows = []
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if len(r) > 5 + i and "Active" in r[5 + i]
                          and "Not" not in r[5 + i]})
        loaded = [s for s in sm if smax and s > 0.5 * max(smax)] or sm
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def reference_solves(conf_bc, T, L, kappa, mu, residue, reps, threads):
    """The reference's own full solve inv_tmD_cg_eoprec (oracle/_ref, its
    unmodified OpenMP code) run `reps` times in one process on the host cores,
    repetition r solving the point-source column r mod 12.  Returns (the last
    repetition's solution, seconds of every repetition, threads, kind); falls
    back to the oracle restatement (kind "port") when the reference build is
    absent."""
    import oracle
    V = T * L ** 3
    if oracle.ref_available():
        sol, rec, _ = oracle.run_ref("cgfull", T, L, {"conf": conf_bc}, (V, 4, 3, 2), kappa=kappa, mu=mu,
                                     niter=100000, residue=residue, reps=reps, point_cols=12, threads=threads)
        return sol, rec["seconds_each"], rec.get("threads", threads), "reference"
    from nissa_b200 import workload as wl
    geo = oracle.Geom(T, L)
    os.environ["OMP_NUM_THREADS"] = str(threads)
    secs, sol = [], None
    for r in range(reps):
        src = wl.point_source(T, L, spin=(r % 12) // 3, col=r % 3)
        t0 = time.perf_counter()
        sol, _, _ = geo.cg_full(conf_bc, kappa, mu, src, 100000, residue)
        secs.append(time.perf_counter() - t0)
    return sol, secs, threads, "port"


def run_reference_arm(args):
    """--impl reference: the reference's own OpenMP full solve on the host
    cores, one whole inv_tmD_cg_eoprec per step (FP64 to the same residue), on
    the same conf, sources and parameters as the GPU arm."""
    ws, rank, _ = dist_setup()
    if rank != 0:
        return
    from nissa_b200 import workload as wl
    W = WORKLOAD
    T, L = W["T"], W["L"]
    threads = os.cpu_count() or 1
    conf = wl.apply_time_bc(wl.gauge_conf(T, L, W["eps"], W["seed"]), T, L, W["bc_t"])
    _, secs, cores, kind = reference_solves(conf, T, L, W["kappa"], W["mu"], W["residue"],
                                            args.warmup + args.steps, threads)
    timed = secs[args.warmup:]
    v = len(timed) / sum(timed)
    sample = ("%s inv_tmD_cg_eoprec on %d^3x%d, FP64 to |r|/|b| <= 1e-10, one whole solve per step (%d warm-up + "
              "%d timed, point-source columns cycled as in the GPU arm), %.2f-%.2f s per solve"
              % ("the reference's own" if kind == "reference" else "the oracle's restatement of", L, T, args.warmup,
                 args.steps, min(timed), max(timed)))
    print(json.dumps({"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws,
                      "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / v,
                      "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                      "data": "synthetic (seeded gauge recipe U=exp(i eps H), point sources)",
                      "config": {"workload": W["name"].split(", mixed")[0] + ", FP64 on the host cores, |r|/|b|<=1e-10",
                                 "T": T, "L": L, "kappa": W["kappa"], "mu": W["mu"], "eps": W["eps"],
                                 "residue_sq": W["residue"], "sources": "12 point spin-colour columns at the origin, "
                                                                     "cycled"},
                      "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
                      "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
          flush=True)


def run_ours(args):
    import torch
    import torch.distributed as dist
    from nissa_b200 import Lattice
    from nissa_b200 import workload as wl

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = "cuda:%d" % local
    if ws > 1:
        dist.init_process_group("nccl", device_id=torch.device(dev), timeout=__import__("datetime").timedelta(
            seconds=600))
    W = WORKLOAD
    T, L = W["T"], W["L"]
    V = T * L ** 3
    kappa, mu, residue = W["kappa"], W["mu"], W["residue"]

    t0 = time.perf_counter()
    conf = wl.gauge_conf(T, L, W["eps"], W["seed"], device=dev)
    log("rank %d: gauge conf %.1fs" % (rank, time.perf_counter() - t0))
    lat = Lattice(T, L, bc_t=W["bc_t"], device=local)
    lat.upload_conf(conf)
    assert lat.conf_is_su3
    tuning = headline_tuning(lat, args)
    plaquette = lat.plaquette()  # global_plaquette_lx_conf of the periodic links, on the device

    def column(k):
        s = torch.zeros((V, 4, 3, 2), dtype=torch.float64, device=dev)
        s[0, (k // 3) % 4, k % 3, 0] = 1.0
        return s

    from nissa_b200 import replicas
    ncol = min(12, args.steps)
    cols = [column(c) for c in replicas.rank_columns(rank, args.steps)[:ncol]]
    sol = torch.empty((V, 4, 3, 2), dtype=torch.float64, device=dev)

    prec = args.precision

    def solve(k, precision=prec, src=None, out=None):
        s = cols[k % ncol] if src is None else src
        return lat.inv_tmD_cg_eoprec(kappa, mu, s, 100000, residue, precision=precision,
                                     out=sol if out is None else out)[1]

    for k in range(args.warmup):
        solve(k)

    def barrier():
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # --- timed region: device-resident inputs -------------------------------------------
    stats = []
    barrier()
    l0 = lat.launch_count
    with ClockSampler(local) as clk:
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for k in range(args.steps):
            stats.append(solve(k))
        e1.record()
        barrier()
    launches = lat.launch_count - l0
    ms_max = replicas.max_over_ranks(e0.elapsed_time(e1))
    value = replicas.whole_job_rate(args.steps, ms_max, ws)
    clocks = clk.summary()

    # --- roofline: the inner solver's hopping kernel, and the FP64 Dslash, timed right after ----
    # --- the timed region (same clocks and power state) --------------------------------------
    peak, peak_kind = peaks()
    hop_prec = prec if prec != "double" else "single"
    hop_ms, hop_bytes = lat.bench_hop(hop_prec, variant=1, nrep=30, flush=True)
    d64_ms, d64_bytes = lat.bench_hop("double", variant=0, nrep=30, flush=True)
    achieved = hop_bytes / (hop_ms * 1e-3) / 1e9
    d64_gbs = d64_bytes / (d64_ms * 1e-3) / 1e9
    traffic, traffic_src = hop_traffic(hop_prec, lat.get_tuning("hop_cfg_" + hop_prec))
    hop_kernel_desc = HOP_KERNEL[hop_prec]
    if args.half_arith and hop_prec == "half":
        hop_kernel_desc = ("pipelined hopping kernel of the FP16 inner solver in FP16 arithmetic (FP16 12-real "
                           "links) + inverse diagonal, the first half of K")
        traffic, traffic_src = hop_traffic("half-fp16-arithmetic", 6)  # its only launch shape

    # --- e2e: the same columns through the C ABI from pinned host buffers -------------------
    # (tms_cg_eoprec_columns: every column's source is copied in and its solution out inside
    # the timed region, the copies of the neighbouring columns overlapping each solve)
    host_src = [torch.zeros((V, 4, 3, 2), dtype=torch.float64).pin_memory() for _ in range(ncol)]
    for k in range(ncol):
        host_src[k].copy_(cols[k].cpu())
    host_sol = [torch.empty((V, 4, 3, 2), dtype=torch.float64).pin_memory() for _ in range(2)]
    # the columns twice: the first column's copy in and the last one's copy out,
    # which nothing overlaps, weigh on 24 solves instead of 12
    e2e_steps = 2 * ncol
    e2e_src = [host_src[k % ncol] for k in range(e2e_steps)]
    e2e_out = [host_sol[k % 2] for k in range(e2e_steps)]
    lat.inv_tmD_cg_eoprec_columns(kappa, mu, e2e_src[:2], 100000, residue, precision=prec,
                                  out=e2e_out[:2])  # warm the host path
    barrier()
    h0 = time.perf_counter()
    _, e2e_stats = lat.inv_tmD_cg_eoprec_columns(kappa, mu, e2e_src, 100000, residue, precision=prec, out=e2e_out)
    barrier()
    e2e_value = replicas.whole_job_rate(e2e_steps, replicas.max_over_ranks((time.perf_counter() - h0) * 1e3), ws)
    assert max(x["lx_rel_res2"] for x in e2e_stats) < 10 * residue
    bytes_per = V * 24 * 8

    # --- plain FP64 GPU CG on the same solves, and the accuracy of the mixed solutions -------
    # (6 columns back to back, CUDA events around the loop as in the timed region; then each
    # column's mixed solution against its FP64 one)
    fp64_steps = min(6, ncol)
    refs = [torch.empty_like(sol) for _ in range(fp64_steps)]
    barrier()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    fp64_stats = [solve(k, precision="double", out=refs[k]) for k in range(fp64_steps)]
    f1.record()
    barrier()
    fp64_sec = replicas.max_over_ranks(f0.elapsed_time(f1)) * 1e-3 / fp64_steps
    errs = []
    for k in range(fp64_steps):
        solve(k, out=sol)
        errs.append(float(torch.linalg.norm(sol - refs[k]) / torch.linalg.norm(refs[k])))
    ref = refs[0]
    del refs[1:]
    accuracy_vs_ref = {}
    mixed_sec = ms_max * 1e-3 / args.steps

    # --- the 12 columns as one batched solve (one pass over the links per operator step) ----
    cols12 = [column(c) for c in range(12)]
    outs12 = [torch.empty_like(sol) for _ in range(12)]
    mus12 = [mu] * 12
    lat.inv_tmD_cg_eoprec_batched(kappa, mus12, cols12, 100000, residue, precision=prec, out=outs12)
    barrier()
    b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b0.record()
    st12 = lat.inv_tmD_cg_eoprec_batched(kappa, mus12, cols12, 100000, residue, precision=prec, out=outs12)[1]
    b1.record()
    barrier()
    batched = {"solves_per_s": replicas.whole_job_rate(12, replicas.max_over_ranks(b0.elapsed_time(b1)), ws),
               "rhs": 12, "iterations_max": max(x["iterations"] for x in st12),
               "true_rel_res2_max": max(x["true_rel_res2"] for x in st12)}
    del cols12, outs12

    # --- the other inner precisions on the same solves (solver-reported device seconds) -----
    variants = {}
    for name, vp, links16 in (("single_links32", "single", 0), ("single", "single", 1), ("half", "half", 1),
                              ("half_fp16_arithmetic", "half", 1)):
        if vp == prec and (links16 or vp == "half") and name != "half_fp16_arithmetic":
            continue
        lat.set_tuning("links_single", links16)
        lat.set_tuning("half_arith", 1 if name == "half_fp16_arithmetic" else 0)
        # FP16 arithmetic drifts faster between reliable updates: recompute at a 0.01 drop
        lat.set_tuning("reliable_delta_half", 0.01 if name == "half_fp16_arithmetic" else 0.005)
        solve(0, precision=vp)
        vs = [solve(k, precision=vp) for k in range(2)]
        variants[name] = {"solves_per_s": 1.0 / statistics.mean(x["seconds"] for x in vs),
                          "iterations": vs[0]["iterations"], "reliable_updates": vs[0]["reliable_updates"],
                          "true_rel_res2_max": max(x["true_rel_res2"] for x in vs)}
        if name == "half_fp16_arithmetic":
            # against the FP32-arithmetic FP16 solver timed the same way, and column 0 against FP64
            solve(0, out=sol)
            variants[name]["rel_err_vs_fp64"] = float(torch.linalg.norm(sol - ref) / torch.linalg.norm(ref))
            lat.set_tuning("half_arith", 0)
            lat.set_tuning("reliable_delta_half", 0.005)
            base = [solve(k, precision=vp) for k in range(2)]
            variants[name]["speedup_vs_fp32_arithmetic"] = (statistics.mean(x["seconds"] for x in base) /
                                                            statistics.mean(x["seconds"] for x in vs))
    # back to the headline's own settings
    lat.set_tuning("links_single", 1)
    lat.set_tuning("half_arith", 1 if args.half_arith else 0)
    lat.set_tuning("reliable_delta_half", 0.01 if args.half_arith else 0.005)

    # --- CPU baseline: one whole reference solve of column 0 (rank 0, N=1 only), and the -------
    # --- headline solution's error against it -------------------------------------------------
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        try:
            conf_bc = wl.apply_time_bc(conf, T, L, W["bc_t"])
            ref_sol, secs, cores, kind = reference_solves(conf_bc, T, L, kappa, mu, residue, 1, os.cpu_count() or 1)
            cpu = {"value": 1.0 / secs[0], "unit": UNIT, "cores": cores, "kind": kind,
                   "sample": "%s inv_tmD_cg_eoprec, one whole FP64 solve of point column 0 on the same 32^3x64 conf "
                             "to |r|/|b| <= 1e-10: %.2f s" % ("the reference's own" if kind == "reference" else
                                                              "the oracle's restatement of", secs[0])}
            ref_d = torch.from_numpy(ref_sol).to(dev)
            solve(0, out=sol)
            solve(0, precision="double", out=ref)
            nref = torch.linalg.norm(ref_d)
            accuracy_vs_ref = {"rel_err_vs_reference": float(torch.linalg.norm(sol - ref_d) / nref),
                               "fp64_rel_err_vs_reference": float(torch.linalg.norm(ref - ref_d) / nref),
                               "reference_column": 0, "reference_kind": kind}
            del ref_d
            # the reference's FP64 e/o Dslash on the same conf (3 repetitions), same bytes model
            import oracle
            if oracle.ref_available():
                x = np.random.default_rng(6).standard_normal((V // 2, 4, 3, 2))
                _, rec, _ = oracle.run_ref("hop", T, L, {"conf": conf_bc, "in": x}, (V // 2, 4, 3, 2), par=1, reps=3,
                                           threads=cores)
                cpu["dslash_gbs"] = d64_bytes / rec["seconds_per_rep"] / 1e9
        except Exception as e:  # the CPU baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "unavailable", "sample": str(e)}

    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return

    # --- the other configurations, as sub-objects of this line (rank 0, N=1) ---------------------
    legs = {}
    if ws == 1 and not args.no_legs:
        lat.close()
        del cols, sol, ref
        torch.cuda.empty_cache()
        for name, fn in (("configs", leg_configs), ("batched_48", leg_batched), ("cgm_32c64", leg_cgm),
                         ("serve", leg_serve)):
            t0 = time.perf_counter()
            try:
                r = fn(args)
            except Exception as e:  # a leg is reported, never required for the headline
                r = {"error": "%s: %s" % (type(e).__name__, e)}
            if name == "configs" and "results" in r:
                for k, v in r["results"].items():
                    legs["configs_8c16" if k.startswith("8^3") else "configs_16c32"] = dict(v, config=k)
            else:
                legs[name] = r
            log("leg %s: %.1f s" % (name, time.perf_counter() - t0))
            torch.cuda.empty_cache()

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": PREC_DTYPE[prec] if not args.half_arith else
                 "f16 storage, f16 arithmetic hop with f32 accumulation inner / f64 reliable updates",
        "data": "synthetic (seeded gauge recipe U=exp(i eps H), point sources)",
        "config": {"workload": W["name"], "T": T, "L": L, "kappa": kappa, "mu": mu, "eps": W["eps"],
                   "residue_sq": residue, "plaquette": plaquette,
                   "sources": "12 point spin-colour columns at the origin, cycled",
                   "inner_precision": prec,
                   "l2": "working set (links 0.2-0.4 GB + spinors) larger than the 126 MB L2",
                   "parallelism": "replicas" if ws > 1 else "1 GPU"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": bytes_per, "d2h_bytes_per_step": bytes_per,
                "steps": e2e_steps},
        "roofline": {"bound": "hbm", "kernel": hop_kernel_desc,
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_kind": peak_kind, "traffic": traffic,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch of this "
                                       "kernel on this workload (%s)" % traffic_src,
                     "ms_per_launch": hop_ms, "alg_bytes_per_launch": hop_bytes},
        "tuning": tuning,
        "variants": variants,
        "batched_12_columns": batched,
        "fp64": {"solves_per_s": 1.0 / fp64_sec, "iterations": fp64_stats[0]["iterations"],
                 "solves_timed": fp64_steps, "mixed_speedup_vs_fp64": fp64_sec / mixed_sec,
                 "dslash_gbs": d64_gbs, "dslash_frac": d64_gbs / peak, "dslash_ms": d64_ms},
        "accuracy": {"mixed_rel_err_vs_fp64": max(errs), **accuracy_vs_ref,
                     "true_rel_res2_max": max(s["true_rel_res2"] for s in stats),
                     "lx_rel_res2_max": max(s["lx_rel_res2"] for s in stats)},
        "solver": {"iterations_mean": statistics.mean(s["iterations"] for s in stats),
                   "reliable_updates_mean": statistics.mean(s["reliable_updates"] for s in stats)},
        "gpu_launches": int(launches),
        "clocks": clocks,
        "cpu_baseline": cpu,
    }
    line.update(legs)
    print(json.dumps(line), flush=True)


def headline_tuning(lat, args):
    """The launch choices of the headline solve: the autotuner's (timed on this
    lattice, cached per device and volume), or --hop-cfg / --tma-rows as given;
    with --half-arith the FP16 inner hop in FP16 arithmetic (opt-in)."""
    prec = args.precision
    if args.hop_cfg >= 0:
        lat.set_tuning("hop_cfg_" + prec, args.hop_cfg)
        if args.tma_rows >= 0:
            lat.set_tuning("tma_rows", args.tma_rows)
        settings = {"hop_cfg_" + prec: args.hop_cfg}
        if args.tma_rows >= 0:
            settings["tma_rows"] = args.tma_rows
        if args.half_arith:
            lat.set_tuning("half_arith", 1)
            lat.set_tuning("reliable_delta_half", 0.01)
            settings.update(half_arith=1, reliable_delta_half=0.01)
        return {"source": "command line", "settings": settings}
    from nissa_b200 import tune
    t0 = time.perf_counter()
    r = tune.autotune(lat, prec)
    out = {"source": "autotuner (cached)" if r["cached"] else "autotuner", "settings": r["settings"],
           "ms_per_iteration": r["ms_per_iteration"], "alg_gbs": r["alg_gbs"],
           "tuning_s": time.perf_counter() - t0,
           "candidates": [{k: (round(v, 5) if isinstance(v, float) else v) for k, v in c.items()}
                          for c in r["candidates"]]}
    log("tuned: %s (%.1f s)" % (r["settings"], out["tuning_s"]))
    if args.half_arith:
        # after tuning: the FP16-arithmetic hop has one launch shape
        lat.set_tuning("half_arith", 1)
        lat.set_tuning("reliable_delta_half", 0.01)
        out["settings"] = dict(out["settings"], half_arith=1, reliable_delta_half=0.01)
    return out


TUNE_VOLUMES = [(16, 8), (32, 16), (48, 24), (64, 32)]


def leg_tune(args):
    """The autotuner's choice per volume (FP16 and FP32 inner hops, and the
    12-RHS batched kernel): every candidate's device time and algorithmic
    bandwidth, timed here into a fresh cache."""
    import tempfile
    from nissa_b200 import Lattice, tune
    from nissa_b200 import workload as wl
    out = {}
    cache = os.path.join(tempfile.mkdtemp(), "tune.json")
    for T, L in TUNE_VOLUMES:
        conf = wl.gauge_conf(T, L, 0.35, 1, device="cuda:0")
        with Lattice(T, L, bc_t=-1.0) as lat:
            lat.upload_conf(conf)
            name = "%d^3x%d" % (L, T)
            out[name] = {p: tune.autotune(lat, p, cache=cache, retune=True) for p in ("half", "single")}
            out[name]["half_batched_12"] = tune.autotune(lat, "half", nrhs=12, cache=cache, retune=True)
        del conf
        log("tuned %s" % name)
    return {"workload": "autotuner per volume", "volumes": out}


def run_kernel_only(args):
    """Profiling entry point: set up the workload's lattice and launch the e/o
    hopping kernel of one precision `nrep` times (L2 flushed between launches)."""
    import torch
    from nissa_b200 import Lattice
    from nissa_b200 import workload as wl
    W = WORKLOAD
    conf = wl.gauge_conf(W["T"], W["L"], W["eps"], W["seed"], device="cuda:0")
    lat = Lattice(W["T"], W["L"], bc_t=W["bc_t"])
    lat.upload_conf(conf)
    if args.hop_cfg >= 0:
        lat.set_tuning("hop_cfg_" + args.kernel_only, args.hop_cfg)
    if args.tma_rows >= 0:
        lat.set_tuning("tma_rows", args.tma_rows)
    if args.half_arith:
        lat.set_tuning("half_arith", 1)
    if args.nrhs > 1:
        if args.mrhs:
            lat.set_tuning("mrhs_per_thread", args.mrhs)
        ms, by = lat.bench_hop_batched(args.kernel_only, nrhs=args.nrhs, nrep=args.nrep, flush=True)
    else:
        ms, by = lat.bench_hop(args.kernel_only, variant=args.variant, nrep=args.nrep, flush=True)
    torch.cuda.synchronize()
    print(json.dumps({"kernel": "hop", "precision": args.kernel_only, "variant": args.variant, "nrhs": args.nrhs,
                      "hop_cfg": lat.get_tuning("hop_cfg_" + args.kernel_only),
                      "tma_rows": lat.get_tuning("tma_rows"), "T": W["T"],
                      "L": W["L"], "ms_per_launch": ms, "alg_bytes_per_launch": by,
                      "achieved_gbs": by / (ms * 1e-3) / 1e9}), flush=True)


CGM_WORKLOAD = dict(name="tm Q^2 multi-shift CGM, 32^3x64, 8 masses log-spaced in [0.002, 0.2], 3 Z2 sources",
                    T=64, L=32, eps=0.35, seed=1, kappa=0.1632, masses=list(np.geomspace(0.002, 0.2, 8)),
                    residue=1e-20, bc_t=-1.0)


def leg_cgm(args):
    """The multi-shift workload (one step = one source solved for all 8 masses:
    FP32 multi-shift to |r|/|b| ~ 1e-6, then per shift a defect correction
    through the mixed-precision e/o solver, every shift to |r|/|b| <= 1e-10
    checked in FP64), against the FP64 multi-shift CG on the same sources."""
    import torch
    from nissa_b200 import Lattice
    from nissa_b200 import workload as wl
    W = dict(CGM_WORKLOAD)
    if args.lattice:
        W["T"], W["L"] = (int(x) for x in args.lattice.split(","))
    T, L = W["T"], W["L"]
    V = T * L ** 3
    conf = wl.gauge_conf(T, L, W["eps"], W["seed"], device="cuda:0")
    lat = Lattice(T, L, bc_t=W["bc_t"])
    lat.upload_conf(conf)
    srcs = [torch.from_numpy(wl.z2_source(T, L, 100 + c, col=c)).cuda() for c in range(3)]
    outs = [torch.empty((V, 4, 3, 2), dtype=torch.float64, device="cuda") for _ in W["masses"]]
    res = {}
    for prec in (args.cgm_precision, "double"):
        lat.inv_tmQ2_cgm(W["kappa"], W["masses"], srcs[0], 100000, W["residue"], precision=prec, out=outs)  # warm
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        stats = []
        for c in range(3):
            _, st = lat.inv_tmQ2_cgm(W["kappa"], W["masses"], srcs[c], 100000, W["residue"], precision=prec,
                                     out=outs)
            stats.append(st)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        res[prec] = {"sources_per_s": 3 / dt, "s_per_source": dt / 3,
                     "iterations": [s["iterations"] for s in stats[0]],
                     "true_rel_res2_max": max(x["true_rel_res2"] for st in stats for x in st)}
    lat.close()
    return {"workload": W["name"].replace("32^3x64", "%d^3x%d" % (L, T)), "kappa": W["kappa"],
            "masses": W["masses"], "residue_sq": W["residue"], "mixed": res[args.cgm_precision],
            "fp64": res["double"],
            "mixed_speedup_vs_fp64": res["double"]["s_per_source"] / res[args.cgm_precision]["s_per_source"]}


BATCH_WORKLOAD = dict(name="48-RHS batched e/o CG, 24^3x48: 12 spin-colour-diluted Z2 sources x mu in "
                           "{+0.003, -0.003, +0.006, -0.006}, mixed %s-inner/FP64-reliable, |r|/|b|<=1e-10",
                      T=48, L=24, eps=0.35, seed=3, kappa=0.1610, mus=[0.003, -0.003, 0.006, -0.006], residue=1e-20,
                      bc_t=-1.0)


def run_batched_once(args):
    """Profiling entry point: one batched solve of the batched workload (the
    48 right-hand sides at 24^3x48, one-RHS-per-thread pipelined kernel), no
    comparisons, for a launch list of one whole batched solve."""
    import torch
    from nissa_b200 import Lattice
    from nissa_b200 import workload as wl
    W = BATCH_WORKLOAD
    T, L = W["T"], W["L"]
    conf = wl.gauge_conf(T, L, W["eps"], W["seed"], device="cuda:0")
    lat = Lattice(T, L, bc_t=W["bc_t"])
    lat.upload_conf(conf)
    del conf
    srcs, mus = [], []
    for k in range(12):
        z = torch.from_numpy(wl.z2_source(T, L, 100 + k, spin=k // 3, col=k % 3)).to("cuda:0")
        for mu in W["mus"]:
            srcs.append(z)
            mus.append(mu)
    lat.set_tuning("mrhs_per_thread", args.mrhs)
    outs = [torch.empty_like(srcs[0]) for _ in srcs]
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    l0 = lat.launch_count
    st = lat.inv_tmD_cg_eoprec_batched(W["kappa"], mus, srcs, 100000, W["residue"], precision=args.precision,
                                       out=outs)[1]
    torch.cuda.synchronize()
    print(json.dumps({"workload": "one batched solve, 48 RHS, 24^3x48", "precision": args.precision,
                      "mrhs_per_thread": args.mrhs, "seconds_first_call": time.perf_counter() - t0,
                      "launches": lat.launch_count - l0, "iterations_max": max(x["iterations"] for x in st),
                      "reliable_updates": max(x["reliable_updates"] for x in st)}), flush=True)
    lat.close()


def leg_batched(args):
    """The batched workload: the 48 right-hand sides solved in one batched
    solve (one launch per operator step for all of them, CUDA graphs,
    autotuned kernel shapes) against the same 48 solved one at a time with
    the same precision; reports right-hand sides per second and the largest
    difference between a batched and an alone solution."""
    import torch
    from nissa_b200 import Lattice, tune
    from nissa_b200 import workload as wl
    W = BATCH_WORKLOAD
    prec = args.precision
    T, L = W["T"], W["L"]
    if args.lattice:
        T, L = (int(x) for x in args.lattice.split(","))
    dev = "cuda:0"
    conf = wl.gauge_conf(T, L, W["eps"], W["seed"], device=dev)
    lat = Lattice(T, L, bc_t=W["bc_t"])
    lat.upload_conf(conf)
    srcs, mus = [], []
    for k in range(12):
        z = torch.from_numpy(wl.z2_source(T, L, 100 + k, spin=k // 3, col=k % 3)).to(dev)
        for mu in W["mus"]:
            srcs.append(z)
            mus.append(mu)
    n = len(srcs)
    tuned_b = tune.autotune(lat, prec, nrhs=n)
    tuned_1 = tune.autotune(lat, prec, nrhs=1)
    outs = [torch.empty_like(srcs[0]) for _ in range(n)]
    alone = [torch.empty_like(srcs[0]) for _ in range(n)]
    kappa, res = W["kappa"], W["residue"]

    def batched():
        return lat.inv_tmD_cg_eoprec_batched(kappa, mus, srcs, 100000, res, precision=prec, out=outs)[1]

    batched()  # capture the graphs
    torch.cuda.synchronize()
    with ClockSampler(0) as clk:
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        st_b = batched()
        e1.record()
        torch.cuda.synchronize()
    ms_b = e0.elapsed_time(e1)
    lat.inv_tmD_cg_eoprec(kappa, mus[0], srcs[0], 100000, res, precision=prec, out=alone[0])
    torch.cuda.synchronize()
    e0.record()
    st_1 = [lat.inv_tmD_cg_eoprec(kappa, mus[i], srcs[i], 100000, res, precision=prec, out=alone[i])[1]
            for i in range(n)]
    e1.record()
    torch.cuda.synchronize()
    ms_1 = e0.elapsed_time(e1)
    diff = max(float(torch.linalg.norm(outs[i] - alone[i]) / torch.linalg.norm(alone[i])) for i in range(n))
    # the plain FP64 GPU CG on the first 8 right-hand sides, one at a time
    n64 = 8
    ref64 = torch.empty_like(srcs[0])
    lat.inv_tmD_cg_eoprec(kappa, mus[0], srcs[0], 100000, res, precision="double", out=ref64)
    torch.cuda.synchronize()
    e0.record()
    st_64 = [lat.inv_tmD_cg_eoprec(kappa, mus[i], srcs[i], 100000, res, precision="double", out=ref64)[1]
             for i in range(n64)]
    e1.record()
    torch.cuda.synchronize()
    ms_64 = e0.elapsed_time(e1) / n64
    lat.close()
    return ({"workload": (W["name"] % PREC_NAME[prec]).replace("24^3x48", "%d^3x%d" % (L, T)),
                      "rhs": n, "precision": prec,
                      "batched": {"rhs_per_s": n / (ms_b * 1e-3), "ms": ms_b,
                                  "iterations_max": max(s["iterations"] for s in st_b),
                                  "true_rel_res2_max": max(s["true_rel_res2"] for s in st_b)},
                      "one_at_a_time": {"rhs_per_s": n / (ms_1 * 1e-3), "ms": ms_1,
                                        "iterations_max": max(s["iterations"] for s in st_1),
                                        "true_rel_res2_max": max(s["true_rel_res2"] for s in st_1)},
                      "fp64_one_at_a_time": {"rhs_per_s": 1e3 / ms_64, "ms_per_rhs": ms_64, "rhs_timed": n64,
                                             "iterations_max": max(s["iterations"] for s in st_64)},
                      "batched_speedup": ms_1 / ms_b,
                      "batched_mixed_speedup_vs_fp64": ms_64 * n / ms_b,
                      "max_rel_diff_batched_vs_alone": diff,
                      "tuning": {"batched": tuned_b, "single": tuned_1}, "clocks": clk.summary()})


def leg_configs(args):
    """The two configurations below the headline volume, each with the
    reference's own CPU code timed on the same inputs (rank 0 host cores):
    (1) 8^3x16 plain FP64 e/o CG, kappa 0.16, mu 0.01, eps 0.4, point source,
    |r|/|b| <= 1e-12; (2) 16^3x32 mixed FP32-inner (12-real links) / FP64
    reliable updates, kappa 0.161, mu 0.005, eps 0.35, the 12 point columns
    one at a time, |r|/|b| <= 1e-10, each solution compared with the FP64 GPU
    solve (itself within 1e-9 of the reference's).  An extra line, not the
    headline."""
    import torch
    from nissa_b200 import Lattice
    from nissa_b200 import workload as wl
    dev = "cuda:0"
    threads = os.cpu_count() or 1
    res = {}

    def timed(fn, n):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = [fn() for _ in range(n)]
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n, out

    def reference_full_solve(conf, T, L, kappa, mu, src, residue):
        try:
            import oracle
            if not oracle.ref_available():
                return None, None
            conf_bc = wl.apply_time_bc(conf, T, L, -1.0)
            sol, rec, _ = oracle.run_ref("cgfull", T, L, {"conf": conf_bc, "in": src}, (T * L ** 3, 4, 3, 2),
                                         kappa=kappa, mu=mu, niter=100000, residue=residue, threads=threads)
            return sol, rec.get("seconds_per_rep")
        except Exception as e:  # the CPU leg is reported, never required
            log("reference CPU solve unavailable: %s" % e)
            return None, None

    # (1) 8^3x16 plain FP64 CG
    T, L = 16, 8
    conf = wl.gauge_conf(T, L, 0.4, 1)
    src = wl.point_source(T, L)
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        s_d = torch.from_numpy(src).to(dev)
        sol = torch.empty_like(s_d)
        ms, st = timed(lambda: lat.inv_tmD_cg_eoprec(0.16, 0.01, s_d, 100000, 1e-24, out=sol)[1], 5)
        ref_sol, ref_s = reference_full_solve(conf, T, L, 0.16, 0.01, src, 1e-24)
        err = None if ref_sol is None else float(np.linalg.norm(sol.cpu().numpy() - ref_sol) / np.linalg.norm(ref_sol))
        res["8^3x16 FP64 CG, point source, 1e-12"] = {
            "gpu_ms_per_solve": ms, "iterations": st[-1]["iterations"], "lx_rel_res2": st[-1]["lx_rel_res2"],
            "reference_cpu_s_per_solve": ref_s, "cpu_threads": threads, "rel_err_vs_reference": err,
            "speedup_vs_reference_cpu": None if ref_s is None else ref_s / (ms * 1e-3)}

    # (2) 16^3x32 mixed FP32 inner, 12 point columns one at a time
    T, L = 32, 16
    conf = wl.gauge_conf(T, L, 0.35, 1, device=dev)
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        lat.set_tuning("links_single", 0)  # the configuration's FP32 12-real links
        cols = [torch.from_numpy(wl.point_source(T, L, spin=k // 3, col=k % 3)).to(dev) for k in range(12)]
        mixed = [torch.empty_like(cols[0]) for _ in range(12)]
        fp64 = [torch.empty_like(cols[0]) for _ in range(12)]

        def solve_all(prec, outs):
            return [lat.inv_tmD_cg_eoprec(0.161, 0.005, cols[k], 100000, 1e-20, precision=prec, out=outs[k])[1]
                    for k in range(12)]
        ms_m, st_m = timed(lambda: solve_all("single", mixed), 1)
        ms_d, st_d = timed(lambda: solve_all("double", fp64), 1)
        lat.set_tuning("links_single", 1)  # the library's default: 16-bit 12-real links
        ms_16, _ = timed(lambda: solve_all("single", [torch.empty_like(cols[0]) for _ in range(12)]), 1)
        errs = [float(torch.linalg.norm(mixed[k] - fp64[k]) / torch.linalg.norm(fp64[k])) for k in range(12)]
        ref_sol, ref_s = reference_full_solve(conf, T, L, 0.161, 0.005, cols[0].cpu().numpy(), 1e-20)
        err_ref = None if ref_sol is None else float(
            np.linalg.norm(fp64[0].cpu().numpy() - ref_sol) / np.linalg.norm(ref_sol))
        res["16^3x32 mixed FP32 (12-real links), 12 point columns, 1e-10"] = {
            "gpu_mixed_ms_per_solve": ms_m / 12, "gpu_fp64_ms_per_solve": ms_d / 12,
            "mixed_speedup_vs_fp64": ms_d / ms_m,
            "gpu_mixed_16bit_links_ms_per_solve": ms_16 / 12,
            "iterations_mixed": [s["iterations"] for s in st_m[-1]],
            "iterations_fp64": [s["iterations"] for s in st_d[-1]],
            "true_rel_res2_max": max(s["true_rel_res2"] for s in st_m[-1]),
            "mixed_rel_err_vs_fp64_max": max(errs),
            "reference_cpu_s_per_solve": ref_s, "cpu_threads": threads,
            "fp64_column0_rel_err_vs_reference": err_ref,
            "speedup_vs_reference_cpu": None if ref_s is None else ref_s / (ms_m / 12 * 1e-3)}
    return {"workload": "configurations below the headline volume", "results": res}


CLOVER_WORKLOAD = dict(name="twisted-clover e/o CG solve (inv_tmclovD_cg_eoprec), 32^3x64, cSW 1.6, point sources, "
                            "|r|/|b|<=1e-10", T=64, L=32, eps=0.35, seed=1, kappa=0.1350, cSW=1.6, mu=0.005,
                       residue=1e-20)


def run_clover(args):
    """The twisted-clover full solve at the headline volume: FP64, FP32-inner and
    FP16-inner (FP64 reliable updates), each solution's true residual checked
    in FP64 and compared with the FP64 solve (an extra line, not the headline)."""
    import torch
    from nissa_b200 import Lattice
    from nissa_b200 import workload as wl
    W = dict(CLOVER_WORKLOAD)
    if args.lattice:
        W["T"], W["L"] = (int(x) for x in args.lattice.split(","))
    T, L = W["T"], W["L"]
    V = T * L ** 3
    dev = "cuda:0"
    lat = Lattice(T, L)
    lat.upload_conf(wl.gauge_conf(T, L, W["eps"], W["seed"], device=dev))
    t0 = time.perf_counter()
    lat.clover_term(W["cSW"])
    t_clover = time.perf_counter() - t0
    src = torch.zeros((V, 4, 3, 2), dtype=torch.float64, device=dev)
    src[0, 0, 0, 0] = 1.0
    sols, res = {}, {}
    for prec in ("double", "single", "half"):
        sols[prec] = torch.empty_like(src)
        lat.inv_tmclovD_cg_eoprec(W["kappa"], W["cSW"], W["mu"], src, 100000, W["residue"], precision=prec,
                                  out=sols[prec])
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _, st = lat.inv_tmclovD_cg_eoprec(W["kappa"], W["cSW"], W["mu"], src, 100000, W["residue"], precision=prec,
                                          out=sols[prec])
        e1.record()
        torch.cuda.synchronize()
        res[prec] = {"ms_per_solve": e0.elapsed_time(e1), "iterations": st["iterations"],
                     "reliable_updates": st["reliable_updates"], "true_rel_res2": st["true_rel_res2"],
                     "lx_rel_res2": st["lx_rel_res2"]}
    for prec in ("single", "half"):
        res[prec]["rel_err_vs_fp64"] = float(torch.linalg.norm(sols[prec] - sols["double"]) /
                                             torch.linalg.norm(sols["double"]))
        res[prec]["speedup_vs_fp64"] = res["double"]["ms_per_solve"] / res[prec]["ms_per_solve"]
    print(json.dumps({"workload": W["name"].replace("32^3x64", "%d^3x%d" % (L, T)), "kappa": W["kappa"],
                      "cSW": W["cSW"], "mu": W["mu"], "clover_term_s": t_clover, "results": res}), flush=True)


SERVE_WORKLOAD = dict(volumes={"8^3x16": (16, 8), "16^3x32": (32, 16), "32^3x64": (64, 32)},
                      probs=[0.5, 0.35, 0.15], eps=0.35, seed=1, rate=20.0, requests=400, nslots=16)


def leg_serve(args):
    """The serving workload: three resident configurations, Poisson arrivals
    at a stated rate, requests batched continuously per volume; p50/p99
    latency and throughput."""
    from nissa_b200 import workload as wl
    from nissa_b200.serve import GpuResidency, SolveServer, latency_summary, poisson_requests, run_load
    W = SERVE_WORKLOAD
    rate = args.rate or W["rate"]
    n = args.requests or W["requests"]
    vols = {k: (T, L, wl.gauge_conf(T, L, W["eps"], W["seed"], device="cuda:0")) for k, (T, L) in W["volumes"].items()}
    res = GpuResidency(vols, nslots=W["nslots"], precision=args.serve_precision,
                       priorities=bool(args.serve_priorities))
    srv = SolveServer(res.backends(), free_memory=res.free_memory, reserve_bytes=2 << 30)
    warm = poisson_requests(6, rate=100.0, volumes=list(vols), probs=[1 / 3] * 3, seed=99)
    run_load(srv, warm, keep_solutions=False)
    sched = poisson_requests(n, rate=rate, volumes=list(vols), probs=W["probs"], seed=W["seed"])
    with ClockSampler(0) as clk:
        results, wall = run_load(srv, sched, keep_solutions=False)
    srv.close()
    summ = latency_summary(results, wall)
    summ.update({"workload": "serving: resident 8^3x16, 16^3x32, 32^3x64; Poisson arrivals",
                 "rate_per_s": rate, "precision": args.serve_precision, "slots_per_volume": W["nslots"],
                 "stream_priorities": "smaller volumes first" if args.serve_priorities else "equal",
                 "max_true_rel_res2_over_target": max(r.stats["true_rel_res2"] / r.request.residue for r in results),
                 "failed": sum(r.stats["status"] != 0 for r in results), "clocks": clk.summary()})
    res.close()
    return summ


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=12)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-legs", action="store_true",
                    help="skip the other configurations (16^3x32 and 8^3x16 columns, 48-RHS batched, multi-shift, "
                         "serving) that the headline line carries as sub-objects")
    ap.add_argument("--lattice", default=None, help="T,L override for quick checks (not the benchmark workload)")
    ap.add_argument("--kernel-only", default=None, choices=["double", "single", "half"],
                    help="only time the e/o hopping kernel of this precision (profiling entry point)")
    ap.add_argument("--variant", type=int, default=1, help="hopping kernel variant for --kernel-only")
    ap.add_argument("--nrep", type=int, default=10, help="launches for --kernel-only")
    ap.add_argument("--nrhs", type=int, default=1, help="right-hand sides for --kernel-only (batched kernel if > 1)")
    ap.add_argument("--mrhs", type=int, default=0, help="right-hand sides per thread of the batched kernel (tuning)")
    ap.add_argument("--hop-cfg", type=int, default=-1,
                    help="hopping-kernel launch shape of the inner precision (default: the autotuner's)")
    ap.add_argument("--half-arith", action="store_true",
                    help="headline with the FP16 inner hop in FP16 arithmetic (opt-in; default FP32 arithmetic)")
    ap.add_argument("--tma-rows", type=int, default=-1,
                    help="lattice rows per tile of the staged launch shape (with --hop-cfg or --kernel-only)")
    ap.add_argument("--workload", default="cg",
                    choices=["cg", "cgm", "serve", "batched", "configs", "clover", "tune", "batched-once"],
                    help="cg: the headline solve; cgm: the multi-shift workload; serve: the serving loop; "
                         "batched: 48 right-hand sides batched vs one at a time; configs: the 8^3x16 and "
                         "16^3x32 configurations with the reference's CPU solve; clover: the twisted-clover "
                         "solve (extra reports); tune: the autotuner's choice and evidence per volume; "
                         "batched-once: one batched solve alone (profiling entry point)")
    ap.add_argument("--rate", type=float, default=0.0, help="serve: Poisson arrival rate (requests/s)")
    ap.add_argument("--requests", type=int, default=0, help="serve: number of requests")
    ap.add_argument("--serve-precision", default="single", choices=["double", "single", "half"])
    ap.add_argument("--serve-priorities", type=int, default=0, choices=[0, 1],
                    help="serve: give the streams of smaller volumes higher priorities")
    ap.add_argument("--cgm-precision", default="half", choices=["single", "half"])
    ap.add_argument("--precision", default="half", choices=["double", "single", "half"],
                    help="inner precision of the headline solve")
    args = ap.parse_args()
    WORKLOAD["name"] = WORKLOAD["name"] % PREC_NAME[args.precision]
    if args.lattice:
        T, L = (int(x) for x in args.lattice.split(","))
        WORKLOAD.update(T=T, L=L, name=WORKLOAD["name"].replace("32^3x64", "%d^3x%d" % (L, T)))
    if args.kernel_only:
        run_kernel_only(args)
        return
    legs = {"cgm": leg_cgm, "serve": leg_serve, "batched": leg_batched, "configs": leg_configs, "tune": leg_tune}
    if args.workload in legs:
        print(json.dumps(legs[args.workload](args)), flush=True)
        return
    if args.workload == "clover":
        run_clover(args)
        return
    if args.workload == "batched-once":
        run_batched_once(args)
        return
    if args.impl == "reference":
        run_reference_arm(args)
    else:
        run_ours(args)

if __name__ == "__main__":
    main()
