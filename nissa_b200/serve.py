"""Solve serving with continuous batching.

Several gauge configurations (one per lattice volume) stay resident on one
GPU.  Solve requests (a volume, kappa, mu, a source, a squared relative
residue) arrive at any time; each volume has one worker thread that drives
one batch session of the C ABI (tms_batch_*): a request is admitted into a
free slot as soon as one frees up and the GPU has the memory for its source
and solution, the session runs one CUDA-graph block of lock-step CG
iterations for every slot in flight, and finished slots are collected and
handed back while the others keep iterating.  Different kappa and mu share a
batch (only the diagonal terms depend on them; the links are read once for
all slots).  Workers of different volumes run concurrently on their own
streams, so their work overlaps on the device.

The scheduling logic is independent of the GPU: a worker talks to its
session through four calls (free_slots, submit, step, collect), so the tests
drive it with a CPU stand-in as well as with the real session.
"""
from __future__ import annotations

import collections
import concurrent.futures
import dataclasses
import itertools
import math
import threading
import time

import numpy as np


@dataclasses.dataclass
class SolveRequest:
    volume: str              # key of a resident configuration
    kappa: float
    mu: float
    residue: float           # squared relative residue, as the reference takes it
    source: str = "point"    # "point" (spin/colour below, at the origin) or "z2"
    seed: int = 0            # Z2 noise seed, or spin*3+colour for a point source
    niter: int = 100000
    id: int = -1
    arrival: float = 0.0     # time.perf_counter() at submission


@dataclasses.dataclass
class SolveResult:
    request: SolveRequest
    solution: object         # lx spinor (torch tensor on the device for the GPU backend)
    stats: dict
    latency: float           # completion - arrival, seconds
    admitted_after: float    # admission - arrival, seconds


class _Worker:
    """One volume: a queue and the loop that drives its batch session."""

    def __init__(self, server, volume, session, make_source, bytes_per_request):
        self.server = server
        self.volume = volume
        self.session = session
        self.make_source = make_source
        self.bytes_per_request = bytes_per_request
        self.queue = collections.deque()
        self.cond = threading.Condition()
        self.running = {}   # slot -> (request, future, source, t_admit)
        self.stop = False
        self.error = None
        self.thread = threading.Thread(target=self._loop, name="solve-" + volume, daemon=True)
        self.thread.start()

    def put(self, req, fut):
        with self.cond:
            self.queue.append((req, fut))
            self.cond.notify()

    def _admit(self):
        for slot in self.session.free_slots():
            with self.cond:
                if not self.queue:
                    return
                if not self.server._memory_ok(self.bytes_per_request):
                    return
                req, fut = self.queue.popleft()
            try:
                src = self.make_source(self.volume, req)
                self.session.submit(slot, src, req.kappa, req.mu, req.niter, req.residue)
            except Exception as e:  # a bad request fails alone
                fut.set_exception(e)
                continue
            self.running[slot] = (req, fut, src, time.perf_counter())

    def _loop(self):
        try:
            while True:
                with self.cond:
                    while not self.queue and not self.running and not self.stop:
                        self.cond.wait()
                    if self.stop and not self.queue and not self.running:
                        return
                self._admit()
                if not self.running:
                    time.sleep(0.001)  # waiting for memory
                    continue
                for slot in self.session.step():
                    req, fut, src, t_adm = self.running.pop(slot)
                    sol, st = self.session.collect(slot)
                    now = time.perf_counter()
                    fut.set_result(SolveResult(req, sol, st, now - req.arrival, t_adm - req.arrival))
        except Exception as e:
            self.error = e
            for req, fut, src, t in self.running.values():
                if not fut.done():
                    fut.set_exception(e)
            with self.cond:
                while self.queue:
                    self.queue.popleft()[1].set_exception(e)


class SolveServer:
    """Continuous-batching solve server over resident configurations.

    backends: {volume: (session, make_source, bytes_per_request)} where session
    offers free_slots/submit/step/collect (a BatchSession on the GPU) and
    make_source(volume, request) builds the request's lx source.
    free_memory: callable returning free device bytes (admission by HBM), or None.
    """

    def __init__(self, backends: dict, free_memory=None, reserve_bytes: int = 0):
        self._ids = itertools.count()
        self._free_memory = free_memory
        self.reserve_bytes = reserve_bytes
        self.workers = {v: _Worker(self, v, s, mk, nb) for v, (s, mk, nb) in backends.items()}

    def _memory_ok(self, need):
        if self._free_memory is None:
            return True
        return self._free_memory() - need >= self.reserve_bytes

    def submit(self, req: SolveRequest) -> concurrent.futures.Future:
        if req.volume not in self.workers:
            raise KeyError("no resident configuration for volume %r" % req.volume)
        req.id = next(self._ids)
        req.arrival = time.perf_counter()
        fut = concurrent.futures.Future()
        self.workers[req.volume].put(req, fut)
        return fut

    def close(self):
        for w in self.workers.values():
            with w.cond:
                w.stop = True
                w.cond.notify()
        for w in self.workers.values():
            w.thread.join()


# ------------------------------------------------------------------ GPU backend

class GpuResidency:
    """Resident lattices on one GPU: a Lattice (conf uploaded), a BatchSession
    and a source maker per volume, plus the free-HBM probe."""

    def __init__(self, volumes: dict, nslots: int = 16, precision: str = "single", device: int = 0,
                 bc_t: float = -1.0, priorities: bool = False):
        import torch
        from .tm import Lattice
        self.torch = torch
        self.device = device
        self.lattices, self.sessions, self.shapes = {}, {}, {}
        self.streams = {}
        # with priorities, smaller volumes get higher stream priorities: their
        # short kernels are scheduled ahead of the waves of a large volume's kernels
        order = sorted(volumes, key=lambda n: volumes[n][0] * volumes[n][1] ** 3)
        least, greatest = torch.cuda.Stream.priority_range()
        for name, (T, L, conf) in volumes.items():
            lat = Lattice(T, L, bc_t=bc_t, device=device)
            lat.upload_conf(conf)
            if priorities:
                lat.set_tuning("stream_priority", min(least, greatest + order.index(name)))
            self.lattices[name] = lat
            self.sessions[name] = lat.batch_session(nslots, precision)
            self.shapes[name] = (T * L ** 3, 4, 3, 2)
            self.streams[name] = torch.cuda.Stream(device=device)

    def make_source(self, volume, req: SolveRequest):
        torch = self.torch
        shape = self.shapes[volume]
        with torch.cuda.stream(self.streams[volume]):
            if req.source == "point":
                s = torch.zeros(shape, dtype=torch.float64, device="cuda:%d" % self.device)
                s[0, (req.seed // 3) % 4, req.seed % 3, 0] = 1.0
            else:
                g = torch.Generator(device="cuda:%d" % self.device)
                g.manual_seed(int(req.seed))
                bits = torch.randint(0, 2, shape, generator=g, device="cuda:%d" % self.device)
                s = (2.0 * bits.to(torch.float64) - 1.0) / math.sqrt(2.0)
        # the library reads the source on its own stream
        self.streams[volume].synchronize()
        return s

    def free_memory(self):
        return self.torch.cuda.mem_get_info(self.device)[0]

    def backends(self):
        out = {}
        for name in self.lattices:
            V = self.shapes[name][0]
            out[name] = (self.sessions[name], self.make_source, 2 * V * 24 * 8)  # source + solution
        return out

    def close(self):
        for s in self.sessions.values():
            s.close()
        for lat in self.lattices.values():
            lat.close()


# ------------------------------------------------------------------ load

def poisson_requests(n: int, rate: float, volumes, probs, seed: int = 0):
    """n requests with exponential inter-arrival times (mean 1/rate): volume
    drawn with probs, kappa ~ U[0.155, 0.163], mu log-uniform in [0.002, 0.05],
    point or Z2 source, |r|/|b| target 1e-8 or 1e-10."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        vol = volumes[rng.choice(len(volumes), p=probs)]
        kappa = rng.uniform(0.155, 0.163)
        mu = math.exp(rng.uniform(math.log(0.002), math.log(0.05)))
        point = rng.random() < 0.5
        tol = 1e-8 if rng.random() < 0.5 else 1e-10
        out.append((t, SolveRequest(volume=vol, kappa=kappa, mu=mu, residue=tol * tol,
                                    source="point" if point else "z2",
                                    seed=int(rng.integers(0, 12)) if point else int(rng.integers(1, 1 << 30)))))
    return out


def _drop_solution(fut):
    if not fut.cancelled() and fut.exception() is None:
        fut.result().solution = None


def run_load(server: SolveServer, schedule, timeout: float = 3600.0, keep_solutions: bool = True):
    """Submit the (time, request) schedule in real time; return the results and the wall time.
    With keep_solutions=False each solution is released as soon as its request
    completes (its device memory returns to the allocator's cache for the next
    request, as a server that hands results on would do); stats and latencies stay."""
    t0 = time.perf_counter()
    futs = []
    for t, req in schedule:
        delay = t0 + t - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        fut = server.submit(req)
        if not keep_solutions:
            fut.add_done_callback(_drop_solution)
        futs.append(fut)
    results = [f.result(timeout=timeout) for f in futs]
    return results, time.perf_counter() - t0


def latency_summary(results, wall):
    """Throughput and latency percentiles, overall and per volume; the p99 of
    the wait for a slot (arrival to admission) and of the time in the batch
    (admission to completion) tell queueing from solving."""
    lat = np.array([r.latency for r in results])
    wait = np.array([r.admitted_after for r in results])
    by = collections.defaultdict(list)
    for r in results:
        by[r.request.volume].append(r.latency)
    return {"requests": len(results), "wall_s": wall, "throughput_solves_per_s": len(results) / wall,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()),
            "admission_wait_p99_s": float(np.percentile(wait, 99)),
            "in_batch_p99_s": float(np.percentile(lat - wait, 99)),
            "per_volume": {v: {"n": len(x), "p50_s": float(np.percentile(x, 50)), "p99_s": float(np.percentile(x, 99))}
                           for v, x in by.items()}}
