"""Scheduling logic of the continuous-batching server, on the CPU: a stand-in
session with the same four calls as the GPU batch session."""
import threading
import time

import pytest

from nissa_b200.serve import SolveRequest, SolveServer, latency_summary, poisson_requests, run_load


class FakeSession:
    """nslots slots; a request needs `steps` steps, given by its residue."""

    def __init__(self, nslots, log):
        self.nslots = nslots
        self.slots = {}
        self.done = set()
        self.log = log
        self.lock = threading.Lock()

    def free_slots(self):
        return [k for k in range(self.nslots) if k not in self.slots]

    def submit(self, slot, src, kappa, mu, niter, residue):
        assert slot not in self.slots
        self.slots[slot] = [int(residue), src]
        self.log.append(("submit", src, time.perf_counter()))

    def step(self):
        time.sleep(0.002)
        fin = []
        for k, v in self.slots.items():
            if k in self.done:
                continue
            v[0] -= 1
            if v[0] <= 0:
                fin.append(k)
                self.done.add(k)
        return fin

    def collect(self, slot):
        steps, src = self.slots.pop(slot)
        self.done.discard(slot)
        return ("solution-of", src), {"status": 0, "iterations": 1}


def make_source(volume, req):
    if req.source == "bad":
        raise ValueError("bad source")
    return (volume, req.seed)


def test_every_request_gets_its_own_result():
    log = []
    srv = SolveServer({"a": (FakeSession(3, log), make_source, 0), "b": (FakeSession(2, log), make_source, 0)})
    futs = [srv.submit(SolveRequest(volume="ab"[i % 2], kappa=0.16, mu=0.01, residue=1 + i % 4, seed=i))
            for i in range(20)]
    res = [f.result(timeout=30) for f in futs]
    srv.close()
    for i, r in enumerate(res):
        assert r.solution == ("solution-of", ("ab"[i % 2], i))
        assert r.latency >= r.admitted_after >= 0


def test_late_short_request_is_admitted_while_long_ones_run():
    """Continuous batching: with one slot busy on a long solve, a request
    arriving later goes into the other slot at once and finishes first."""
    log = []
    srv = SolveServer({"v": (FakeSession(2, log), make_source, 0)})
    long = srv.submit(SolveRequest(volume="v", kappa=0.16, mu=0.01, residue=200, seed=1))
    time.sleep(0.02)
    short = srv.submit(SolveRequest(volume="v", kappa=0.16, mu=0.01, residue=2, seed=2))
    rs = short.result(timeout=30)
    assert not long.done()
    assert rs.admitted_after < 0.05
    long.result(timeout=30)
    srv.close()


def test_admission_waits_for_memory():
    free = [0]
    log = []
    srv = SolveServer({"v": (FakeSession(4, log), make_source, 100)}, free_memory=lambda: free[0])
    f = srv.submit(SolveRequest(volume="v", kappa=0.16, mu=0.01, residue=1, seed=3))
    time.sleep(0.05)
    assert not f.done() and not log
    free[0] = 1000
    assert f.result(timeout=30).solution == ("solution-of", ("v", 3))
    srv.close()


def test_bad_request_fails_alone():
    log = []
    srv = SolveServer({"v": (FakeSession(2, log), make_source, 0)})
    bad = srv.submit(SolveRequest(volume="v", kappa=0.16, mu=0.01, residue=1, source="bad"))
    good = srv.submit(SolveRequest(volume="v", kappa=0.16, mu=0.01, residue=1, seed=5))
    with pytest.raises(ValueError):
        bad.result(timeout=30)
    assert good.result(timeout=30).solution == ("solution-of", ("v", 5))
    with pytest.raises(KeyError):
        srv.submit(SolveRequest(volume="nope", kappa=0.16, mu=0.01, residue=1))
    srv.close()


def test_poisson_schedule_and_summary():
    sched = poisson_requests(200, rate=1000.0, volumes=["a", "b", "c"], probs=[0.5, 0.35, 0.15], seed=3)
    ts = [t for t, _ in sched]
    assert ts == sorted(ts)
    vols = [r.volume for _, r in sched]
    assert 0.35 < vols.count("a") / 200 < 0.65
    assert all(0.155 <= r.kappa <= 0.163 and 0.002 <= r.mu <= 0.05 for _, r in sched)
    assert all(min(abs(r.residue / 1e-16 - 1), abs(r.residue / 1e-20 - 1)) < 1e-9 for _, r in sched)
    log = []
    srv = SolveServer({v: (FakeSession(4, log), make_source, 0) for v in "abc"})
    for _, r in sched:
        r.residue = 1
    results, wall = run_load(srv, sched[:40])
    srv.close()
    s = latency_summary(results, wall)
    assert s["requests"] == 40 and s["p99_s"] >= s["p50_s"] > 0
    assert s["admission_wait_p99_s"] >= 0 and s["in_batch_p99_s"] > 0


def test_run_load_can_release_solutions():
    """keep_solutions=False drops each solution when its request completes
    (its memory goes back to the allocator); the stats and latencies stay."""
    sched = poisson_requests(12, rate=1000.0, volumes=["a", "b"], probs=[0.5, 0.5], seed=5)
    for _, r in sched:
        r.residue = 1
    srv = SolveServer({v: (FakeSession(4, []), make_source, 0) for v in "ab"})
    results, wall = run_load(srv, sched, keep_solutions=False)
    srv.close()
    assert len(results) == 12
    assert all(r.solution is None and r.stats["status"] == 0 and r.latency >= 0 for r in results)
