"""The N > 1 path (independent replicas, one per GPU) on CPU: two gloo ranks
run the host-side aggregation the bench and the serving loop use: the max
over ranks of a device time, the whole-job rate, every rank's share of the
work and the gathering of per-request results to rank 0."""
import multiprocessing as mp
import os
import socket
import traceback

import pytest

from nissa_b200 import replicas


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    try:
        import torch.distributed as dist
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                          LOCAL_RANK=str(rank))
        import datetime
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        assert replicas.dist_env() == (world, rank, rank)
        # device time: rank r took 10 (r + 1) ms for 12 solves
        ms = 10.0 * (rank + 1)
        ms_max = replicas.max_over_ranks(ms)
        rate = replicas.whole_job_rate(12, ms_max, world)
        # serving: each rank serves its share of 20 requests with the CPU stand-in session
        from nissa_b200.serve import SolveRequest, SolveServer, latency_summary, run_load
        from test_serve import FakeSession, make_source
        sched = [(0.001 * i, SolveRequest(volume="v", kappa=0.16, mu=0.01, residue=1 + i % 3, seed=i))
                 for i in range(20)]
        mine = replicas.serve_share(sched, rank, world)
        srv = SolveServer({"v": (FakeSession(4, []), make_source, 1)})
        results, wall = run_load(srv, mine)
        srv.close()
        seeds = [r.request.seed for r in results]
        got = replicas.gather_to_root({"rank": rank, "seeds": seeds, "lat": [r.latency for r in results],
                                       "wall": wall})
        if rank == 0:
            all_seeds = sorted(s for g in got for s in g["seeds"])
            q.put(("ok", rank, ms_max, rate, all_seeds, [g["rank"] for g in got]))
        else:
            q.put(("ok", rank, ms_max, rate, None, None))
        dist.barrier()
        dist.destroy_process_group()
    except Exception:
        q.put(("err", rank, traceback.format_exc()))


def test_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    errs = [o for o in out if o[0] == "err"]
    assert not errs, errs[0][2]
    by = {o[1]: o for o in out}
    for r in (0, 1):
        assert by[r][2] == 20.0                        # max over ranks
        assert by[r][3] == pytest.approx(2 * 12 / 0.020)  # both ranks' solves over the slowest time
    assert by[0][4] == list(range(20))                 # every request served exactly once
    assert by[0][5] == [0, 1]


def test_shares_without_process_group():
    assert replicas.share(range(7), 1, 3) == [1, 4]
    assert replicas.rank_columns(1, 4) == [4, 5, 6, 7]
    assert replicas.rank_columns(2, 12) == list(range(12))
    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.gather_to_root({"a": 1}) == [{"a": 1}]
    sched = list(enumerate("abcde"))
    assert replicas.serve_share(sched, 0, 2) == [(0, "a"), (2, "c"), (4, "e")]
