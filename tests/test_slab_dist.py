"""The time-slab exchange and CG across processes, on CPU: two gloo ranks,
one slab each.  The ring exchange must deliver slab k+1's forward face and
slab k-1's backward face to slab k, and the slab CG (its scalar products
all-reduced) must solve a time-coupled stand-in operator that reads its
time neighbours only through those faces, as the dense solve of the whole
system does."""
import multiprocessing as mp
import os
import socket
import traceback

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


class RingSlab:
    """CPU stand-in of a slab with the same pack / kern_half interface: a
    field of T_loc time slices of 3 reals; the operator couples each slice to
    its time neighbours (kern = 2.5 - 0.25 S^2 with S the sum of the two time
    shifts, symmetric positive definite), reading across slab edges only from
    the ghost faces."""

    def __init__(self, t0, T_loc):
        self.t0, self.T_loc = t0, T_loc

    def pack(self, par_in, f):
        return f[:1].clone(), f[-1:].clone()

    def kern_half(self, which, kappa, mu, inp, gf, gb, x=None, anis=None):
        import torch
        ext = torch.cat([gb, inp, gf])
        s = ext[2:] + ext[:-2]
        return s if which == 0 else 2.5 * x - 0.25 * s


def _rank_main(rank, world, port, T, q):
    try:
        import torch
        import torch.distributed as dist
        from nissa_b200 import slab as sl
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        import datetime
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        n = T // world
        t0 = rank * n
        # exchange schedule: faces carry (sender rank, kind)
        fwd = torch.full((4, 6, 2), 100.0 * rank + 1.0, dtype=torch.float64)
        bwd = torch.full((4, 6, 2), 100.0 * rank + 2.0, dtype=torch.float64)
        gf, gb = sl.exchange_dist(fwd, bwd)
        prev, nxt = sl.ring_targets(rank, world)
        ok_ex = bool(torch.all(gf == 100.0 * nxt + 1.0)) and bool(torch.all(gb == 100.0 * prev + 2.0))
        # the CG over slabs of the stand-in operator
        rng = np.random.default_rng(7)
        b = rng.standard_normal((T, 3))
        ss = sl.SlabSet([RingSlab(t0, n)], distributed=True)
        x, it, tres = ss.cg(0.16, 0.01, [torch.from_numpy(b[t0:t0 + n].copy())], 1000, 1e-24)
        got = [None] * world
        dist.all_gather_object(got, x[0].numpy())
        if rank == 0:
            S = np.zeros((T, T))
            for t in range(T):
                S[t, (t + 1) % T] += 1
                S[t, (t - 1) % T] += 1
            K = 2.5 * np.eye(T) - 0.25 * S @ S
            ref = np.linalg.solve(K @ K, b)
            err = float(np.linalg.norm(np.concatenate(got) - ref) / np.linalg.norm(ref))
            q.put(("ok", rank, ok_ex, it, tres, err))
        else:
            q.put(("ok", rank, ok_ex, it, tres, None))
        dist.barrier()
        dist.destroy_process_group()
    except Exception:
        q.put(("err", rank, traceback.format_exc()))


@pytest.mark.parametrize("world", [2, 3])
def test_slab_ring_exchange_and_cg_gloo(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    T = 12
    ps = [ctx.Process(target=_rank_main, args=(r, world, port, T, q)) for r in range(world)]
    for p in ps:
        p.start()
    out = [q.get(timeout=180) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    errs = [o for o in out if o[0] == "err"]
    assert not errs, errs[0][2]
    by = {o[1]: o for o in out}
    assert all(by[r][2] for r in range(world))          # every slab got its neighbours' faces
    assert len({by[r][3] for r in range(world)}) == 1    # the same iteration count on every rank
    assert by[0][4] < 1e-23 and by[0][5] < 1e-10         # the dense solve of the whole system


def test_ring_targets_and_bounds():
    from nissa_b200 import slab as sl
    assert sl.ring_targets(0, 4) == (3, 1)
    assert sl.ring_targets(3, 4) == (2, 0)
    assert sl.slab_bounds(16, 4) == [(0, 4), (4, 4), (8, 4), (12, 4)]
    with pytest.raises(ValueError):
        sl.slab_bounds(12, 4)  # slabs of 3 slices: odd
