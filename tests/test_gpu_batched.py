"""Batched (multi-RHS) e/o solves through the C ABI: each right-hand side of a
batch must give the same solution as its own single solve (within the mixed
precision tolerance) and reach its own target, whatever else is in the batch."""
import numpy as np
import pytest

import oracle
from nissa_b200 import Lattice, TmError
from nissa_b200 import workload as wl
from conftest import rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,mrhs", [("double", 1), ("double", 2), ("single", 1), ("single", 0),
                                            ("half", 0), ("half", 2), ("half", 4)])
def test_batched_matches_single_solves(cuda_device, precision, mrhs):
    """Every shape of the batched kernel: R right-hand sides per thread, or one
    with its gathers pipelined through shared memory (mrhs 0)."""
    T, L = 16, 8
    kappa = 0.1610
    conf = wl.gauge_conf(T, L, 0.35, seed=51)
    srcs = [wl.z2_source(T, L, 60 + c, spin=c // 3, col=c % 3) for c in range(6)]
    mus = [0.005, -0.005, 0.01, -0.01, 0.003, 0.02]
    res = [1e-20, 1e-20, 1e-18, 1e-20, 1e-16, 1e-20]
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        lat.set_tuning("mrhs_per_thread", mrhs)
        sols, st = lat.inv_tmD_cg_eoprec_batched(kappa, mus, srcs, 100000, res, precision=precision)
        for k in range(len(srcs)):
            ref, sref = lat.inv_tmD_cg_eoprec(kappa, mus[k], srcs[k], 100000, 1e-24, precision="double")
            assert st[k]["true_rel_res2"] < res[k], (k, st[k])
            tol = 1e-9 if res[k] <= 1e-20 else 1e-6
            assert rel(sols[k], ref) < tol, (k, rel(sols[k], ref))


def test_batched_double_matches_oracle(cuda_device, golden_small):
    g = golden_small
    T, L = int(g["T"]), int(g["L"])
    with Lattice(T, L) as lat:
        lat.upload_conf(g["conf"])
        sols, st = lat.inv_tmD_cg_eoprec_batched(float(g["kappa"]), [float(g["mu"])] * 2,
                                                 [g["in_lx"], 2 * g["in_lx"]], 10000, [1e-24, 1e-24])
        assert rel(sols[0], g["cgfull"]) < 1e-9
        assert rel(sols[1], 2 * g["cgfull"]) < 1e-9
        assert abs(st[0]["iterations"] - int(g["cgfull_iters"])) <= 1


def test_batched_argument_errors(cuda_device):
    with Lattice(4, 4) as lat:
        lat.upload_conf(wl.gauge_conf(4, 4, 0.4, 1))
        x = wl.random_spinor(lat.V, 2)
        with pytest.raises(TmError) as e:
            lat.inv_tmD_cg_eoprec_batched(0.16, [0.01, 0.01], [x, np.zeros_like(x)], 100, 1e-20)
        assert e.value.status == 8
        with pytest.raises(TmError) as e:
            lat.inv_tmD_cg_eoprec_batched(0.16, [0.01] * 65, [x] * 65, 100, 1e-20)
        assert e.value.status == 3


@pytest.mark.parametrize("precision", ["double", "single"])
def test_session_admits_while_running(cuda_device, precision):
    """Continuous batching: right-hand sides with different kappa and mu are
    submitted while others are iterating; every result equals its own single
    solve."""
    T, L = 8, 8
    conf = wl.gauge_conf(T, L, 0.35, seed=61)
    reqs = [(0.156 + 0.001 * k, 0.002 * (k + 1), wl.z2_source(T, L, 70 + k)) for k in range(7)]
    res = 1e-20
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        refs = [lat.inv_tmD_cg_eoprec(kp, mu, s, 100000, 1e-24)[0] for kp, mu, s in reqs]
        out = {}
        with lat.batch_session(3, precision) as ses:
            pending = list(range(len(reqs)))
            running = {}
            steps = 0
            while pending or running:
                for slot in ses.free_slots():
                    if not pending:
                        break
                    k = pending.pop(0)
                    kp, mu, s = reqs[k]
                    ses.submit(slot, s, kp, mu, 100000, res)
                    running[slot] = k
                for slot in ses.step():
                    sol, st = ses.collect(slot)
                    assert st["status"] == 0 and st["true_rel_res2"] < res
                    out[running.pop(slot)] = sol
                steps += 1
                assert steps < 10000
        for k in range(len(reqs)):
            assert rel(out[k], refs[k]) < 1e-9, k
