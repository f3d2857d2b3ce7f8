"""The serving loop on the GPU: three resident volumes, a Poisson mix of
requests of different volumes, kappa, mu, sources and tolerances admitted
continuously into batch sessions.  Each result must equal the same request
solved alone (a plain inv_tmD_cg_eoprec call), within 100*sqrt(residue)
relative, and reach its own target residual."""
import math

import numpy as np
import pytest

from nissa_b200 import workload as wl
from nissa_b200.serve import GpuResidency, SolveServer, latency_summary, poisson_requests, run_load
from conftest import rel

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["single", "half"])
def test_mix_equals_alone(cuda_device, precision):
    vols = {"4^4": (4, 4, wl.gauge_conf(4, 4, 0.35, 81)), "8^3x8": (8, 8, wl.gauge_conf(8, 8, 0.35, 82)),
            "8^3x16": (16, 8, wl.gauge_conf(16, 8, 0.35, 83))}
    res = GpuResidency(vols, nslots=4, precision=precision)
    srv = SolveServer(res.backends(), free_memory=res.free_memory)
    sched = poisson_requests(16, rate=400.0, volumes=list(vols), probs=[0.5, 0.35, 0.15], seed=7)
    results, wall = run_load(srv, sched, timeout=600)
    srv.close()
    s = latency_summary(results, wall)
    assert s["requests"] == 16
    for r in results:
        q = r.request
        assert r.stats["status"] == 0
        assert r.stats["true_rel_res2"] < q.residue
        lat = res.lattices[q.volume]
        src = res.make_source(q.volume, q)
        alone, st = lat.inv_tmD_cg_eoprec(q.kappa, q.mu, src, 100000, q.residue, precision=precision)
        err = rel(r.solution.cpu().numpy(), alone.cpu().numpy())
        assert err < 100 * math.sqrt(q.residue), (q, err)
    res.close()
