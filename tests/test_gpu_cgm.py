"""Multi-shift CGM on the tm Q^2 operator and the full-lattice CG of Q(+m)Q(-m)
through the C ABI, against the reference's fixture (FP64) and the oracle."""
import numpy as np
import pytest

import oracle
from nissa_b200 import Lattice, TmError
from nissa_b200 import workload as wl
from conftest import rel

pytestmark = pytest.mark.gpu


def test_cgm_double_matches_reference_fixture(cuda_device, golden_small):
    g = golden_small
    T, L = int(g["T"]), int(g["L"])
    with Lattice(T, L) as lat:
        lat.upload_conf(g["conf"])
        sols, st = lat.inv_tmQ2_cgm(float(g["kappa"]), g["masses"], g["in_lx"], 10000, g["residues"])
        for k in range(len(g["masses"])):
            assert abs(st[k]["iterations"] - int(g["cgm_iters"])) <= 1
            assert rel(sols[k], g["cgm"][k]) < 1e-9, k
            assert st[k]["true_rel_res2"] < 2e-20


@pytest.mark.parametrize("precision,batched", [("single", 0), ("half", 0), ("half", 1)])
def test_cgm_mixed_reaches_every_target(cuda_device, precision, batched):
    """Both forms of the mixed solver's per-shift correction (shift after shift,
    or all shifts as batched e/o solves) reach every target."""
    T, L = 16, 8
    kappa = 0.1632
    masses = np.array([0.005, 0.02, 0.08, 0.2])
    conf = wl.gauge_conf(T, L, 0.35, seed=41)
    src = wl.z2_source(T, L, 5, col=1)
    geo = oracle.Geom(T, L)
    ref, _, _ = geo.cgm(wl.apply_time_bc(conf, T, L), kappa, masses, np.full(4, 1e-24), src, 100000)
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        lat.set_tuning("cgm_refine_batched", batched)
        sols, st = lat.inv_tmQ2_cgm(kappa, masses, src, 100000, 1e-20, precision=precision)
        for k in range(len(masses)):
            assert st[k]["true_rel_res2"] < 1e-20, (k, st[k])
            assert rel(sols[k], ref[k]) < 1e-8, k


def test_cg_tmQ2_matches_single_shift(cuda_device):
    T, L = 8, 4
    kappa, m = 0.16, 0.03
    conf = wl.gauge_conf(T, L, 0.4, seed=43)
    src = wl.random_spinor(T * L ** 3, 44)
    geo = oracle.Geom(T, L)
    ref, _, _ = geo.cgm(wl.apply_time_bc(conf, T, L), kappa, [m], [1e-26], src, 100000)
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        for prec in ("double", "single", "half"):
            sol, st = lat.inv_tmQ2_cg(kappa, m, src, 100000, 1e-22, precision=prec)
            assert st["true_rel_res2"] < 1e-22, prec
            assert rel(sol, ref[0]) < 1e-9, prec
        # the operator check: Q(+m)Q(-m) sol = src
        back = lat.apply_tmQ2(kappa, m, sol)
        assert rel(back, src) < 1e-10


def test_cgm_argument_errors(cuda_device):
    with Lattice(4, 4) as lat:
        lat.upload_conf(wl.gauge_conf(4, 4, 0.4, 1))
        src = wl.random_spinor(lat.V, 1)
        with pytest.raises(TmError) as e:
            lat.inv_tmQ2_cgm(0.16, np.linspace(0.01, 0.3, 33), src, 100, 1e-20)
        assert e.value.status == 3
        with pytest.raises(TmError) as e:
            lat.inv_tmQ2_cgm(0.16, [0.1], np.zeros_like(src), 100, 1e-20)
        assert e.value.status == 8
        with pytest.raises(TmError) as e:
            lat.inv_tmQ2_cgm(0.16, [0.01, 0.1], src, 3, 1e-24)
        assert e.value.status == 1
