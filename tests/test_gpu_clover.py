"""The twisted-clover e/o path through the C ABI, against the reference's own
outputs (tests/golden/ref_T4L4_clover.npz, made by the reference build) and
against the oracle on further sizes, anisotropy and both parities."""
import os

import numpy as np
import pytest

import oracle
from nissa_b200 import Lattice, TmError
from nissa_b200 import workload as wl
from conftest import GOLDEN, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def golden_clover():
    return dict(np.load(os.path.join(GOLDEN, "ref_T4L4_clover.npz")))


def test_clover_matches_reference_fixture(cuda_device, golden_clover):
    g = golden_clover
    T, L = int(g["T"]), int(g["L"])
    kappa, mu, cSW = float(g["kappa"]), float(g["mu"]), float(g["cSW"])
    with Lattice(T, L, bc_t=float(g["bc_t"])) as lat:
        lat.upload_conf(g["conf"])
        lat.clover_term(cSW)
        assert rel(lat.clover_get(), g["clover"]) < 1e-14
        for dag in (0, 1):
            assert rel(lat.tmclovDkern_eoprec_eos(kappa, mu, dag, g["x"]), g["kern_dag%d" % dag]) < 1e-14
        assert rel(lat.tmclovDkern_eoprec_square_eos(kappa, mu, g["x"]), g["kern2"]) < 1e-14
        sol, st = lat.inv_tmclovD_cg_eoprec(kappa, cSW, mu, g["src"], 10000, 1e-24)
        assert abs(st["iterations"] - int(g["cgfull_iters"])) <= 1
        assert rel(sol, g["cgfull"]) < 1e-9
        assert st["lx_rel_res2"] < 1e-22


@pytest.mark.parametrize("anis", [None, 1.2])
def test_clover_operators_match_oracle(cuda_device, anis):
    T, L = 8, 4
    kappa, mu, cSW = 0.131, 0.02, 1.3
    conf = wl.gauge_conf(T, L, 0.35, seed=51)
    geo = oracle.Geom(T, L)
    V, Vh = geo.V, geo.Vh
    conf_bc = wl.apply_time_bc(conf, T, L, -1.0)
    Cl = geo.clover_term(conf_bc, cSW)
    inv = geo.inv_clover_term(Cl, kappa, mu)
    Cl_eo = geo.split(Cl.reshape(V, -1)).reshape(2, Vh, 4, 3, 3, 2)
    inv_eo = geo.split(inv.reshape(V, -1)).reshape(2, Vh, 2, 6, 6, 2)
    ceo = geo.split(conf_bc)
    x = wl.random_spinor(Vh, 52)
    xl = wl.random_spinor(V, 53)
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        lat.clover_term(cSW)
        assert rel(lat.clover_get(), Cl) < 1e-14
        for par in (0, 1):
            for dag in (0, 1):
                assert rel(lat.tmclovDee_or_oo_eos(par, kappa, mu, dag, x), geo.tmclovDee(Cl_eo[par], kappa, dag, mu, x)) < 1e-14
        for dag in (0, 1):
            assert rel(lat.inv_tmclovDee_or_oo_eos(kappa, mu, dag, x), geo.inv_tmclovDee(inv_eo[0], dag, x)) < 1e-13
            assert rel(lat.tmclovDkern_eoprec_eos(kappa, mu, dag, x, anis=anis),
                       geo.tmclov_kern(ceo, kappa, Cl_eo[1], inv_eo[0], dag, mu, x, anis=anis)) < 1e-13
        assert rel(lat.tmclovDkern_eoprec_square_eos(kappa, mu, x, anis=anis),
                   geo.tmclov_kern2(ceo, kappa, Cl_eo[1], inv_eo[0], mu, x, anis=anis)) < 1e-13
        assert rel(lat.apply_tmclovQ(kappa, mu, xl, anis=anis), geo.tmclovQ(conf_bc, kappa, Cl, mu, xl, anis=anis)) < 1e-14


@pytest.mark.parametrize("precision", ["single", "half"])
def test_clover_mixed_precision(cuda_device, precision):
    T, L = 16, 8
    kappa, mu, cSW = 0.136, 0.01, 1.5
    conf = wl.gauge_conf(T, L, 0.35, seed=54)
    src = wl.random_spinor(T * L ** 3 // 2, 55)
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        lat.clover_term(cSW)
        ref, st0 = lat.inv_tmclovDkern_eoprec_square_eos_cg(kappa, mu, src, 100000, 1e-22)
        sol, st = lat.inv_tmclovDkern_eoprec_square_eos_cg(kappa, mu, src, 100000, 1e-20, precision=precision)
        assert st["true_rel_res2"] < 1e-20
        assert rel(sol, ref) < 1e-8
        assert st["iterations"] <= 1.1 * st0["iterations"] + 5
        # the full solve in mixed precision reaches the reference's final check
        srcl = wl.random_spinor(T * L ** 3, 56)
        s64, _ = lat.inv_tmclovD_cg_eoprec(kappa, cSW, mu, srcl, 100000, 1e-22)
        sm, stm = lat.inv_tmclovD_cg_eoprec(kappa, cSW, mu, srcl, 100000, 1e-20, precision=precision)
        assert stm["lx_rel_res2"] < 1e-19
        assert rel(sm, s64) < 1e-8


def test_clover_errors(cuda_device):
    with Lattice(4, 4) as lat:
        lat.upload_conf(wl.gauge_conf(4, 4, 0.4, seed=57))
        x = wl.random_spinor(lat.Vh, 1)
        with pytest.raises(TmError) as e:
            lat.tmclovDkern_eoprec_square_eos(0.13, 0.01, x)
        assert e.value.status == 7
        lat.clover_term(1.0)
        lat.tmclovDkern_eoprec_square_eos(0.13, 0.01, x)
        lat.upload_conf(wl.gauge_conf(4, 4, 0.4, seed=58))  # a new conf voids the clover term
        with pytest.raises(TmError):
            lat.tmclovDkern_eoprec_square_eos(0.13, 0.01, x)


@pytest.mark.parametrize("precision", ["single", "half"])
def test_clover_paired_x_updates_match_unpaired(cuda_device, precision):
    """The twisted-clover mixed solver with the every-other-iteration x update
    (even graph length) and with the per-iteration one (odd length): same
    iteration count, solutions equal to the solver's accuracy."""
    T, L = 16, 8
    kappa, mu, cSW = 0.136, 0.01, 1.5
    src = wl.random_spinor(T * L ** 3 // 2, 65)
    sols, its = [], []
    with Lattice(T, L) as lat:
        lat.upload_conf(wl.gauge_conf(T, L, 0.35, seed=64))
        lat.clover_term(cSW)
        for gi in (8, 7):
            lat.set_tuning("graph_iters", gi)
            sol, st = lat.inv_tmclovDkern_eoprec_square_eos_cg(kappa, mu, src, 100000, 1e-20, precision=precision)
            assert st["true_rel_res2"] < 1e-20 and st["reliable_updates"] >= 2
            sols.append(sol)
            its.append(st["iterations"])
    assert abs(its[0] - its[1]) <= 1
    assert rel(sols[0], sols[1]) < 1e-8
