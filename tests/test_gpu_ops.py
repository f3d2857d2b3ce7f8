"""CUDA operators (through the C ABI) against the oracle and the reference's
own outputs.  FP64 operators must agree to 1e-14 relative (the Dslash parity
bar); geometry tables must be bit-exact."""
import numpy as np
import pytest

import oracle
from nissa_b200 import Lattice, TmError
from nissa_b200 import workload as wl
from conftest import rel

pytestmark = pytest.mark.gpu

TOL = 1e-14


GEOM_KEYS = ("parity", "eo_of_lx", "lx_of_eo", "neighup_eo", "neighdw_eo")


@pytest.mark.parametrize("T,L", [(4, 4), (16, 8)])
def test_geometry_tables_match_reference_dump(cuda_device, golden_geom, T, L):
    """Device tables against the reference's own loclx_parity, loceo_of_loclx,
    loclx_of_loceo and loceo_neighup/dw (geometry_eo.cpp:41-100), bit-exact."""
    with Lattice(T, L) as lat:
        mine = lat.geometry_tables()
    for k in GEOM_KEYS:
        assert np.array_equal(mine[k], golden_geom["T%dL%d_%s" % (T, L, k)]), k


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
@pytest.mark.parametrize("T,L", [(64, 32), (12, 6)])
def test_geometry_tables_match_live_reference(cuda_device, T, L):
    """The same at the headline volume (and a non-power-of-two one), against a
    live dump by the reference build."""
    with Lattice(T, L) as lat:
        mine = lat.geometry_tables()
    ref = oracle.ref_geometry(T, L)
    for k in GEOM_KEYS:
        assert np.array_equal(mine[k], ref[k]), k


@pytest.mark.parametrize("T,L", [(8, 6), (12, 4)])
def test_geometry_tables_bit_exact(cuda_device, T, L):
    with Lattice(T, L) as lat:
        mine = lat.geometry_tables()
    ref = oracle.Geom(T, L).tables()
    for k in GEOM_KEYS:
        assert np.array_equal(mine[k], ref[k]), k


def test_operators_match_reference_fixture(cuda_device, golden_small):
    g = golden_small
    T, L = int(g["T"]), int(g["L"])
    k, mu = float(g["kappa"]), float(g["mu"])
    with Lattice(T, L, bc_t=float(g["bc_t"])) as lat:
        lat.upload_conf(g["conf"])
        assert lat.conf_is_su3
        assert rel(lat.tmn2Deo_or_tmn2Doe_eos(0, g["in_odd"]), g["hop0"]) < TOL
        assert rel(lat.tmn2Deo_or_tmn2Doe_eos(1, g["in_even"]), g["hop1"]) < TOL
        assert rel(lat.tmn2Deo_or_tmn2Doe_eos(1, g["in_even"], anis=float(g["anis"])), g["hop1_anis"]) < TOL
        assert rel(lat.tmDkern_eoprec_eos(k, mu, g["in_odd"]), g["kern"]) < TOL
        assert rel(lat.tmDkern_eoprec_square_eos(k, mu, g["in_odd"]), g["kern2"]) < TOL
        assert rel(lat.apply_tmQ(k, mu, g["in_lx"]), g["tmQ"]) < TOL


@pytest.mark.parametrize("T,L,eps", [(16, 8, 0.4), (32, 16, 0.35), (8, 6, 0.35)])
def test_operators_match_oracle(cuda_device, T, L, eps):
    conf = wl.gauge_conf(T, L, eps, seed=T + L)
    conf_bc = wl.apply_time_bc(conf, T, L, -1.0)
    geo = oracle.Geom(T, L)
    ceo = geo.split(conf_bc)
    rng = np.random.default_rng(7)
    x = rng.standard_normal((geo.Vh, 4, 3, 2))
    xl = rng.standard_normal((geo.V, 4, 3, 2))
    k, mu = 0.161, 0.005
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        for par in (0, 1):
            assert rel(lat.tmn2Deo_or_tmn2Doe_eos(par, x), geo.hop(ceo, par, x)) < TOL
        assert rel(lat.tmDee_or_oo_eos(k, mu, x), geo.tmDee(k, mu, x)) < TOL
        assert rel(lat.inv_tmDee_or_oo_eos(k, mu, x), geo.inv_tmDee(k, mu, x)) < TOL
        assert rel(lat.tmDkern_eoprec_eos(k, -mu, x), geo.kern(ceo, k, -mu, x)) < TOL
        assert rel(lat.tmDkern_eoprec_square_eos(k, mu, x, anis=0.9), geo.kern2(ceo, k, mu, x, anis=0.9)) < TOL
        assert rel(lat.apply_tmQ(k, mu, xl), geo.tmQ(conf_bc, k, mu, xl)) < TOL
        assert rel(lat.apply_tmQ2(k, mu, xl), geo.tmQ2(conf_bc, k, mu, xl)) < TOL


def test_bc_included_upload_is_equivalent(cuda_device):
    T, L = 8, 4
    conf = wl.gauge_conf(T, L, 0.4, seed=3)
    x = np.random.default_rng(1).standard_normal((T * L ** 3 // 2, 4, 3, 2))
    with Lattice(T, L) as a, Lattice(T, L) as b, Lattice(T, L, bc_t=+1.0) as c:
        a.upload_conf(conf)
        b.upload_conf(wl.apply_time_bc(conf, T, L, -1.0), bc_included=True)
        c.upload_conf(wl.apply_time_bc(conf, T, L, -1.0))  # periodic lattice, sign carried by the links
        ya, yb, yc = (lat.tmn2Deo_or_tmn2Doe_eos(1, x) for lat in (a, b, c))
        assert np.array_equal(ya, yb)
        assert rel(yc, ya) < TOL
        assert b.conf_is_su3 and not c.conf_is_su3


def test_eo_layout_upload(cuda_device):
    T, L = 8, 4
    conf = wl.gauge_conf(T, L, 0.4, seed=4)
    geo = oracle.Geom(T, L)
    x = np.random.default_rng(2).standard_normal((geo.Vh, 4, 3, 2))
    with Lattice(T, L) as a, Lattice(T, L) as b:
        a.upload_conf(conf)
        b.upload_conf(geo.split(conf), layout="eo")
        assert np.array_equal(a.tmn2Deo_or_tmn2Doe_eos(0, x), b.tmn2Deo_or_tmn2Doe_eos(0, x))


def test_device_pointer_mode(cuda_device):
    import torch
    T, L = 8, 4
    conf = wl.gauge_conf(T, L, 0.4, seed=5)
    geo = oracle.Geom(T, L)
    x = np.random.default_rng(3).standard_normal((geo.Vh, 4, 3, 2))
    with Lattice(T, L) as lat:
        lat.upload_conf(torch.from_numpy(conf).cuda())
        y = lat.tmDkern_eoprec_square_eos(0.16, 0.01, torch.from_numpy(x).cuda())
        assert y.is_cuda
        assert rel(y.cpu().numpy(), geo.kern2(geo.split(wl.apply_time_bc(conf, T, L)), 0.16, 0.01, x)) < TOL


def test_errors(cuda_device):
    with Lattice(4, 4) as lat:
        with pytest.raises(TmError) as e:
            lat.tmn2Deo_or_tmn2Doe_eos(0, np.zeros((128, 4, 3, 2)))
        assert e.value.status == 7  # no conf yet
        lat.upload_conf(wl.gauge_conf(4, 4, 0.4, 1))
        with pytest.raises(TmError) as e:
            lat.tmn2Deo_or_tmn2Doe_eos(2, np.zeros((128, 4, 3, 2)))
        assert e.value.status == 3
        with pytest.raises(TmError) as e:
            lat.tmDkern_eoprec_eos(-0.1, 0.0, np.zeros((128, 4, 3, 2)))
        assert e.value.status == 3
