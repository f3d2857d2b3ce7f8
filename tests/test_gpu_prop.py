"""The caller-side steps around a propagator solve (get_qprop's basis
rotations, the twisted doublet) through the C ABI, against numpy and the
oracle."""
import numpy as np
import pytest

import oracle
from nissa_b200 import Lattice
from nissa_b200 import workload as wl
from conftest import rel

pytestmark = pytest.mark.gpu


def rotate_np(r, x):
    """P- (r=0) / P+ (r=1): diag(1-+i, 1-+i, 1+-i, 1+-i)/sqrt2 (new_types/dirac.cpp:60-61)."""
    z = x[..., 0] + 1j * x[..., 1]
    s = 1.0 if r == 1 else -1.0
    d = np.array([1 + 1j * s, 1 + 1j * s, 1 - 1j * s, 1 - 1j * s]) / np.sqrt(2.0)
    w = z * d[None, :, None]
    return np.stack([w.real, w.imag], axis=-1)


@pytest.mark.parametrize("cSW", [0.0, 1.4])
def test_get_qprop(cuda_device, cSW):
    T, L = 8, 4
    kappa, mu = 0.14, 0.02
    conf = wl.gauge_conf(T, L, 0.35, seed=61)
    src = wl.random_spinor(T * L ** 3, 62)
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        for r in (0, 1):
            assert rel(lat.rotate_twisted(r, src), rotate_np(r, src)) < 1e-15
            prop, st = lat.get_qprop(r, kappa, mu, src, 1e-24, cSW=cSW)
            if cSW:
                x, _ = lat.inv_tmclovD_cg_eoprec(kappa, cSW, mu, rotate_np(r, src), 100000, 1e-24)
            else:
                x, _ = lat.inv_tmD_cg_eoprec(kappa, mu, rotate_np(r, src), 100000, 1e-24)
            assert rel(prop, rotate_np(r, x)) < 1e-12
            assert st["lx_rel_res2"] < 1e-22
            # without the source rotation (a non-twisted run) only the sink is rotated
            prop2, _ = lat.get_qprop(r, kappa, mu, src, 1e-24, cSW=cSW, rotate_source=False)
            if cSW:
                y, _ = lat.inv_tmclovD_cg_eoprec(kappa, cSW, mu, src, 100000, 1e-24)
            else:
                y, _ = lat.inv_tmD_cg_eoprec(kappa, mu, src, 100000, 1e-24)
            assert rel(prop2, rotate_np(r, y)) < 1e-12


def test_reconstruct_tm_doublet(cuda_device):
    T, L = 8, 4
    kappa, mu = 0.14, 0.03
    conf = wl.gauge_conf(T, L, 0.35, seed=63)
    x = wl.random_spinor(T * L ** 3, 64)
    geo = oracle.Geom(T, L)
    qm = geo.tmQ(wl.apply_time_bc(conf, T, L, -1.0), kappa, +mu, x)
    z = x[..., 0] + 1j * x[..., 1]
    qp = (qm[..., 0] + 1j * qm[..., 1]) - 2j * mu * z
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        om, op = lat.reconstruct_tm_doublet(kappa, mu, x)
        assert rel(om, qm) < 1e-14
        assert rel(op, np.stack([qp.real, qp.imag], axis=-1)) < 1e-14
