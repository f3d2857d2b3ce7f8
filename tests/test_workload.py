import numpy as np

import oracle
from nissa_b200 import workload as wl


def test_gauge_links_special_unitary():
    c = wl.gauge_conf(4, 4, 0.4, 3)
    U = c.view(np.complex128).reshape(-1, 3, 3)
    assert np.abs(U @ U.conj().transpose(0, 2, 1) - np.eye(3)).max() < 1e-14
    assert np.abs(np.linalg.det(U) - 1).max() < 1e-14


def test_gauge_seeded_and_plaquette_range():
    a = wl.gauge_conf(8, 4, 0.35, 5)
    b = wl.gauge_conf(8, 4, 0.35, 5)
    assert np.array_equal(a, b)
    p = oracle.Geom(8, 4).plaquette(a)
    assert 0.45 < p < 0.6


def test_time_bc_only_touches_last_time_links():
    T, L = 4, 4
    c = wl.gauge_conf(T, L, 0.4, 1)
    d = wl.apply_time_bc(c, T, L, -1.0).reshape(T, L ** 3, 4, 3, 3, 2)
    c = c.reshape(T, L ** 3, 4, 3, 3, 2)
    assert np.array_equal(d[:T - 1], c[:T - 1])
    assert np.array_equal(d[T - 1, :, 1:], c[T - 1, :, 1:])
    assert np.array_equal(d[T - 1, :, 0], -c[T - 1, :, 0])


def test_sources():
    s = wl.point_source(4, 4, 5, 2, 1)
    assert s.sum() == 1.0 and s[5, 2, 1, 0] == 1.0
    z = wl.z2_source(4, 4, 7)
    assert np.allclose(np.abs(z), 1 / np.sqrt(2))
    zc = wl.z2_source(4, 4, 7, col=1)
    assert np.all(zc[:, :, [0, 2]] == 0) and np.allclose(np.abs(zc[:, :, 1]), 1 / np.sqrt(2))
