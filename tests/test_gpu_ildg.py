"""ILDG files and the device plaquette, through the C ABI.

The writer is pinned by the reference's own reader (read_ildg_gauge_conf run
by the reference build, oracle/_ref), the reader by files the reference reads
identically and by its 4^3x8 fixture (committed under tests/golden) with the
golden plaquette 0.6350055722288719
(test/nissa/src/plaquette_computation.cpp:7-8).  The device plaquette is
compared with the oracle's global_plaquette_lx_conf."""
import os

import numpy as np
import pytest

import oracle
from nissa_b200 import Lattice, TmError
from nissa_b200 import workload as wl
from conftest import KAT_CONF, KAT_PLAQUETTE

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("T,L", [(8, 4), (16, 8)])
def test_round_trip_and_plaquette(cuda_device, tmp_path, T, L):
    conf = wl.gauge_conf(T, L, 0.35, seed=41)
    path = str(tmp_path / "conf.ildg")
    with Lattice(T, L) as lat:
        lat.write_ildg(path, conf)
        back = lat.read_ildg(path)
        assert np.array_equal(back, conf)
        lat.load_ildg(path)
        geo = oracle.Geom(T, L)
        p = lat.plaquette()
        assert abs(p - geo.plaquette(conf)) < 1e-14
        pbc = lat.plaquette(with_bc=True)
        assert abs(pbc - geo.plaquette(wl.apply_time_bc(conf, T, L, -1.0))) < 1e-14
        # single-precision files read back within float rounding
        lat.write_ildg(path, conf, precision=32)
        b32 = lat.read_ildg(path)
        assert np.max(np.abs(b32 - conf)) < 1e-6


@pytest.mark.skipif(not oracle.ref_available(), reason="reference build absent")
def test_reference_reader_reads_our_file(cuda_device, tmp_path):
    T, L = 8, 4
    conf = wl.gauge_conf(T, L, 0.4, seed=42)
    path = str(tmp_path / "conf.ildg")
    with Lattice(T, L) as lat:
        lat.write_ildg(path, conf)
    ref, rec, _ = oracle.run_ref("ildg2raw", T, L, {}, (T * L ** 3, 4, 3, 3, 2), ildg=path)
    assert np.array_equal(ref, conf)


def test_size_mismatch_and_missing_file(cuda_device, tmp_path):
    conf = wl.gauge_conf(8, 4, 0.35, seed=43)
    path = str(tmp_path / "conf.ildg")
    with Lattice(8, 4) as lat:
        lat.write_ildg(path, conf)
        with pytest.raises(TmError) as e:
            lat.read_ildg(str(tmp_path / "absent.ildg"))
        assert e.value.status == 9
        with pytest.raises(TmError):
            lat.plaquette()  # no conf uploaded yet
    with Lattice(4, 4) as lat:
        with pytest.raises(TmError) as e:
            lat.read_ildg(path)
        assert e.value.status == 3


def test_reference_fixture_golden_plaquette(cuda_device):
    """The reference's own known answer: its 4^3x8 test configuration
    (test/data/L4T8conf, committed as tests/golden/L4T8conf) read by the device
    ILDG reader has plaquette 0.6350055722288719
    (test/nissa/src/plaquette_computation.cpp:7-8)."""
    with Lattice(8, 4) as lat:
        lat.load_ildg(KAT_CONF)
        assert abs(lat.plaquette() - KAT_PLAQUETTE) < 1e-14
