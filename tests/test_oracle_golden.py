"""The CPU oracle (oracle/tmoracle.c) against fixtures produced by the
reference's own code (tests/golden/make_golden.py) and against the reference's
own known-answer value (test/nissa/src/plaquette_computation.cpp:7-8)."""
import os
import struct

import numpy as np
import pytest

import oracle
from nissa_b200 import workload as wl
from conftest import KAT_CONF, KAT_PLAQUETTE, rel

TOL_OP = 1e-14


def test_operators_match_reference(golden_small):
    g = golden_small
    T, L = int(g["T"]), int(g["L"])
    geo = oracle.Geom(T, L)
    conf = wl.apply_time_bc(g["conf"], T, L, float(g["bc_t"]))
    ceo = geo.split(conf)
    k, mu = float(g["kappa"]), float(g["mu"])
    assert rel(geo.hop(ceo, 0, g["in_odd"]), g["hop0"]) < TOL_OP
    assert rel(geo.hop(ceo, 1, g["in_even"]), g["hop1"]) < TOL_OP
    assert rel(geo.hop(ceo, 1, g["in_even"], anis=float(g["anis"])), g["hop1_anis"]) < TOL_OP
    assert rel(geo.kern(ceo, k, mu, g["in_odd"]), g["kern"]) < TOL_OP
    assert rel(geo.kern2(ceo, k, mu, g["in_odd"]), g["kern2"]) < TOL_OP
    assert rel(geo.tmQ(conf, k, mu, g["in_lx"]), g["tmQ"]) < TOL_OP


def test_solvers_match_reference(golden_small):
    g = golden_small
    T, L = int(g["T"]), int(g["L"])
    geo = oracle.Geom(T, L)
    conf = wl.apply_time_bc(g["conf"], T, L, float(g["bc_t"]))
    ceo = geo.split(conf)
    k, mu = float(g["kappa"]), float(g["mu"])
    sol, it, res = geo.cg_eos(ceo, k, mu, g["in_odd"], 10000, 1e-24)
    assert it == int(g["cg_iters"])
    assert rel(sol, g["cg"]) < 1e-12
    assert res < 2e-24
    sol, it, lxres = geo.cg_full(conf, k, mu, g["in_lx"], 10000, 1e-24)
    assert it == int(g["cgfull_iters"])
    assert rel(sol, g["cgfull"]) < 1e-12
    sols, it, tr = geo.cgm(conf, k, g["masses"], g["residues"], g["in_lx"], 10000)
    assert it == int(g["cgm_iters"])
    for i in range(len(g["masses"])):
        assert rel(sols[i], g["cgm"][i]) < 1e-10
        assert tr[i] < 1e-19


def test_config1_cg_matches_reference(golden_cg):
    """Plain FP64 CG on 8^3x16 (kappa 0.16, mu 0.01, point source, 1e-12)."""
    g = golden_cg
    T, L = int(g["T"]), int(g["L"])
    conf = wl.apply_time_bc(wl.gauge_conf(T, L, float(g["eps"]), int(g["seed"])), T, L, float(g["bc_t"]))
    geo = oracle.Geom(T, L)
    assert abs(geo.plaquette(conf) - float(g["plaquette_bc"])) < 1e-13
    sol, it, lxres = geo.cg_full(conf, float(g["kappa"]), float(g["mu"]), wl.point_source(T, L), 100000,
                                 float(g["residue"]))
    assert abs(it - int(g["iters"])) <= 1
    assert rel(sol[::8], g["sol_every8"]) < 1e-9
    assert abs(np.sum(sol ** 2) / float(g["sol_norm2"]) - 1) < 1e-9
    assert lxres < 1e-22


def _read_ildg_binary(path):
    """Minimal LIME reader: the 'ildg-binary-data' record as big-endian doubles."""
    with open(path, "rb") as f:
        data = f.read()
    pos = 0
    while pos + 144 <= len(data):
        magic, _ver, _flags, length = struct.unpack(">IHHQ", data[pos:pos + 16])
        assert magic == 0x456789AB
        rtype = data[pos + 16:pos + 144].split(b"\0")[0].decode()
        payload = data[pos + 144:pos + 144 + length]
        if rtype == "ildg-binary-data":
            return np.frombuffer(payload, ">f8").astype(np.float64)
        pos += 144 + ((length + 7) // 8) * 8
    raise ValueError("no ildg-binary-data record")


def test_plaquette_known_answer():
    """Golden plaquette 0.6350055722288719 of the reference's 4^3x8 fixture
    (test/data/L4T8conf, committed as tests/golden/L4T8conf;
    test/nissa/src/plaquette_computation.cpp:7-8).  ILDG stores sites with x
    fastest and links in the order x,y,z,t (io/reader.hpp:75-99 reorders)."""
    raw = _read_ildg_binary(KAT_CONF)
    T, L = 8, 4
    ildg = raw.reshape(T, L, L, L, 4, 3, 3, 2)  # [t][z][y][x][mu_ildg=x,y,z,t]
    conf = np.empty((T, L, L, L, 4, 3, 3, 2))   # [t][x][y][z][mu=t,x,y,z]
    lx = ildg.transpose(0, 3, 2, 1, 4, 5, 6, 7)
    conf[..., 0, :, :, :] = lx[..., 3, :, :, :]
    conf[..., 1, :, :, :] = lx[..., 0, :, :, :]
    conf[..., 2, :, :, :] = lx[..., 1, :, :, :]
    conf[..., 3, :, :, :] = lx[..., 2, :, :, :]
    plaq = oracle.Geom(T, L).plaquette(conf.reshape(-1, 4, 3, 3, 2))
    assert abs(plaq - KAT_PLAQUETTE) / KAT_PLAQUETTE < 1e-14


@pytest.mark.parametrize("T,L", [(4, 4), (16, 8)])
def test_geometry_tables_match_reference(golden_geom, T, L):
    """The oracle's tables equal the reference's own (set_eo_geometry,
    geometry_eo.cpp:41-100), dumped by its build into ref_geom.npz."""
    mine = oracle.Geom(T, L).tables()
    for k in ("parity", "eo_of_lx", "lx_of_eo", "neighup_eo", "neighdw_eo"):
        assert np.array_equal(mine[k], golden_geom["T%dL%d_%s" % (T, L, k)]), k


def test_unit_conf_plaquette_and_free_hop():
    T, L = 4, 4
    geo = oracle.Geom(T, L)
    conf = np.zeros((geo.V, 4, 3, 3, 2))
    for i in range(3):
        conf[:, :, i, i, 0] = 1
    assert abs(geo.plaquette(conf) - 1.0) < 1e-15
    # on the free field a constant spinor with spin content in the +1 space of
    # every (1 -/+ gamma_mu) projector pair hops to 2*4 = 8 times itself for the
    # identity part: check linearity and the constant-field eigenvalue of K
    ceo = geo.split(conf)
    x = np.random.default_rng(0).standard_normal((geo.Vh, 4, 3, 2))
    a = geo.hop(ceo, 0, x)
    b = geo.hop(ceo, 0, 2 * x)
    assert rel(b, 2 * a) < 1e-15


@pytest.fixture(scope="module")
def golden_clover():
    return dict(np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ref_T4L4_clover.npz")))


def test_clover_oracle_matches_reference(golden_clover):
    """Twisted clover: clover term, twisted inverse, Schur operator (both dagger
    flags), its square and the full e/o solve against the reference's own outputs."""
    g = golden_clover
    T, L = int(g["T"]), int(g["L"])
    kappa, mu, cSW = float(g["kappa"]), float(g["mu"]), float(g["cSW"])
    geo = oracle.Geom(T, L)
    V, Vh = geo.V, geo.Vh
    conf_bc = wl.apply_time_bc(g["conf"], T, L, float(g["bc_t"]))
    Cl = geo.clover_term(conf_bc, cSW)
    assert rel(Cl, g["clover"]) < 1e-14
    inv = geo.inv_clover_term(Cl, kappa, mu)
    assert rel(inv[::8], g["invclover_every8"]) < 1e-14
    ceo = geo.split(conf_bc)
    Cl_eo = geo.split(Cl.reshape(V, -1)).reshape(2, Vh, 4, 3, 3, 2)
    inv_eo = geo.split(inv.reshape(V, -1)).reshape(2, Vh, 2, 6, 6, 2)
    for dag in (0, 1):
        assert rel(geo.tmclov_kern(ceo, kappa, Cl_eo[1], inv_eo[0], dag, mu, g["x"]), g["kern_dag%d" % dag]) < 1e-14
    assert rel(geo.tmclov_kern2(ceo, kappa, Cl_eo[1], inv_eo[0], mu, g["x"]), g["kern2"]) < 1e-14
    sol, it, lxres = geo.tmclov_cg_full(conf_bc, kappa, cSW, mu, g["src"], 10000, 1e-24)
    assert it == int(g["cgfull_iters"])
    assert rel(sol, g["cgfull"]) < 1e-12
    assert lxres < 1e-23
