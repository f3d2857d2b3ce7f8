"""Generate the golden fixtures of this directory by running the REFERENCE's own
code (nissa, built by oracle/ref_build into oracle/_ref/nissa_ref) on seeded
inputs.

    python tests/golden/make_golden.py [--ref <reference checkout>]

(default checkout: $NISSA_REFERENCE, else the one oracle/ref_build/Makefile reads)

Fixtures:
  ref_T4L4.npz      4^4 lattice: every operator on the path and the CG / full
                    solve / multi-shift solves, inputs included.
  ref_T4L4_clover.npz  4^4 twisted clover: clover term, inverse, Schur operator,
                    its square and the full e/o solve.
  ref_geom.npz      the reference's own e/o geometry tables (loclx_parity,
                    loceo_of_loclx, loclx_of_loceo, loceo_neighup/dw of
                    set_eo_geometry, geometry_eo.cpp:41-100) for 4^4 and 8^3x16.
  L4T8conf          the reference's own 4^3x8 ILDG test configuration
                    (test/data/L4T8conf, copied unchanged); its known
                    plaquette is 0.6350055722288719
                    (test/nissa/src/plaquette_computation.cpp:7-8).
  ref_T16L8_cg.npz  8^3x16 lattice, the plain FP64 CG workload (kappa=0.16,
                    mu=0.01, eps=0.4, point source, |r|/|b| <= 1e-12): the
                    conf is regenerated from its seed, the fixture keeps the
                    iteration count, |x|^2 and the solution on every 8th site.

The reference sees the links with the antiperiodic time sign folded into the
t=T-1 time links (its operators read links as given); the fixtures keep the
periodic links plus bc_t = -1.
"""
from __future__ import annotations

import argparse
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402
from nissa_b200 import workload as wl  # noqa: E402


def iters_from(stdout: str, key: str) -> int:
    m = re.findall(key + r"\s*:\s*(\d+)", stdout)
    return int(m[-1]) if m else -1


def make_small(path):
    T, L = 4, 4
    V, Vh = T * L ** 3, T * L ** 3 // 2
    kappa, mu = 0.16, 0.01
    conf = wl.gauge_conf(T, L, 0.4, seed=11)
    conf_bc = wl.apply_time_bc(conf, T, L, -1.0)
    rng = np.random.Generator(np.random.Philox(12))
    in_odd = rng.standard_normal((Vh, 4, 3, 2))
    in_even = rng.standard_normal((Vh, 4, 3, 2))
    in_lx = rng.standard_normal((V, 4, 3, 2))
    sh = (Vh, 4, 3, 2)
    out = {}
    out["hop0"], _, _ = oracle.run_ref("hop", T, L, {"conf": conf_bc, "in": in_odd}, sh, par=0)
    out["hop1"], _, _ = oracle.run_ref("hop", T, L, {"conf": conf_bc, "in": in_even}, sh, par=1)
    out["hop1_anis"], _, _ = oracle.run_ref("hop", T, L, {"conf": conf_bc, "in": in_even}, sh, par=1, anis=1.3)
    out["kern"], _, _ = oracle.run_ref("kern", T, L, {"conf": conf_bc, "in": in_odd}, sh, kappa=kappa, mu=mu)
    out["kern2"], _, _ = oracle.run_ref("kern2", T, L, {"conf": conf_bc, "in": in_odd}, sh, kappa=kappa, mu=mu)
    out["tmQ"], _, _ = oracle.run_ref("tmQ", T, L, {"conf": conf_bc, "in": in_lx}, (V, 4, 3, 2), kappa=kappa, mu=mu)
    out["cg"], _, so = oracle.run_ref("cg", T, L, {"conf": conf_bc, "in": in_odd}, sh, kappa=kappa, mu=mu,
                                      niter=10000, residue=1e-24)
    out["cg_iters"] = np.array(iters_from(so, "Total cg iterations"))
    out["cgfull"], _, so = oracle.run_ref("cgfull", T, L, {"conf": conf_bc, "in": in_lx}, (V, 4, 3, 2), kappa=kappa,
                                          mu=mu, niter=10000, residue=1e-24)
    out["cgfull_iters"] = np.array(iters_from(so, "Total cg iterations"))
    masses = np.array([0.01, 0.05, 0.2])
    residues = np.array([1e-20, 1e-20, 1e-20])
    out["cgm"], _, so = oracle.run_ref("cgm", T, L, {"conf": conf_bc, "in": in_lx}, (3, V, 4, 3, 2), kappa=kappa,
                                       masses=masses, residues=residues, niter=10000)
    out["cgm_iters"] = np.array(iters_from(so, "Total cgm iterations"))
    np.savez_compressed(path, T=T, L=L, bc_t=-1.0, kappa=kappa, mu=mu, anis=1.3, conf=conf, in_odd=in_odd,
                        in_even=in_even, in_lx=in_lx, masses=masses, residues=residues, **out)
    print("wrote", path, {k: (v.shape if hasattr(v, "shape") else v) for k, v in out.items()})


def make_cg(path):
    T, L = 16, 8
    kappa, mu, eps, seed = 0.1600, 0.01, 0.4, 1
    conf = wl.gauge_conf(T, L, eps, seed=seed)
    conf_bc = wl.apply_time_bc(conf, T, L, -1.0)
    src = wl.point_source(T, L, 0, 0, 0)
    sol, rec, so = oracle.run_ref("cgfull", T, L, {"conf": conf_bc, "in": src}, (T * L ** 3, 4, 3, 2), kappa=kappa,
                                  mu=mu, niter=100000, residue=1e-24)
    _, prec, _ = oracle.run_ref("plaq", T, L, {"conf": conf_bc}, None)
    np.savez_compressed(path, T=T, L=L, bc_t=-1.0, kappa=kappa, mu=mu, eps=eps, seed=seed, residue=1e-24,
                        iters=iters_from(so, "Total cg iterations"), sol_norm2=float(np.sum(sol ** 2)),
                        sol_every8=sol[::8], plaquette_bc=prec["plaquette"], seconds=rec["seconds_per_rep"])
    print("wrote", path, "iters", iters_from(so, "Total cg iterations"), "plaq", prec["plaquette"])


def make_geom(path):
    out = {}
    for T, L in ((4, 4), (16, 8)):
        for k, v in oracle.ref_geometry(T, L).items():
            out["T%dL%d_%s" % (T, L, k)] = v
    np.savez_compressed(path, **out)
    print("wrote", path, sorted(out))


def copy_known_answer_conf(ref_root, path):
    import shutil
    shutil.copyfile(os.path.join(ref_root, "test", "data", "L4T8conf"), path)
    print("copied", path, os.path.getsize(path), "bytes")


def make_clover(path):
    """Twisted clover on 4^4: the clover term, its twisted inverse (every 8th
    site), the Schur operator for both dagger flags, its square, and the full
    e/o solve inv_tmclovD_cg_eoprec (|r|/|b| <= 1e-12) with its iteration count."""
    T, L = 4, 4
    V, Vh = T * L ** 3, T * L ** 3 // 2
    kappa, mu, cSW = 0.135, 0.03, 1.6
    conf = wl.gauge_conf(T, L, 0.4, seed=5)
    conf_bc = wl.apply_time_bc(conf, T, L, -1.0)
    rng = np.random.Generator(np.random.Philox(13))
    x = rng.standard_normal((Vh, 4, 3, 2))
    src = rng.standard_normal((V, 4, 3, 2))
    sh = (Vh, 4, 3, 2)
    out = {}
    out["clover"], _, _ = oracle.run_ref("clover", T, L, {"conf": conf_bc}, (V, 4, 3, 3, 2), cSW=cSW)
    inv, _, _ = oracle.run_ref("invclover", T, L, {"conf": conf_bc}, (V, 2, 6, 6, 2), cSW=cSW, kappa=kappa, mu=mu)
    out["invclover_every8"] = inv[::8]
    for dag in (0, 1):
        out["kern_dag%d" % dag], _, _ = oracle.run_ref("clovkern", T, L, {"conf": conf_bc, "in": x}, sh, cSW=cSW,
                                                       kappa=kappa, mu=mu, dag=dag)
    out["kern2"], _, _ = oracle.run_ref("clovkern2", T, L, {"conf": conf_bc, "in": x}, sh, cSW=cSW, kappa=kappa, mu=mu)
    out["cgfull"], _, so = oracle.run_ref("clovcgfull", T, L, {"conf": conf_bc, "in": src}, (V, 4, 3, 2), cSW=cSW,
                                          kappa=kappa, mu=mu, niter=10000, residue=1e-24)
    out["cgfull_iters"] = np.array(iters_from(so, "Total cg iterations"))
    np.savez_compressed(path, T=T, L=L, bc_t=-1.0, kappa=kappa, mu=mu, cSW=cSW, conf=conf, x=x, src=src, **out)
    print("wrote", path, {k: (v.shape if hasattr(v, "shape") else v) for k, v in out.items()})


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=None)
    ap.add_argument("--only", default=None, help="comma-separated subset: small,cg,clover,geom,kat")
    a = ap.parse_args()
    ref_root = a.ref or oracle.reference_root()
    oracle.build_ref(ref_root)
    only = set(a.only.split(",")) if a.only else {"small", "cg", "clover", "geom", "kat"}
    if "geom" in only:
        make_geom(os.path.join(HERE, "ref_geom.npz"))
    if "kat" in only:
        copy_known_answer_conf(ref_root, os.path.join(HERE, "L4T8conf"))
    if "small" in only:
        make_small(os.path.join(HERE, "ref_T4L4.npz"))
    if "cg" in only:
        make_cg(os.path.join(HERE, "ref_T16L8_cg.npz"))
    if "clover" in only:
        make_clover(os.path.join(HERE, "ref_T4L4_clover.npz"))
