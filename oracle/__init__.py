"""CPU oracle for the twisted-mass Wilson hot path (TEST INFRASTRUCTURE ONLY).

Python bindings of ``tmoracle.c``, a plain-C restatement of the reference
library's algorithms (each C function cites the reference file:line it
follows), and a runner for the reference's own code built by
``oracle/ref_build`` into ``oracle/_ref/nissa_ref``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this package, and only as the checker or the timed CPU
baseline.  The product (``nissa_b200``) never imports it.

Array conventions (numpy float64, the reference's CPU AoS layout):
  lx conf  (V, 4, 3, 3, 2)   eo conf (2, Vh, 4, 3, 3, 2)
  lx spinor (V, 4, 3, 2)     eo spinor (Vh, 4, 3, 2)
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD_DIR = os.path.join(HERE, "_build")
LIB_PATH = os.path.join(BUILD_DIR, "libtmoracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_BIN = os.path.join(REF_DIR, "nissa_ref")
SRC = os.path.join(HERE, "tmoracle.c")

_lib = None


def build(force: bool = False) -> str:
    """Compile the C restatement into oracle/_build/libtmoracle.so."""
    os.makedirs(BUILD_DIR, exist_ok=True)
    stale = (not os.path.exists(LIB_PATH)) or os.path.getmtime(LIB_PATH) < max(
        os.path.getmtime(SRC), os.path.getmtime(os.path.join(HERE, "tmoracle.h")))
    if force or stale:
        tmp = LIB_PATH + ".tmp%d" % os.getpid()
        subprocess.check_call(["/usr/bin/gcc", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared",
                               "-std=c11", SRC, "-o", tmp, "-lm"])
        os.replace(tmp, LIB_PATH)
    return LIB_PATH


def reference_root() -> str:
    """The reference checkout: $NISSA_REFERENCE, else the default of the build
    recipe (oracle/ref_build/Makefile, the one file that names it)."""
    env = os.environ.get("NISSA_REFERENCE")
    if env:
        return env
    try:
        return subprocess.run(["make", "-s", "-C", os.path.join(HERE, "ref_build"), "print-ref"], capture_output=True,
                              text=True, check=True).stdout.strip()
    except Exception:
        return ""


def build_ref(ref_root: str | None = None, jobs: int = 8) -> str | None:
    """Build the reference's own code into oracle/_ref/nissa_ref (needs the reference tree)."""
    ref_root = ref_root or reference_root()
    if not ref_root or not os.path.isdir(os.path.join(ref_root, "src")):
        return REF_BIN if os.path.exists(REF_BIN) else None
    subprocess.check_call(["make", "-s", "-j%d" % jobs, "-C", os.path.join(HERE, "ref_build"), "REF=" + ref_root])
    return REF_BIN


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.c_void_p
        D = ctypes.c_double
        I = ctypes.c_int
        L.orc_geom_create.restype = P
        L.orc_geom_create.argtypes = [I, I]
        L.orc_geom_destroy.argtypes = [P]
        L.orc_geom_tables.argtypes = [P] + [P] * 7
        L.orc_split_lx_to_eo.argtypes = [P, P, I, P]
        L.orc_paste_eo_to_lx.argtypes = [P, P, I, P]
        L.orc_hop_eo.argtypes = [P, P, I, I, D, P, P]
        L.orc_tmDee.argtypes = [P, D, D, P, P]
        L.orc_inv_tmDee.argtypes = [P, D, D, P, P]
        L.orc_kern.argtypes = [P, P, D, I, D, D, P, P]
        L.orc_kern2.argtypes = [P, P, D, I, D, D, P, P]
        L.orc_cg_eos.restype = I
        L.orc_cg_eos.argtypes = [P, P, D, I, D, D, I, D, P, P, P, P]
        L.orc_cg_full.restype = I
        L.orc_cg_full.argtypes = [P, P, D, I, D, D, I, D, P, P, P]
        L.orc_tmQ.argtypes = [P, P, D, I, D, D, P, P]
        L.orc_tmQ2.argtypes = [P, P, D, I, D, D, P, P]
        L.orc_cgm.restype = I
        L.orc_cgm.argtypes = [P, P, D, I, D, I, P, P, I, P, P, P]
        L.orc_plaquette.restype = D
        L.orc_plaquette.argtypes = [P, P]
        I64 = ctypes.c_int64
        L.orc_clover_term.argtypes = [P, P, D, P]
        L.orc_inv_clover_term.argtypes = [I64, P, D, D, P]
        L.orc_tmclovDee.argtypes = [I64, P, D, I, D, P, P]
        L.orc_inv_tmclovDee.argtypes = [I64, P, I, P, P]
        L.orc_tmclov_kern.argtypes = [P, P, D, I, D, P, P, I, D, P, P]
        L.orc_tmclov_kern2.argtypes = [P, P, D, I, D, P, P, D, P, P]
        L.orc_tmclov_cg_eos.restype = I
        L.orc_tmclov_cg_eos.argtypes = [P, P, D, I, D, P, P, D, I, D, P, P, P, P]
        L.orc_tmclovQ.argtypes = [P, P, D, I, D, P, D, P, P]
        L.orc_tmclov_cg_full.restype = I
        L.orc_tmclov_cg_full.argtypes = [P, P, D, I, D, D, D, I, D, P, P, P]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _anis(anis):
    return (0, 0.0) if anis is None else (1, float(anis))


class Geom:
    """T x L^3 lattice as the reference's initGrid(T, L) builds it."""

    def __init__(self, T: int, L: int):
        self.T, self.L = T, L
        self.V = T * L ** 3
        self.Vh = self.V // 2
        self._g = lib().orc_geom_create(T, L)
        if not self._g:
            raise ValueError("lattice sizes must be positive and even")

    def __del__(self):
        if getattr(self, "_g", None):
            lib().orc_geom_destroy(self._g)
            self._g = None

    def tables(self):
        V = self.V
        t = dict(parity=np.empty(V, np.int32), eo_of_lx=np.empty(V, np.int32), lx_of_eo=np.empty((2, V // 2), np.int32),
                 neighup_eo=np.empty((2, V // 2, 4), np.int32), neighdw_eo=np.empty((2, V // 2, 4), np.int32),
                 neighup_lx=np.empty((V, 4), np.int32), neighdw_lx=np.empty((V, 4), np.int32))
        lib().orc_geom_tables(self._g, *[_p(t[k]) for k in ("parity", "eo_of_lx", "lx_of_eo", "neighup_eo",
                                                            "neighdw_eo", "neighup_lx", "neighdw_lx")])
        return t

    # ------------------------------------------------------------ remaps
    def split(self, lx):
        lx = _c(lx)
        ndeg = lx.size // self.V
        eo = np.empty((2, self.Vh) + lx.shape[1:], np.float64)
        lib().orc_split_lx_to_eo(self._g, _p(lx), ndeg, _p(eo))
        return eo

    def paste(self, eo):
        eo = _c(eo)
        ndeg = eo.size // self.V
        lx = np.empty((self.V,) + eo.shape[2:], np.float64)
        lib().orc_paste_eo_to_lx(self._g, _p(eo), ndeg, _p(lx))
        return lx

    # --------------------------------------------------------- operators
    def hop(self, conf_eo, par_out, inp, anis=None):
        conf_eo, inp = _c(conf_eo), _c(inp)
        out = np.empty((self.Vh, 4, 3, 2))
        lib().orc_hop_eo(self._g, _p(conf_eo), int(par_out), *_anis(anis), _p(inp), _p(out))
        return out

    def tmDee(self, kappa, mu, inp):
        inp = _c(inp)
        out = np.empty_like(inp)
        lib().orc_tmDee(self._g, kappa, mu, _p(inp), _p(out))
        return out

    def inv_tmDee(self, kappa, mu, inp):
        inp = _c(inp)
        out = np.empty_like(inp)
        lib().orc_inv_tmDee(self._g, kappa, mu, _p(inp), _p(out))
        return out

    def kern(self, conf_eo, kappa, mu, inp, anis=None):
        conf_eo, inp = _c(conf_eo), _c(inp)
        out = np.empty((self.Vh, 4, 3, 2))
        lib().orc_kern(self._g, _p(conf_eo), kappa, *_anis(anis), mu, _p(inp), _p(out))
        return out

    def kern2(self, conf_eo, kappa, mu, inp, anis=None):
        conf_eo, inp = _c(conf_eo), _c(inp)
        out = np.empty((self.Vh, 4, 3, 2))
        lib().orc_kern2(self._g, _p(conf_eo), kappa, *_anis(anis), mu, _p(inp), _p(out))
        return out

    def tmQ(self, conf_lx, kappa, mu, inp, anis=None):
        conf_lx, inp = _c(conf_lx), _c(inp)
        out = np.empty((self.V, 4, 3, 2))
        lib().orc_tmQ(self._g, _p(conf_lx), kappa, *_anis(anis), mu, _p(inp), _p(out))
        return out

    def tmQ2(self, conf_lx, kappa, mu, inp, anis=None):
        conf_lx, inp = _c(conf_lx), _c(inp)
        out = np.empty((self.V, 4, 3, 2))
        lib().orc_tmQ2(self._g, _p(conf_lx), kappa, *_anis(anis), mu, _p(inp), _p(out))
        return out

    # ----------------------------------------------------------- solvers
    def cg_eos(self, conf_eo, kappa, mu, src, niter, residue, guess=None, anis=None):
        """Returns (sol, iterations, true |r|^2/|b|^2)."""
        conf_eo, src = _c(conf_eo), _c(src)
        guess = None if guess is None else _c(guess)
        sol = np.empty((self.Vh, 4, 3, 2))
        res = ctypes.c_double(0)
        it = lib().orc_cg_eos(self._g, _p(conf_eo), kappa, *_anis(anis), mu, int(niter), float(residue), _p(guess),
                              _p(src), _p(sol), ctypes.byref(res))
        return sol, it, res.value

    def cg_full(self, conf_lx, kappa, mu, src_lx, niter, residue, anis=None):
        """inv_tmD_cg_eoprec: returns (sol_lx, iterations, lx |g5 Q x - b|^2/|b|^2)."""
        conf_lx, src_lx = _c(conf_lx), _c(src_lx)
        sol = np.empty((self.V, 4, 3, 2))
        res = ctypes.c_double(0)
        it = lib().orc_cg_full(self._g, _p(conf_lx), kappa, *_anis(anis), mu, int(niter), float(residue), _p(src_lx),
                               _p(sol), ctypes.byref(res))
        return sol, it, res.value

    # ------------------------------------------------------ twisted clover
    def clover_term(self, conf_lx, cSW):
        """clover_term: [V][4][3][3][2] (four leaves, anti-symmetrised, times -cSW/4)."""
        conf_lx = _c(conf_lx)
        out = np.empty((self.V, 4, 3, 3, 2))
        lib().orc_clover_term(self._g, _p(conf_lx), float(cSW), _p(out))
        return out

    @staticmethod
    def inv_clover_term(Cl, kappa, mass):
        """invert_twisted_clover_term: [sites][2][6][6][2]."""
        Cl = _c(Cl)
        n = Cl.shape[0]
        out = np.empty((n, 2, 6, 6, 2))
        lib().orc_inv_clover_term(n, _p(Cl), float(kappa), float(mass), _p(out))
        return out

    @staticmethod
    def tmclovDee(Cl, kappa, dag, mu, inp):
        Cl, inp = _c(Cl), _c(inp)
        out = np.empty_like(inp)
        lib().orc_tmclovDee(Cl.shape[0], _p(Cl), float(kappa), int(dag), float(mu), _p(inp), _p(out))
        return out

    @staticmethod
    def inv_tmclovDee(invCl, dag, inp):
        invCl, inp = _c(invCl), _c(inp)
        out = np.empty_like(inp)
        lib().orc_inv_tmclovDee(invCl.shape[0], _p(invCl), int(dag), _p(inp), _p(out))
        return out

    def tmclov_kern(self, conf_eo, kappa, Cl_odd, invCl_evn, dag, mu, inp, anis=None):
        conf_eo, Cl_odd, invCl_evn, inp = _c(conf_eo), _c(Cl_odd), _c(invCl_evn), _c(inp)
        out = np.empty_like(inp)
        lib().orc_tmclov_kern(self._g, _p(conf_eo), float(kappa), *_anis(anis), _p(Cl_odd), _p(invCl_evn), int(dag),
                              float(mu), _p(inp), _p(out))
        return out

    def tmclov_kern2(self, conf_eo, kappa, Cl_odd, invCl_evn, mu, inp, anis=None):
        conf_eo, Cl_odd, invCl_evn, inp = _c(conf_eo), _c(Cl_odd), _c(invCl_evn), _c(inp)
        out = np.empty_like(inp)
        lib().orc_tmclov_kern2(self._g, _p(conf_eo), float(kappa), *_anis(anis), _p(Cl_odd), _p(invCl_evn),
                               float(mu), _p(inp), _p(out))
        return out

    def tmclov_cg_eos(self, conf_eo, kappa, Cl_odd, invCl_evn, mu, src, niter, residue, guess=None, anis=None):
        conf_eo, Cl_odd, invCl_evn, src = _c(conf_eo), _c(Cl_odd), _c(invCl_evn), _c(src)
        guess = None if guess is None else _c(guess)
        sol = np.empty((self.Vh, 4, 3, 2))
        res = ctypes.c_double(0)
        it = lib().orc_tmclov_cg_eos(self._g, _p(conf_eo), float(kappa), *_anis(anis), _p(Cl_odd), _p(invCl_evn),
                                     float(mu), int(niter), float(residue), _p(guess), _p(src), _p(sol),
                                     ctypes.byref(res))
        return sol, it, res.value

    def tmclovQ(self, conf_lx, kappa, Cl_lx, mu, inp, anis=None):
        conf_lx, Cl_lx, inp = _c(conf_lx), _c(Cl_lx), _c(inp)
        out = np.empty_like(inp)
        lib().orc_tmclovQ(self._g, _p(conf_lx), float(kappa), *_anis(anis), _p(Cl_lx), float(mu), _p(inp), _p(out))
        return out

    def tmclov_cg_full(self, conf_lx, kappa, cSW, mu, src_lx, niter, residue, anis=None):
        """inv_tmclovD_cg_eoprec: returns (sol_lx, iterations, lx |g5 Q x - b|^2/|b|^2)."""
        conf_lx, src_lx = _c(conf_lx), _c(src_lx)
        sol = np.empty((self.V, 4, 3, 2))
        res = ctypes.c_double(0)
        it = lib().orc_tmclov_cg_full(self._g, _p(conf_lx), float(kappa), *_anis(anis), float(cSW), float(mu),
                                      int(niter), float(residue), _p(src_lx), _p(sol), ctypes.byref(res))
        return sol, it, res.value

    def cgm(self, conf_lx, kappa, masses, residues, src, niter, anis=None):
        """Multi-shift CG on Q(+m)Q(-m): returns (sols[nshift], iterations, true residues)."""
        conf_lx, src = _c(conf_lx), _c(src)
        masses = np.ascontiguousarray(masses, np.float64)
        residues = np.ascontiguousarray(residues, np.float64)
        ns = len(masses)
        sols = np.empty((ns, self.V, 4, 3, 2))
        tr = np.empty(ns)
        it = lib().orc_cgm(self._g, _p(conf_lx), kappa, *_anis(anis), ns, _p(masses), _p(residues), int(niter),
                           _p(src), _p(sols), _p(tr))
        return sols, it, tr

    def plaquette(self, conf_lx):
        conf_lx = _c(conf_lx)
        return lib().orc_plaquette(self._g, _p(conf_lx))


# ------------------------------------------------------------------ reference runner

def ref_available() -> bool:
    return os.path.exists(REF_BIN)


def run_ref(op: str, T: int, L: int, arrays: dict, out_shape, threads: int | None = None, out_dtype=np.float64,
            binary: str | None = None, env: dict | None = None, **params):
    """Run the reference's own code (oracle/_ref/nissa_ref, or `binary`: the
    same driver linked otherwise) on raw arrays.

    ``arrays`` maps 'conf'/'in' to numpy arrays; returns (output array or None,
    JSON record, stdout text)."""
    exe = binary or REF_BIN
    if not os.path.exists(exe):
        raise RuntimeError("%s missing: run oracle.build_ref()" % exe)
    with tempfile.TemporaryDirectory() as d:
        argv = [exe, op, "T=%d" % T, "L=%d" % L]
        for k, a in arrays.items():
            path = os.path.join(d, k + ".bin")
            _c(a).tofile(path)
            argv.append("%s=%s" % (k, path))
        out_path = os.path.join(d, "out.bin")
        argv.append("out=" + out_path)
        for k, v in params.items():
            if isinstance(v, (list, tuple, np.ndarray)):
                v = ",".join(repr(float(x)) for x in v)
            argv.append("%s=%s" % (k, v))
        env = dict(os.environ, **(env or {}))
        env["NISSA_DO_NOT_TRAP_SIGNALS"] = "1"
        if threads:
            env["OMP_NUM_THREADS"] = str(threads)
        cp = subprocess.run(argv, cwd=d, env=env, capture_output=True, text=True)
        recs = [l for l in cp.stdout.splitlines() if l.startswith('{"op"')]
        if cp.returncode != 0 or not recs:
            raise RuntimeError("nissa_ref %s failed (%d): %s" % (op, cp.returncode, (cp.stdout + cp.stderr)[-2000:]))
        rec = json.loads(recs[-1])
        if "sample_iters" in params:
            # bounded sample: the reference ended through its non-convergence path
            return None, rec, cp.stdout
        out = None
        if out_shape is not None and os.path.exists(out_path):
            out = np.fromfile(out_path, out_dtype).reshape(out_shape)
        return out, rec, cp.stdout


def ref_geometry(T: int, L: int) -> dict:
    """The reference's own e/o tables (set_eo_geometry, geometry_eo.cpp:41-100)
    as its build leaves them for a T x L^3 lattice on one rank, keyed like
    Geom.tables(): parity, eo_of_lx, lx_of_eo, neighup_eo, neighdw_eo."""
    V = T * L ** 3
    Vh = V // 2
    flat, _, _ = run_ref("geom", T, L, {}, (11 * V,), out_dtype=np.int32)
    o = 0
    out = {}
    for k, shape in (("parity", (V,)), ("eo_of_lx", (V,)), ("lx_of_eo", (2, Vh)), ("neighup_eo", (2, Vh, 4)),
                     ("neighdw_eo", (2, Vh, 4))):
        n = int(np.prod(shape))
        out[k] = flat[o:o + n].reshape(shape).copy()
        o += n
    return out
