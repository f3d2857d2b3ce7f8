"""Host-side mirror of the reference's twisted-mass interface.

Method names, argument meanings and error behaviour follow the reference
library nissa (paths relative to its src/):

  tmn2Deo_or_tmn2Doe_eos          dirac_operators/tmD_eoprec/dirac_operator_tmD_eoprec_portable.hpp:33-169
  tmDee_or_oo_eos / inv_...       dirac_operator_tmD_eoprec_portable.hpp:171-222
  tmDkern_eoprec_eos              dirac_operator_tmD_eoprec_portable.cpp:36-51
  tmDkern_eoprec_square_eos       dirac_operator_tmD_eoprec_portable.cpp:54-65
  apply_tmQ / apply_tmQ2          dirac_operators/tmQ/dirac_operator_tmQ_portable.cpp:29-176, tmQ2/dirac_operator_tmQ2.cpp
  inv_tmDkern_eoprec_square_eos_cg inverters/twisted_mass/cg_invert_tmD_eoprec.cpp:61-78
  inv_tmD_cg_eoprec               inverters/twisted_mass/cg_invert_tmD_eoprec.cpp:152-213

The reference CRASHes on a non-converged solve, a NaN or an invalid source
norm; here the same conditions raise TmError (with the status code of the C
ABI).  ``residue`` is the squared relative residue, as in the reference.
Every call goes through the C ABI of libtmsolve.so: there is no CPU path.

Arrays are numpy float64 (host) or torch float64 tensors (host or CUDA) in the
reference's CPU layout: eo spinor (Vh, 4, 3, 2), lx spinor (V, 4, 3, 2),
lx conf (V, 4, 3, 3, 2), eo conf (2, Vh, 4, 3, 3, 2).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib

STATUS = {0: "OK", 1: "NOT_CONVERGED", 2: "NAN", 3: "BAD_ARG", 4: "OOM", 5: "TIMEOUT", 6: "CUDA_ERROR",
          7: "NO_CONF", 8: "INVALID_SOURCE"}
PRECISION = {"double": 0, "single": 1, "half": 2}


class TmError(RuntimeError):
    def __init__(self, status: int, message: str, stats: dict | None = None, result=None):
        super().__init__("%s: %s" % (STATUS.get(status, status), message))
        self.status = status
        self.stats = stats
        self.result = result


def _is_torch(a):
    return type(a).__module__.startswith("torch")


class _Buf:
    """Pointer + pointer-mode of an input/output array."""

    def __init__(self, a, shape=None, out=False):
        self.keep = None
        if a is None:
            self.ptr, self.device = None, False
            return
        if _is_torch(a):
            if not a.is_contiguous() or str(a.dtype) != "torch.float64":
                raise TypeError("torch tensors must be contiguous float64")
            self.ptr, self.device = a.data_ptr(), a.is_cuda
            self.keep = a
        else:
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
                if out:
                    raise TypeError("output arrays must be contiguous float64 numpy arrays")
                a = np.ascontiguousarray(a, dtype=np.float64)
            self.ptr, self.device = a.ctypes.data, False
            self.keep = a
        if shape is not None and int(np.prod(shape)) != (a.numel() if _is_torch(a) else a.size):
            raise ValueError("array has %d elements, expected shape %s" % (
                a.numel() if _is_torch(a) else a.size, tuple(shape)))


class BatchSession:
    """Continuous batching on one lattice (tms_batch_* of the C ABI): up to
    ``nslots`` inv_tmD_cg_eoprec solves in flight, each with its own kappa,
    mu and residue; new right-hand sides are submitted into free slots while
    others keep iterating.  Driven by one host thread."""

    def __init__(self, lattice: "Lattice", nslots: int, precision: str = "single", anis=None):
        self.lat = lattice
        self.lib = lattice.lib
        self.nslots = nslots
        a = Lattice._anis(anis)
        h = ctypes.c_void_p()
        st = self.lib.tms_batch_open(lattice.h, int(nslots), PRECISION[precision], a[0], a[1], ctypes.byref(h))
        lattice._check(st, "tms_batch_open")
        self.h = h
        self._fin = (ctypes.c_int * nslots)()
        self._keep = {}

    def free_slots(self):
        return [k for k in range(self.nslots) if k not in self._keep]

    def submit(self, slot: int, source_lx, kappa: float, mu: float, niter: int, residue: float):
        b = _Buf(source_lx, (self.lat.V, 4, 3, 2))
        self.lat._mode(b)
        st = self.lib.tms_batch_submit(self.h, int(slot), b.ptr, float(kappa), float(mu), int(niter), float(residue))
        self.lat._check(st, "tms_batch_submit")
        self._keep[slot] = b

    def step(self):
        """One block of lock-step iterations; returns the slots that finished."""
        nf = ctypes.c_int(0)
        st = self.lib.tms_batch_step(self.h, self._fin, ctypes.byref(nf))
        self.lat._check(st, "tms_batch_step")
        return [k for k in range(self.nslots) if self._fin[k]]

    def collect(self, slot: int, out=None):
        """Solution of a finished slot (and frees it): returns (sol, stats)."""
        like = self._keep[slot].keep
        sol = self.lat._new_out(like, (self.lat.V, 4, 3, 2)) if out is None else out
        o = _Buf(sol, (self.lat.V, 4, 3, 2), out=True)
        self.lat._mode(o)
        stats = _lib.Stats()
        st = self.lib.tms_batch_collect(self.h, int(slot), o.ptr, ctypes.byref(stats))
        del self._keep[slot]
        if st not in (0, 1, 2):
            self.lat._check(st, "tms_batch_collect")
        d = stats.as_dict()
        d["status"] = st
        return sol, d

    def close(self):
        if getattr(self, "h", None):
            self.lib.tms_batch_close(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class Lattice:
    """One T x LX x LY x LZ lattice with a resident gauge configuration on one GPU.

    The per-instance counterpart of the reference's initGrid(T, L) plus its
    e/o geometry (base/init.cpp:563-798, geometry/geometry_eo.cpp:41-100).
    ``bc_t`` is the time boundary sign (-1 antiperiodic), applied in the
    stencil when a hop crosses the time boundary."""

    def __init__(self, T: int, L: int, bc_t: float = -1.0, device: int = 0, LX=None, LY=None, LZ=None):
        self.lib = _lib.load()
        self.T = T
        self.LX, self.LY, self.LZ = LX or L, LY or L, LZ or L
        self.V = T * self.LX * self.LY * self.LZ
        self.Vh = self.V // 2
        self.bc_t = bc_t
        self.device = device
        h = ctypes.c_void_p()
        st = self.lib.tms_create4(ctypes.byref(h), T, self.LX, self.LY, self.LZ, float(bc_t), device)
        if st != 0:
            raise TmError(st, "tms_create(T=%d, L=%s)" % (T, (self.LX, self.LY, self.LZ)))
        self.h = h

    def close(self):
        # a view that borrows another object's context (_owner False) never destroys it
        if getattr(self, "h", None) and getattr(self, "_owner", True):
            self.lib.tms_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ------------------------------------------------------------ helpers
    def _check(self, st, what, stats=None, result=None):
        if st != 0:
            msg = self.lib.tms_last_error(self.h)
            raise TmError(st, "%s: %s" % (what, msg.decode() if msg else ""), stats, result)

    def _mode(self, *bufs):
        dev = [b.device for b in bufs if b.ptr is not None]
        if dev and any(d != dev[0] for d in dev):
            raise TypeError("mixing host and device arrays in one call")
        mode = 1 if (dev and dev[0]) else 0
        if mode:
            # the library reads device inputs on its own stream: the torch work
            # that produced them (on torch's current stream) must be complete
            import torch
            torch.cuda.current_stream(self.device).synchronize()
        self.lib.tms_set_pointer_mode(self.h, mode)
        return mode

    def _new_out(self, like, shape):
        if like is not None and _is_torch(like):
            import torch
            return torch.empty(shape, dtype=torch.float64, device=like.device)
        return np.empty(shape, np.float64)

    @staticmethod
    def _anis(anis):
        return (0, 1.0) if anis is None else (1, float(anis))

    # --------------------------------------------------------------- conf
    def upload_conf(self, conf, layout: str = "lx", bc_included: bool = False):
        """Make ``conf`` the resident gauge configuration.  With bc_included the
        links already carry the time boundary sign (the form in which the
        reference's operators see them); it is divided out and re-applied in the
        stencil."""
        shape = (self.V, 4, 3, 3, 2) if layout == "lx" else (2, self.Vh, 4, 3, 3, 2)
        b = _Buf(conf, shape)
        self._mode(b)
        st = self.lib.tms_conf_upload(self.h, b.ptr, 0 if layout == "lx" else 1, 1 if bc_included else 0)
        self._check(st, "tms_conf_upload")

    def read_ildg(self, path: str) -> np.ndarray:
        """read_ildg_gauge_conf (io/reader.hpp:75-99): the conf of an ILDG file in the
        reference's lx layout (V, 4, 3, 3, 2), periodic links as stored."""
        conf = np.empty((self.V, 4, 3, 3, 2), np.float64)
        self._check(self.lib.tms_read_ildg(self.h, os.fsencode(path), conf.ctypes.data), "tms_read_ildg")
        return conf

    def write_ildg(self, path: str, conf, precision: int = 64):
        """Write an lx conf (V, 4, 3, 3, 2) as an ILDG file (32- or 64-bit big-endian)."""
        c = np.ascontiguousarray(np.asarray(conf, np.float64).reshape(self.V, 4, 3, 3, 2))
        self._check(self.lib.tms_write_ildg(self.h, os.fsencode(path), c.ctypes.data, int(precision)),
                    "tms_write_ildg")

    def load_ildg(self, path: str, bc_included: bool = False):
        """Read an ILDG file and make it the resident configuration."""
        self._check(self.lib.tms_conf_load_ildg(self.h, os.fsencode(path), 1 if bc_included else 0),
                    "tms_conf_load_ildg")

    def plaquette(self, with_bc: bool = False) -> float:
        """global_plaquette_lx_conf of the resident conf, on the device (FP64)."""
        p = ctypes.c_double()
        self._check(self.lib.tms_conf_plaquette(self.h, 1 if with_bc else 0, ctypes.byref(p)), "tms_conf_plaquette")
        return p.value

    @property
    def conf_is_su3(self) -> bool:
        return bool(self.lib.tms_conf_is_su3(self.h))

    def geometry_tables(self):
        V = self.V
        t = dict(parity=np.empty(V, np.int32), eo_of_lx=np.empty(V, np.int32), lx_of_eo=np.empty((2, V // 2), np.int32),
                 neighup_eo=np.empty((2, V // 2, 4), np.int32), neighdw_eo=np.empty((2, V // 2, 4), np.int32))
        st = self.lib.tms_geometry_tables(self.h, *[t[k].ctypes.data for k in ("parity", "eo_of_lx", "lx_of_eo",
                                                                                   "neighup_eo", "neighdw_eo")])
        self._check(st, "tms_geometry_tables")
        return t

    # ---------------------------------------------------------- operators
    def _unary(self, fn, args, inp, shape, out=None):
        i = _Buf(inp, shape)
        o = self._new_out(inp, shape) if out is None else out
        ob = _Buf(o, shape, out=True)
        self._mode(i, ob)
        self._check(fn(self.h, *args(i.ptr, ob.ptr)), fn.__name__)
        return o

    def tmn2Deo_or_tmn2Doe_eos(self, par_out: int, inp, anis=None, out=None):
        """out (parity par_out) = -2 x hopping of inp (the opposite parity)."""
        a = self._anis(anis)
        return self._unary(self.lib.tms_hop_eo, lambda i, o: (int(par_out), i, o, a[0], a[1]), inp,
                           (self.Vh, 4, 3, 2), out)

    def tmDee_or_oo_eos(self, kappa, mu, inp, out=None):
        return self._unary(self.lib.tms_tmDee, lambda i, o: (kappa, mu, i, o), inp, (self.Vh, 4, 3, 2), out)

    def inv_tmDee_or_oo_eos(self, kappa, mu, inp, out=None):
        return self._unary(self.lib.tms_inv_tmDee, lambda i, o: (kappa, mu, i, o), inp, (self.Vh, 4, 3, 2), out)

    def tmDkern_eoprec_eos(self, kappa, mu, inp, anis=None, out=None):
        a = self._anis(anis)
        return self._unary(self.lib.tms_kern_eoprec, lambda i, o: (kappa, a[0], a[1], mu, i, o), inp,
                           (self.Vh, 4, 3, 2), out)

    def tmDkern_eoprec_square_eos(self, kappa, mu, inp, anis=None, out=None):
        a = self._anis(anis)
        return self._unary(self.lib.tms_kern_eoprec_square, lambda i, o: (kappa, a[0], a[1], mu, i, o), inp,
                           (self.Vh, 4, 3, 2), out)

    def apply_tmQ(self, kappa, mu, inp, anis=None, out=None):
        a = self._anis(anis)
        return self._unary(self.lib.tms_apply_tmQ, lambda i, o: (kappa, a[0], a[1], mu, i, o), inp,
                           (self.V, 4, 3, 2), out)

    def apply_tmQ2(self, kappa, mu, inp, anis=None, out=None):
        a = self._anis(anis)
        return self._unary(self.lib.tms_apply_tmQ2, lambda i, o: (kappa, a[0], a[1], mu, i, o), inp,
                           (self.V, 4, 3, 2), out)

    # ---------------------------------------------------- instrumentation
    @property
    def launch_count(self) -> int:
        """CUDA kernels launched by this lattice's context so far."""
        return int(self.lib.tms_launch_count(self.h))

    @property
    def hop_stage_timeouts(self) -> int:
        """Tiles of the staged hop (launch shape 7) whose wait for their copies gave up (0 normally)."""
        return int(self.lib.tms_hop_stage_timeouts(self.h))

    def set_tuning(self, key: str, value: float):
        """Set a tuning knob of the C ABI (see tms_set_tuning in include/tmsolve.h)."""
        self._check(self.lib.tms_set_tuning(self.h, key.encode(), float(value)), "tms_set_tuning")

    def get_tuning(self, key: str):
        """Current value of a tuning knob (an int where the knob is integral)."""
        v = ctypes.c_double()
        self._check(self.lib.tms_get_tuning(self.h, key.encode(), ctypes.byref(v)), "tms_get_tuning")
        return int(v.value) if v.value == int(v.value) and not key.startswith(("reliable_delta", "cgm_floor")) \
            else v.value

    def bench_hop(self, precision="double", variant=0, nrep=20, flush=True):
        """Mean device time (ms) of one e/o hopping launch and its algorithmic bytes."""
        ms, by = ctypes.c_double(), ctypes.c_double()
        st = self.lib.tms_bench_hop(self.h, PRECISION[precision], int(variant), int(nrep), 1 if flush else 0,
                                    ctypes.byref(ms), ctypes.byref(by))
        self._check(st, "tms_bench_hop")
        return ms.value, by.value

    def bench_hop_batched(self, precision="single", nrhs=12, nrep=20, flush=True):
        """Mean device time (ms) of one batched hopping launch and its algorithmic bytes."""
        ms, by = ctypes.c_double(), ctypes.c_double()
        st = self.lib.tms_bench_hop_batched(self.h, PRECISION[precision], int(nrhs), int(nrep), 1 if flush else 0,
                                            ctypes.byref(ms), ctypes.byref(by))
        self._check(st, "tms_bench_hop_batched")
        return ms.value, by.value

    # ------------------------------------------------------------ solvers
    def inv_tmDkern_eoprec_square_eos_cg(self, kappa, mu, source, niter, residue, guess=None, anis=None,
                                         precision="double", out=None, raise_on_error=True):
        """Solve K(+mu)K(-mu) sol = source on odd sites.  Returns (sol, stats)."""
        shape = (self.Vh, 4, 3, 2)
        s, g = _Buf(source, shape), _Buf(guess, shape)
        sol = self._new_out(source, shape) if out is None else out
        o = _Buf(sol, shape, out=True)
        self._mode(s, g, o)
        stats = _lib.Stats()
        a = self._anis(anis)
        st = self.lib.tms_cg_eoprec_square(self.h, o.ptr, g.ptr, s.ptr, kappa, a[0], a[1], mu, int(niter),
                                           float(residue), PRECISION[precision], ctypes.byref(stats))
        if raise_on_error:
            self._check(st, "inv_tmDkern_eoprec_square_eos_cg", stats.as_dict(), sol)
        return sol, stats.as_dict()

    def inv_tmQ2_cg(self, kappa, m, source_lx, niter, residue, guess=None, anis=None, precision="double", out=None,
                    raise_on_error=True):
        """Full-lattice CG on Q(+m)Q(-m) (lx spinors).  Returns (sol, stats)."""
        shape = (self.V, 4, 3, 2)
        s, g = _Buf(source_lx, shape), _Buf(guess, shape)
        sol = self._new_out(source_lx, shape) if out is None else out
        o = _Buf(sol, shape, out=True)
        self._mode(s, g, o)
        stats = _lib.Stats()
        a = self._anis(anis)
        st = self.lib.tms_cg_tmQ2(self.h, o.ptr, g.ptr, s.ptr, kappa, a[0], a[1], m, int(niter), float(residue),
                                  PRECISION[precision], ctypes.byref(stats))
        if raise_on_error:
            self._check(st, "inv_tmQ2_cg", stats.as_dict(), sol)
        return sol, stats.as_dict()

    def inv_tmQ2_cgm(self, kappa, masses, source_lx, niter, residues, anis=None, precision="double", out=None,
                     raise_on_error=True):
        """Multi-shift CG: (Q_W^2 + m_k^2) sol_k = source for every mass.  Returns (sols, [stats])."""
        shape = (self.V, 4, 3, 2)
        nm = len(masses)
        residues = np.broadcast_to(np.asarray(residues, np.float64), (nm,)).copy()
        masses = np.ascontiguousarray(masses, np.float64)
        s = _Buf(source_lx, shape)
        if out is None:
            out = [self._new_out(source_lx, shape) for _ in range(nm)]
        obufs = [_Buf(o, shape, out=True) for o in out]
        self._mode(s, *obufs)
        ptrs = (ctypes.c_void_p * nm)(*[b.ptr for b in obufs])
        stats = (_lib.Stats * nm)()
        a = self._anis(anis)
        st = self.lib.tms_cgm_tmQ2(self.h, ctypes.cast(ptrs, ctypes.c_void_p), s.ptr, kappa, a[0], a[1],
                                   masses.ctypes.data, nm, int(niter), residues.ctypes.data, PRECISION[precision],
                                   ctypes.cast(stats, ctypes.c_void_p))
        sd = [x.as_dict() for x in stats]
        if raise_on_error:
            self._check(st, "inv_tmQ2_cgm", sd, out)
        return out, sd

    def inv_tmD_cg_eoprec_batched(self, kappa, mus, sources_lx, niter, residues, anis=None, precision="double",
                                  out=None, raise_on_error=True):
        """inv_tmD_cg_eoprec for several sources (one twisted mass each) solved
        together.  Returns (sols, [stats])."""
        shape = (self.V, 4, 3, 2)
        nr = len(sources_lx)
        mus = np.broadcast_to(np.asarray(mus, np.float64), (nr,)).copy()
        residues = np.broadcast_to(np.asarray(residues, np.float64), (nr,)).copy()
        sb = [_Buf(x, shape) for x in sources_lx]
        if out is None:
            out = [self._new_out(sources_lx[0], shape) for _ in range(nr)]
        ob = [_Buf(o, shape, out=True) for o in out]
        self._mode(*sb, *ob)
        sp = (ctypes.c_void_p * nr)(*[b.ptr for b in sb])
        op = (ctypes.c_void_p * nr)(*[b.ptr for b in ob])
        stats = (_lib.Stats * nr)()
        a = self._anis(anis)
        st = self.lib.tms_cg_eoprec_batched(self.h, nr, ctypes.cast(op, ctypes.c_void_p),
                                            ctypes.cast(sp, ctypes.c_void_p), kappa, a[0], a[1], mus.ctypes.data,
                                            int(niter), residues.ctypes.data, PRECISION[precision],
                                            ctypes.cast(stats, ctypes.c_void_p))
        sd = [x.as_dict() for x in stats]
        if raise_on_error:
            self._check(st, "inv_tmD_cg_eoprec_batched", sd, out)
        return out, sd

    def inv_tmD_cg_eoprec_columns(self, kappa, mu, sources_lx, niter, residue, anis=None, precision="double",
                                  out=None, raise_on_error=True):
        """inv_tmD_cg_eoprec for several sources one after the other; with host
        buffers the copies of the neighbouring columns overlap each solve.
        Returns (sols, [stats])."""
        shape = (self.V, 4, 3, 2)
        nc = len(sources_lx)
        sb = [_Buf(x, shape) for x in sources_lx]
        if out is None:
            out = [self._new_out(sources_lx[0], shape) for _ in range(nc)]
        ob = [_Buf(o, shape, out=True) for o in out]
        self._mode(*sb, *ob)
        sp = (ctypes.c_void_p * nc)(*[b.ptr for b in sb])
        op = (ctypes.c_void_p * nc)(*[b.ptr for b in ob])
        stats = (_lib.Stats * nc)()
        a = self._anis(anis)
        st = self.lib.tms_cg_eoprec_columns(self.h, nc, ctypes.cast(op, ctypes.c_void_p),
                                            ctypes.cast(sp, ctypes.c_void_p), kappa, a[0], a[1], mu, int(niter),
                                            float(residue), PRECISION[precision], ctypes.cast(stats, ctypes.c_void_p))
        sd = [x.as_dict() for x in stats]
        if raise_on_error:
            self._check(st, "inv_tmD_cg_eoprec_columns", sd, out)
        return out, sd

    def batch_session(self, nslots: int, precision: str = "single", anis=None) -> BatchSession:
        return BatchSession(self, nslots, precision, anis)

    # ------------------------------------------------- around a propagator solve
    def rotate_twisted(self, r: int, inp, out=None):
        """safe_dirac_prod_spincolor with P- (r=0) or P+ (r=1) on an lx spinor."""
        return self._unary(self.lib.tms_rotate_twisted, lambda i, o: (int(r), i, o), inp, (self.V, 4, 3, 2), out)

    def get_qprop(self, r: int, kappa, mu, source_lx, residue, cSW=0.0, rotate_source=True, niter=1000000,
                  anis=None, precision="double", out=None, raise_on_error=True):
        """get_qprop (projects/ib/prop.cpp:41-112): P(r) source -> solve -> P(r) sink.  Returns (prop, stats)."""
        shape = (self.V, 4, 3, 2)
        s = _Buf(source_lx, shape)
        sol = self._new_out(source_lx, shape) if out is None else out
        o = _Buf(sol, shape, out=True)
        self._mode(s, o)
        stats = _lib.Stats()
        a = self._anis(anis)
        st = self.lib.tms_get_qprop(self.h, int(r), 1 if rotate_source else 0, kappa, a[0], a[1], float(cSW), mu,
                                    int(niter), float(residue), PRECISION[precision], s.ptr, o.ptr,
                                    ctypes.byref(stats))
        if raise_on_error:
            self._check(st, "get_qprop", stats.as_dict(), sol)
        return sol, stats.as_dict()

    def reconstruct_tm_doublet(self, kappa, mu, inp, anis=None):
        """(outminus, outplus) = (Q(+mu) in, Q(+mu) in - 2 i mu in)."""
        shape = (self.V, 4, 3, 2)
        i = _Buf(inp, shape)
        om, op = self._new_out(inp, shape), self._new_out(inp, shape)
        bm, bp = _Buf(om, shape, out=True), _Buf(op, shape, out=True)
        self._mode(i, bm, bp)
        a = self._anis(anis)
        self._check(self.lib.tms_reconstruct_tm_doublet(self.h, kappa, a[0], a[1], mu, i.ptr, bm.ptr, bp.ptr),
                    "reconstruct_tm_doublet")
        return om, op

    # ------------------------------------------------------ twisted clover
    def clover_term(self, cSW: float):
        """clover_term(Cl, cSW, conf): computed and kept on the device for the resident conf."""
        self._check(self.lib.tms_clover_term(self.h, float(cSW)), "tms_clover_term")

    def clover_get(self) -> np.ndarray:
        """The kept clover term in the reference's lx layout (V, 4, 3, 3, 2), on the host."""
        out = np.empty((self.V, 4, 3, 3, 2), np.float64)
        b = _Buf(out, out.shape, out=True)
        self._mode(b)
        self._check(self.lib.tms_clover_get(self.h, b.ptr), "tms_clover_get")
        return out

    def tmclovDee_or_oo_eos(self, par, kappa, mu, dag, inp, out=None):
        return self._unary(self.lib.tms_tmclovDee, lambda i, o: (int(par), kappa, mu, int(bool(dag)), i, o), inp,
                           (self.Vh, 4, 3, 2), out)

    def inv_tmclovDee_or_oo_eos(self, kappa, mu, dag, inp, out=None):
        return self._unary(self.lib.tms_inv_tmclovDee, lambda i, o: (kappa, mu, int(bool(dag)), i, o), inp,
                           (self.Vh, 4, 3, 2), out)

    def tmclovDkern_eoprec_eos(self, kappa, mu, dag, inp, anis=None, out=None):
        a = self._anis(anis)
        return self._unary(self.lib.tms_tmclovDkern_eoprec, lambda i, o: (kappa, a[0], a[1], mu, int(bool(dag)), i, o),
                           inp, (self.Vh, 4, 3, 2), out)

    def tmclovDkern_eoprec_square_eos(self, kappa, mu, inp, anis=None, out=None):
        a = self._anis(anis)
        return self._unary(self.lib.tms_tmclovDkern_eoprec_square, lambda i, o: (kappa, a[0], a[1], mu, i, o), inp,
                           (self.Vh, 4, 3, 2), out)

    def apply_tmclovQ(self, kappa, mu, inp, anis=None, out=None):
        a = self._anis(anis)
        return self._unary(self.lib.tms_apply_tmclovQ, lambda i, o: (kappa, a[0], a[1], mu, i, o), inp,
                           (self.V, 4, 3, 2), out)

    def inv_tmclovDkern_eoprec_square_eos_cg(self, kappa, mu, source, niter, residue, guess=None, anis=None,
                                             precision="double", out=None, raise_on_error=True):
        """Solve K_clov(false)K_clov(true) sol = source on odd sites (kept clover term).  Returns (sol, stats)."""
        shape = (self.Vh, 4, 3, 2)
        s, g = _Buf(source, shape), _Buf(guess, shape)
        sol = self._new_out(source, shape) if out is None else out
        o = _Buf(sol, shape, out=True)
        self._mode(s, g, o)
        stats = _lib.Stats()
        a = self._anis(anis)
        st = self.lib.tms_cg_tmclov_eoprec_square(self.h, o.ptr, g.ptr, s.ptr, kappa, a[0], a[1], mu, int(niter),
                                                  float(residue), PRECISION[precision], ctypes.byref(stats))
        if raise_on_error:
            self._check(st, "inv_tmclovDkern_eoprec_square_eos_cg", stats.as_dict(), sol)
        return sol, stats.as_dict()

    def inv_tmclovD_cg_eoprec(self, kappa, cSW, mu, source_lx, niter, residue, anis=None, precision="double",
                              out=None, raise_on_error=True):
        """Full solve of the twisted-clover operator (lx spinors) via e/o preconditioning.  Returns (sol, stats)."""
        shape = (self.V, 4, 3, 2)
        s = _Buf(source_lx, shape)
        sol = self._new_out(source_lx, shape) if out is None else out
        o = _Buf(sol, shape, out=True)
        self._mode(s, o)
        stats = _lib.Stats()
        a = self._anis(anis)
        st = self.lib.tms_cg_tmclov_eoprec(self.h, o.ptr, s.ptr, kappa, a[0], a[1], float(cSW), mu, int(niter),
                                           float(residue), PRECISION[precision], ctypes.byref(stats))
        if raise_on_error:
            self._check(st, "inv_tmclovD_cg_eoprec", stats.as_dict(), sol)
        return sol, stats.as_dict()

    def inv_tmD_cg_eoprec(self, kappa, mu, source_lx, niter, residue, anis=None, precision="double", out=None,
                          raise_on_error=True, guess_Koo=None):
        """Full solve D_tm sol = source (lx spinors) via e/o preconditioning,
        the Eq. (9) CG started from guess_Koo (odd sites) when given.  Returns (sol, stats)."""
        shape = (self.V, 4, 3, 2)
        s = _Buf(source_lx, shape)
        sol = self._new_out(source_lx, shape) if out is None else out
        o = _Buf(sol, shape, out=True)
        g = _Buf(guess_Koo, (self.Vh, 4, 3, 2))
        self._mode(s, o, g)
        stats = _lib.Stats()
        a = self._anis(anis)
        st = self.lib.tms_cg_eoprec_guess(self.h, o.ptr, g.ptr, s.ptr, kappa, a[0], a[1], mu, int(niter),
                                          float(residue), PRECISION[precision], ctypes.byref(stats))
        if raise_on_error:
            self._check(st, "inv_tmD_cg_eoprec", stats.as_dict(), sol)
        return sol, stats.as_dict()
