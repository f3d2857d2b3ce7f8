"""Time-slab decomposition of the e/o twisted-mass operator and its CG.

A lattice of T time slices is split into slabs of consecutive slices (one per
GPU, or several contexts on one GPU); each slab is a context of the C ABI
(tms_create_slab) holding its own links.  Before every hop the slabs exchange
two faces around a ring:

  * slab k packs, from its input field, the forward face (its first slice,
    projected) for slab k-1 and the backward face (its last slice, projected
    and multiplied by its own time links) for slab k+1 (tms_slab_pack);
  * slab k's hop then reads the forward face of slab k+1 and the backward
    face of slab k-1 (tms_slab_hop, tms_slab_kern_half).

This is the reference's split of the lattice with a halo exchange before each
hop (base/field.cpp:11-56) and an all-reduce after each scalar product
(base/field.hpp:904), restricted to time and exchanging half spinors.  The
exchange is a ring of point-to-point transfers: in one process, copies between
the slabs' device buffers (several contexts on one or several GPUs); across
processes, torch.distributed send/recv (NCCL between GPUs, gloo on CPU), with
every rank taking the same steps in the same order.  Scalar products are
summed over slabs (in slab order within a process, by all_reduce across
processes).

Slab operators equal the single-context operators on the whole lattice bit
for bit; the slab CG follows cg_invert_template_threaded.hpp:17-150 (squared
relative residue, final true residual) with its sums taken over slabs.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .tm import Lattice, TmError, _Buf


class Slab:
    """Time slices [t0, t0 + T_loc) of a T x LX x LY x LZ lattice on one GPU."""

    def __init__(self, T: int, t0: int, T_loc: int, L: int, bc_t: float = -1.0, device: int = 0, LX=None, LY=None,
                 LZ=None):
        self.lib = _lib.load()
        self.T, self.t0, self.T_loc = T, t0, T_loc
        self.LX, self.LY, self.LZ = LX or L, LY or L, LZ or L
        self.V = T_loc * self.LX * self.LY * self.LZ
        self.Vh = self.V // 2
        self.device = device
        h = ctypes.c_void_p()
        st = self.lib.tms_create_slab(ctypes.byref(h), T, t0, T_loc, self.LX, self.LY, self.LZ, float(bc_t), device)
        if st != 0:
            raise TmError(st, "tms_create_slab(T=%d, t0=%d, T_loc=%d)" % (T, t0, T_loc))
        self.h = h
        self.face = int(self.lib.tms_slab_face_sites(self.h))
        # the generic checks of a context, through a view that borrows the handle
        # (only this object destroys it)
        self._lat = Lattice.__new__(Lattice)
        self._lat.lib, self._lat.h, self._lat._owner = self.lib, self.h, False
        self._lat.V, self._lat.Vh, self._lat.device = self.V, self.Vh, device

    def close(self):
        if getattr(self, "h", None):
            self.lib.tms_destroy(self.h)
            self.h = None
            self._lat.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload_conf(self, conf_slab_lx, bc_included: bool = False):
        """The slab's own links, lx layout (T_loc * LX * LY * LZ, 4, 3, 3, 2)."""
        self._lat.upload_conf(conf_slab_lx, "lx", bc_included)

    def _call(self, fn, what, *bufs_and_args):
        bufs = [b for b in bufs_and_args if isinstance(b, _Buf)]
        self._lat._mode(*bufs)
        args = [b.ptr if isinstance(b, _Buf) else b for b in bufs_and_args]
        self._lat._check(fn(self.h, *args), what)

    def new_face(self, like):
        import torch
        if hasattr(like, "device"):
            return torch.empty((self.face, 6, 2), dtype=torch.float64, device=like.device)
        return np.empty((self.face, 6, 2), np.float64)

    def pack(self, par_in: int, inp):
        """The forward face (for the previous slab) and the backward face (for the next one) of `inp`."""
        f, b = self.new_face(inp), self.new_face(inp)
        sh = (self.Vh, 4, 3, 2)
        self._call(self.lib.tms_slab_pack, "tms_slab_pack", int(par_in), _Buf(inp, sh), _Buf(f, (self.face, 6, 2),
                                                                                            out=True),
                   _Buf(b, (self.face, 6, 2), out=True))
        return f, b

    def _out(self, like, out):
        return self._lat._new_out(like, (self.Vh, 4, 3, 2)) if out is None else out

    def hop(self, par_out: int, inp, ghost_fwd, ghost_bwd, anis=None, out=None):
        """tmn2Deo_or_tmn2Doe_eos on the slab, given the faces received for `inp`."""
        o = self._out(inp, out)
        a = Lattice._anis(anis)
        sh, fs = (self.Vh, 4, 3, 2), (self.face, 6, 2)
        self._call(self.lib.tms_slab_hop, "tms_slab_hop", int(par_out), _Buf(inp, sh), _Buf(ghost_fwd, fs),
                   _Buf(ghost_bwd, fs), _Buf(o, sh, out=True), a[0], a[1])
        return o

    def kern_half(self, which: int, kappa: float, mu: float, inp, ghost_fwd, ghost_bwd, x=None, anis=None, out=None):
        """which 0: (1/2k + i mu g5)^-1 D_eo inp (even); 1: g5((1/2k + i mu g5) x - D_oe inp / 4) (odd)."""
        o = self._out(inp, out)
        a = Lattice._anis(anis)
        sh, fs = (self.Vh, 4, 3, 2), (self.face, 6, 2)
        xb = _Buf(x, sh) if x is not None else _Buf(None)
        bufs = [_Buf(inp, sh), _Buf(ghost_fwd, fs), _Buf(ghost_bwd, fs), xb, _Buf(o, sh, out=True)]
        self._lat._mode(*bufs)
        st = self.lib.tms_slab_kern_half(self.h, int(which), float(kappa), float(mu), bufs[0].ptr, bufs[1].ptr,
                                         bufs[2].ptr, xb.ptr, bufs[4].ptr, a[0], a[1])
        self._lat._check(st, "tms_slab_kern_half")
        return o


# ------------------------------------------------------------------ exchange
def ring_targets(k: int, n: int):
    """Slab k sends its forward face to slab k-1 and its backward face to slab k+1
    (mod n); it receives the forward face of k+1 and the backward face of k-1."""
    return (k - 1) % n, (k + 1) % n


def exchange_local(faces):
    """In one process: faces[k] = (fwd_k, bwd_k) packed by slab k; returns the
    ghosts (fwd of k+1, bwd of k-1) each slab's hop reads.  Faces on different
    devices are copied to the receiver's device."""
    n = len(faces)
    ghosts = []
    for k in range(n):
        fwd = faces[(k + 1) % n][0]
        bwd = faces[(k - 1) % n][1]
        dev = getattr(faces[k][0], "device", None)
        if dev is not None:
            fwd, bwd = fwd.to(dev, non_blocking=True), bwd.to(dev, non_blocking=True)
        ghosts.append((fwd, bwd))
    return ghosts


def exchange_dist(fwd, bwd, group=None):
    """Across processes (one slab per rank, ranks in slab order): send fwd to
    rank-1 and bwd to rank+1, receive the forward face of rank+1 and the
    backward face of rank-1.  Every rank posts its two receives and two sends
    and waits for all four (no rank waits on an unposted transfer)."""
    import torch
    import torch.distributed as dist
    n = dist.get_world_size(group)
    k = dist.get_rank(group)
    prev, nxt = ring_targets(k, n)
    gf, gb = torch.empty_like(fwd), torch.empty_like(bwd)
    if n == 1:
        gf.copy_(fwd)
        gb.copy_(bwd)
        return gf, gb
    ops = [dist.P2POp(dist.irecv, gf, nxt, group), dist.P2POp(dist.irecv, gb, prev, group),
           dist.P2POp(dist.isend, fwd, prev, group), dist.P2POp(dist.isend, bwd, nxt, group)]
    for r in dist.batch_isend_irecv(ops):
        r.wait()
    return gf, gb


# ------------------------------------------------------------------ operators and CG
class SlabSet:
    """The slabs of one lattice driven together: either all slabs in this
    process (`slabs` a list, exchange by copies) or this rank's slab of a
    torch.distributed group (`slabs` a one-element list, `group` set)."""

    def __init__(self, slabs, group=None, distributed: bool = False):
        self.slabs = list(slabs)
        self.group = group
        self.distributed = distributed

    def _exchange(self, faces):
        if self.distributed:
            return [exchange_dist(faces[0][0], faces[0][1], self.group)]
        return exchange_local(faces)

    def hop(self, par_out, fields, anis=None):
        faces = [s.pack(1 - par_out, f) for s, f in zip(self.slabs, fields)]
        ghosts = self._exchange(faces)
        return [s.hop(par_out, f, g[0], g[1], anis) for s, f, g in zip(self.slabs, fields, ghosts)]

    def kern(self, kappa, mu, x, anis=None):
        """tmDkern_eoprec_eos on odd fields x (one per slab)."""
        faces = [s.pack(1, f) for s, f in zip(self.slabs, x)]
        ghosts = self._exchange(faces)
        te = [s.kern_half(0, kappa, mu, f, g[0], g[1], anis=anis) for s, f, g in zip(self.slabs, x, ghosts)]
        faces = [s.pack(0, f) for s, f in zip(self.slabs, te)]
        ghosts = self._exchange(faces)
        return [s.kern_half(1, kappa, mu, t, g[0], g[1], x=f, anis=anis)
                for s, t, g, f in zip(self.slabs, te, ghosts, x)]

    def kern2(self, kappa, mu, x, anis=None):
        """tmDkern_eoprec_square_eos: K(+mu) K(-mu) x, as the single-context operator."""
        return self.kern(kappa, mu, self.kern(kappa, -mu, x, anis), anis)

    def dot(self, a, b):
        """Re(a, b) over all slabs: per-slab FP64 sums, added in slab order."""
        import torch
        parts = [float(torch.sum(x * y)) for x, y in zip(a, b)]
        if self.distributed:
            import torch.distributed as dist
            t = torch.tensor([parts[0]], dtype=torch.float64)
            if a[0].is_cuda and dist.get_backend(self.group) == "nccl":
                t = t.to(a[0].device)
            dist.all_reduce(t, group=self.group)
            return float(t.item())
        s = 0.0
        for v in parts:
            s += v
        return s

    def cg(self, kappa, mu, src, niter, residue, anis=None):
        """inv_tmDkern_eoprec_square_eos_cg over the slabs (FP64): solves
        K(+mu)K(-mu) sol = src; stops when |r|^2 < residue |src|^2, then checks
        the true residual.  Returns (sol, iterations, true |r|^2 / |src|^2)."""
        import torch
        b2 = self.dot(src, src)
        if not (b2 > 0):
            raise TmError(8, "invalid source norm %g" % b2)
        x = [torch.zeros_like(s) for s in src]
        r = [s.clone() for s in src]
        p = [s.clone() for s in src]
        rr = b2
        target = residue * b2
        it = 0
        while it < niter:
            s = self.kern2(kappa, mu, p, anis)
            pap = self.dot(p, s)
            alpha = rr / pap
            for k in range(len(x)):
                x[k].add_(p[k], alpha=alpha)
                r[k].sub_(s[k], alpha=alpha)
            rr_new = self.dot(r, r)
            it += 1
            if rr_new < target:
                break
            beta = rr_new / rr
            for k in range(len(p)):
                p[k].mul_(beta).add_(r[k])
            rr = rr_new
        ax = self.kern2(kappa, mu, x, anis)
        res = [s_ - a_ for s_, a_ in zip(src, ax)]
        return x, it, self.dot(res, res) / b2


def split_conf(conf_lx, T: int, L: int, bounds):
    """The lx links of each slab [t0, t0 + T_loc) of a T x L^3 conf (V, 4, 3, 3, 2)."""
    c = conf_lx.reshape((T, L ** 3) + tuple(conf_lx.shape[1:]))
    return [c[t0:t0 + n].reshape((n * L ** 3,) + tuple(conf_lx.shape[1:])) for t0, n in bounds]


def split_eo(field_eo, T: int, L: int, bounds):
    """The e/o sites of each slab: e/o index = lx >> 1 numbers a slab's sites
    consecutively from t0 * L^3 / 2."""
    h = L ** 3 // 2
    return [field_eo[t0 * h:(t0 + n) * h] for t0, n in bounds]


def slab_bounds(T: int, nslab: int):
    """Equal even slabs: [(t0, T_loc)]."""
    if T % nslab or (T // nslab) % 2:
        raise ValueError("T=%d does not split into %d even slabs" % (T, nslab))
    n = T // nslab
    return [(k * n, n) for k in range(nslab)]
