"""Time-slab decomposition on one GPU: the lattice split into 2, 4 or 8
slabs, each a context of its own (tms_create_slab), exchanging their faces
by device copies before every hop.  The slab hop and Schur operator must
equal the single-context operators on the whole lattice (the same arithmetic
in the same order: bit for bit), and the CG over the slabs, whose scalar
products are summed over slabs, must reach the single-context solution with
the same iteration count (+-1)."""
import numpy as np
import pytest

from nissa_b200 import Lattice
from nissa_b200 import slab as sl
from nissa_b200 import workload as wl
from conftest import rel

pytestmark = pytest.mark.gpu

KAPPA, MU = 0.1600, 0.0100


def _setup(T, L, nslab, bc_included=False, seed=51):
    import torch
    conf = wl.gauge_conf(T, L, 0.4, seed=seed)
    bounds = sl.slab_bounds(T, nslab)
    up = wl.apply_time_bc(conf, T, L, -1.0) if bc_included else conf
    slabs = []
    for (t0, n), c in zip(bounds, sl.split_conf(up, T, L, bounds)):
        s = sl.Slab(T, t0, n, L, bc_t=-1.0)
        s.upload_conf(torch.from_numpy(np.ascontiguousarray(c)).cuda(), bc_included=bc_included)
        slabs.append(s)
    return conf, bounds, slabs


@pytest.mark.parametrize("T,L,nslab", [(16, 8, 2), (16, 8, 4), (8, 4, 4), (12, 6, 2)])
def test_slab_hop_equals_single_context(cuda_device, T, L, nslab):
    import torch
    conf, bounds, slabs = _setup(T, L, nslab)
    Vh = T * L ** 3 // 2
    x = wl.random_spinor(Vh, 61)
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        ss = sl.SlabSet(slabs)
        xs = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in sl.split_eo(x, T, L, bounds)]
        for par in (0, 1):
            for anis in (None, 1.3):
                ref = lat.tmn2Deo_or_tmn2Doe_eos(par, x, anis=anis)
                got = np.concatenate([o.cpu().numpy() for o in ss.hop(par, xs, anis)])
                assert np.array_equal(got, ref), (par, anis, rel(got, ref))
    for s in slabs:
        s.close()


@pytest.mark.parametrize("bc_included", [False, True])
def test_slab_schur_square_equals_single_context(cuda_device, bc_included):
    import torch
    T, L, nslab = 16, 8, 4
    conf, bounds, slabs = _setup(T, L, nslab, bc_included)
    Vh = T * L ** 3 // 2
    x = wl.random_spinor(Vh, 62)
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        ref = lat.tmDkern_eoprec_square_eos(KAPPA, MU, x)
        ref1 = lat.tmDkern_eoprec_eos(KAPPA, -MU, x)
    ss = sl.SlabSet(slabs)
    xs = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in sl.split_eo(x, T, L, bounds)]
    got1 = np.concatenate([o.cpu().numpy() for o in ss.kern(KAPPA, -MU, xs)])
    got = np.concatenate([o.cpu().numpy() for o in ss.kern2(KAPPA, MU, xs)])
    assert np.array_equal(got1, ref1), rel(got1, ref1)
    assert np.array_equal(got, ref), rel(got, ref)
    for s in slabs:
        s.close()


@pytest.mark.parametrize("nslab", [2, 4])
def test_slab_cg_matches_single_context(cuda_device, nslab):
    import torch
    T, L = 16, 8
    conf, bounds, slabs = _setup(T, L, nslab, seed=52)
    Vh = T * L ** 3 // 2
    b = wl.random_spinor(Vh, 63)
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        ref, st = lat.inv_tmDkern_eoprec_square_eos_cg(KAPPA, MU, b, 10000, 1e-24)
    ss = sl.SlabSet(slabs)
    bs = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in sl.split_eo(b, T, L, bounds)]
    xs, it, tres = ss.cg(KAPPA, MU, bs, 10000, 1e-24)
    got = np.concatenate([o.cpu().numpy() for o in xs])
    assert tres < 1e-23
    assert abs(it - st["iterations"]) <= 1, (it, st["iterations"])
    assert rel(got, ref) < 1e-9
    for s in slabs:
        s.close()


def test_slab_arguments_checked(cuda_device):
    from nissa_b200 import TmError
    with pytest.raises(TmError):
        sl.Slab(16, 1, 8, 4)   # odd first slice
    with pytest.raises(TmError):
        sl.Slab(16, 10, 8, 4)  # beyond the lattice
    with sl.Slab(16, 0, 8, 4) as s:
        assert s.face == 4 ** 3 // 2
        with pytest.raises(TmError):
            s.pack(0, np.zeros((s.Vh, 4, 3, 2)))  # no conf yet
