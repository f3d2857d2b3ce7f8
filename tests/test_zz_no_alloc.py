"""The allocation-free hopping entry point, tms_hop_eo_noalloc.

It exists for callers that cannot let a library allocate device memory: an
application whose device memory is all owned by its own pool (as the
reference's memory manager owns it) and must not see allocations appear
behind its back, or code in a phase where a cudaMalloc/cudaFree would
synchronise the whole device.  It keeps its scratch in one fixed device array
inside the library, so it is checked here against the ordinary entry point
tms_hop_eo (same kernel, scratch allocated by a context), through the C ABI,
on two calls in a row, which share and reuse that array.

This file is collected last on purpose: it must pass alone in a fresh process
and after every other test.
"""
import ctypes

import numpy as np
import pytest

from nissa_b200 import Lattice, _lib
from nissa_b200 import workload as wl
from conftest import rel

pytestmark = pytest.mark.gpu

TOL = 1e-14  # the FP64 operator tolerance used by every other operator test


def _noalloc(lib, T, L, conf_dev, par_out, in_dev, out_dev, anis=None, layout=0, flags=0):
    err = ctypes.create_string_buffer(256)
    st = lib.tms_hop_eo_noalloc(T, L, -1.0, conf_dev.data_ptr(), layout, flags, par_out, in_dev.data_ptr(),
                                out_dev.data_ptr(), 0 if anis is None else 1, 1.0 if anis is None else anis, None,
                                err, len(err))
    return st, err.value.decode()


@pytest.mark.parametrize("layout,bc_included", [("lx", False), ("eo", False), ("lx", True), ("eo", True)])
def test_noalloc_hop_matches_context_hop(cuda_device, layout, bc_included):
    """Both conf layouts (lx and e/o rows) and both boundary forms (periodic
    links, or the time sign already folded into the t=T-1 links), each passed
    identically to the ordinary entry point and to the allocation-free one."""
    import torch
    import oracle
    lib = _lib.load()
    T, L = 16, 8  # 8192 sites: within TMS_NOALLOC_MAX_SITES
    conf = wl.gauge_conf(T, L, 0.4, seed=31)
    if bc_included:
        conf = wl.apply_time_bc(conf, T, L, -1.0)
    if layout == "eo":
        conf = oracle.Geom(T, L).split(conf)
    Vh = T * L ** 3 // 2
    x0 = wl.random_spinor(Vh, 32)
    x1 = wl.random_spinor(Vh, 33)
    with Lattice(T, L, bc_t=-1.0) as lat:
        lat.upload_conf(conf, layout=layout, bc_included=bc_included)
        ref0 = lat.tmn2Deo_or_tmn2Doe_eos(0, x0)
        ref1 = lat.tmn2Deo_or_tmn2Doe_eos(1, x1, anis=1.2)
    conf_d = torch.from_numpy(np.ascontiguousarray(conf)).cuda()
    out_d = torch.empty((Vh, 4, 3, 2), dtype=torch.float64, device="cuda")
    lay = 0 if layout == "lx" else 1
    flags = 1 if bc_included else 0  # TMS_CONF_BC_INCLUDED
    # two calls in a row: the second reuses (and overwrites) the scratch the first one left
    st, msg = _noalloc(lib, T, L, conf_d, 0, torch.from_numpy(x0).cuda(), out_d, layout=lay, flags=flags)
    assert st == 0, msg
    assert rel(out_d.cpu().numpy(), ref0) < TOL
    st, msg = _noalloc(lib, T, L, conf_d, 1, torch.from_numpy(x1).cuda(), out_d, anis=1.2, layout=lay, flags=flags)
    assert st == 0, msg
    assert rel(out_d.cpu().numpy(), ref1) < TOL


def test_noalloc_rejects_oversized_lattice(cuda_device):
    import torch
    lib = _lib.load()
    T, L = 64, 8  # 32768 sites: beyond the fixed scratch
    V = T * L ** 3
    assert V > 16384
    conf_d = torch.zeros((V, 4, 3, 3, 2), dtype=torch.float64, device="cuda")
    x = torch.zeros((V // 2, 4, 3, 2), dtype=torch.float64, device="cuda")
    st, msg = _noalloc(lib, T, L, conf_d, 0, x, x.clone())
    assert st == 3  # TMS_ERR_BAD_ARG
    assert "exceeds" in msg and "16384" in msg
