"""The drop-in boundary exercised from the reference's side: the reference
build's own driver and callers linked with integration/tm_b200_shim.cpp in
place of the three translation units it replaces (integration/Makefile ->
integration/_build/nissa_ref_b200), so inv_tmD_cg_eoprec, the Schur
operators and apply_tmQ run on the GPU through the C ABI.  Its outputs must
match the unmodified reference build (oracle/_ref/nissa_ref) on the same
inputs: operators to 1e-14, the FP64 solve to 1e-9 with the reference's
iteration count, and the opt-in mixed-precision solve to the FP64 target."""
import os
import re

import numpy as np
import pytest

import oracle
from nissa_b200 import workload as wl
from conftest import ROOT, rel

pytestmark = pytest.mark.gpu

SHIM_BIN = os.path.join(ROOT, "integration", "_build", "nissa_ref_b200")
need = pytest.mark.skipif(not (os.path.exists(SHIM_BIN) and oracle.ref_available()),
                          reason="shim or reference build absent (make -C integration)")


def _iters(stdout):
    m = re.findall(r"Total cg iterations\s*:\s*(\d+)", stdout)
    return int(m[-1]) if m else -1


@need
def test_shim_operators_match_reference(cuda_device):
    T, L = 4, 4
    conf = wl.apply_time_bc(wl.gauge_conf(T, L, 0.4, seed=71), T, L, -1.0)
    Vh, V = T * L ** 3 // 2, T * L ** 3
    rng = np.random.default_rng(72)
    x = rng.standard_normal((Vh, 4, 3, 2))
    xl = rng.standard_normal((V, 4, 3, 2))
    for op, arrays, shape, kw in (("kern", {"conf": conf, "in": x}, (Vh, 4, 3, 2), {}),
                                  ("kern2", {"conf": conf, "in": x}, (Vh, 4, 3, 2), {}),
                                  ("kern2", {"conf": conf, "in": x}, (Vh, 4, 3, 2), {"anis": 1.2}),
                                  ("tmQ", {"conf": conf, "in": xl}, (V, 4, 3, 2), {})):
        ref, _, _ = oracle.run_ref(op, T, L, arrays, shape, kappa=0.16, mu=0.01, **kw)
        got, _, _ = oracle.run_ref(op, T, L, arrays, shape, binary=SHIM_BIN, kappa=0.16, mu=0.01, **kw)
        assert rel(got, ref) < 1e-14, (op, kw, rel(got, ref))


@need
def test_shim_full_solve_matches_reference(cuda_device):
    """inv_tmD_cg_eoprec on 8^3x16 (the plain FP64 configuration, 1e-12), the
    reference's own call path with the library underneath."""
    T, L = 16, 8
    conf = wl.apply_time_bc(wl.gauge_conf(T, L, 0.4, seed=1), T, L, -1.0)
    src = wl.point_source(T, L)
    shape = (T * L ** 3, 4, 3, 2)
    kw = dict(kappa=0.16, mu=0.01, niter=100000, residue=1e-24)
    ref, _, out_r = oracle.run_ref("cgfull", T, L, {"conf": conf, "in": src}, shape, **kw)
    got, _, out_g = oracle.run_ref("cgfull", T, L, {"conf": conf, "in": src}, shape, binary=SHIM_BIN, **kw)
    assert rel(got, ref) < 1e-9
    assert abs(_iters(out_g) - _iters(out_r)) <= 1, (_iters(out_g), _iters(out_r))
    # the mixed-precision inner solver only when asked for, to the same true residual
    kw["residue"] = 1e-20
    ref2, _, _ = oracle.run_ref("cgfull", T, L, {"conf": conf, "in": src}, shape, **kw)
    mix, _, out_m = oracle.run_ref("cgfull", T, L, {"conf": conf, "in": src}, shape, binary=SHIM_BIN,
                                   env={"NISSA_B200_PRECISION": "half"}, **kw)
    assert rel(mix, ref2) < 1e-8
    # library tuning from the environment: the FP16-arithmetic hop, another launch shape
    tuned, _, _ = oracle.run_ref("cgfull", T, L, {"conf": conf, "in": src}, shape, binary=SHIM_BIN,
                                 env={"NISSA_B200_PRECISION": "half",
                                      "NISSA_B200_TUNING": "half_arith=1,reliable_delta_half=0.01,tma_rows=0"}, **kw)
    assert rel(tuned, ref2) < 1e-8


@need
def test_shim_sees_a_conf_rewritten_in_place(cuda_device):
    """The driver's 'cg' op applies the CG twice on one EoField whose links
    are rewritten in place between the calls (kern2twice): the shim must
    upload the new links, as the reference's operator sees them."""
    T, L = 4, 4
    conf = wl.apply_time_bc(wl.gauge_conf(T, L, 0.4, seed=73), T, L, -1.0)
    x = np.random.default_rng(74).standard_normal((T * L ** 3 // 2, 4, 3, 2))
    shape = (T * L ** 3 // 2, 4, 3, 2)
    ref, _, _ = oracle.run_ref("kern2twice", T, L, {"conf": conf, "in": x}, shape, kappa=0.16, mu=0.01)
    got, _, _ = oracle.run_ref("kern2twice", T, L, {"conf": conf, "in": x}, shape, binary=SHIM_BIN, kappa=0.16,
                               mu=0.01)
    assert rel(got, ref) < 1e-14
