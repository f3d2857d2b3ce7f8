"""Every launch shape and link format of the low-precision hops gives the same
solution: mixed-precision solves under each tuning choice must reach the
target true residual, agree with the FP64 solve and take about as many
iterations.  Shapes 3 and 4 select the two-sites-per-thread packed-FP32
kernel, which pairs the sites t and t+T/2 (T a multiple of 4; other T fall
back to the one-site kernel); shape 5 the one-site kernel with the two spin
rows of each half spinor in packed-FP32 lanes, 6 the same with its gathers
streamed through shared memory by cp.async, 7 row tiles staged in shared
memory by bulk copies (LZ a multiple of 8).  The staged kernel's bounded
waits must never give up."""
import numpy as np
import pytest

from nissa_b200 import Lattice, TmError
from nissa_b200 import workload as wl
from conftest import rel

pytestmark = pytest.mark.gpu

KAPPA, MU = 0.1610, 0.005


def _solve_all(lat, src, prec, settings):
    out = []
    for key, val in settings:
        lat.set_tuning(key, val)
        sol, st = lat.inv_tmDkern_eoprec_square_eos_cg(KAPPA, MU, src, 100000, 1e-20, precision=prec)
        out.append((key, val, sol, st))
    return out


@pytest.mark.parametrize("T,L", [(16, 8), (8, 4), (6, 4), (4, 16)])
@pytest.mark.parametrize("precision", ["single", "half"])
def test_hop_shapes_agree(cuda_device, T, L, precision):
    conf = wl.gauge_conf(T, L, 0.35, seed=31)
    src = wl.random_spinor(T * L ** 3 // 2, 7)
    key = "hop_cfg_" + precision
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        ref, st0 = lat.inv_tmDkern_eoprec_square_eos_cg(KAPPA, MU, src, 100000, 1e-22)
        links = [0, 1] if precision == "single" else [0]
        for ls in links:
            lat.set_tuning("links_single", ls)
            for key_, val, sol, st in _solve_all(lat, src, precision, [(key, v) for v in range(8)]):
                assert st["true_rel_res2"] < 1e-20, (ls, val, st)
                assert rel(sol, ref) < 1e-8, (ls, val)
                assert st["iterations"] <= 1.1 * st0["iterations"] + 5, (ls, val, st["iterations"], st0["iterations"])
        assert lat.hop_stage_timeouts == 0


@pytest.mark.parametrize("T,L", [(16, 8), (8, 16)])
@pytest.mark.parametrize("precision", ["single", "half"])
def test_tile_rows_agree(cuda_device, T, L, precision):
    """The staged shape under every site tiling (rows per tile) solves to the
    target and agrees with the FP64 solution; its waits never give up."""
    from nissa_b200 import tune
    conf = wl.gauge_conf(T, L, 0.35, seed=33)
    src = wl.random_spinor(T * L ** 3 // 2, 9)
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        ref, st0 = lat.inv_tmDkern_eoprec_square_eos_cg(KAPPA, MU, src, 100000, 1e-22)
        lat.set_tuning("hop_cfg_" + precision, tune.TILED_SHAPE)
        rows = tune.tile_rows_choices(L, L)
        assert rows
        for key_, val, sol, st in _solve_all(lat, src, precision, [("tma_rows", r) for r in rows + [0]]):
            assert st["true_rel_res2"] < 1e-20, (val, st)
            assert rel(sol, ref) < 1e-8, val
            assert st["iterations"] <= 1.1 * st0["iterations"] + 5, (val, st["iterations"], st0["iterations"])
        assert lat.hop_stage_timeouts == 0
        for bad in (3, L + 1, -1, 0.5):
            with pytest.raises(TmError):
                lat.set_tuning("tma_rows", bad)


@pytest.mark.parametrize("T,L", [(16, 8), (8, 4), (6, 4)])
def test_half_arith_solves(cuda_device, T, L):
    """The FP16-arithmetic hop (tuning half_arith) under the FP16-spinor e/o
    solver: the FP64 reliable updates still bring the solve to the target true
    residual, within 1e-8 of the FP64 solution, in about the same iterations."""
    conf = wl.gauge_conf(T, L, 0.35, seed=34)
    src = wl.random_spinor(T * L ** 3 // 2, 10)
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        ref, st0 = lat.inv_tmDkern_eoprec_square_eos_cg(KAPPA, MU, src, 100000, 1e-22)
        lat.set_tuning("half_arith", 1)
        assert lat.get_tuning("half_arith") == 1
        sol, st = lat.inv_tmDkern_eoprec_square_eos_cg(KAPPA, MU, src, 100000, 1e-20, precision="half")
        assert st["true_rel_res2"] < 1e-20, st
        assert rel(sol, ref) < 1e-8
        assert st["iterations"] <= 1.2 * st0["iterations"] + 5, (st["iterations"], st0["iterations"])
        lat.set_tuning("half_arith", 0)
        sol0, _ = lat.inv_tmDkern_eoprec_square_eos_cg(KAPPA, MU, src, 100000, 1e-20, precision="half")
        assert rel(sol0, ref) < 1e-8
        with pytest.raises(TmError):
            lat.set_tuning("half_arith", 2)


def test_full_lattice_packed(cuda_device):
    """The full-lattice operator (both parities in one launch) under the packed kernel."""
    T, L = 8, 4
    conf = wl.gauge_conf(T, L, 0.35, seed=32)
    src = wl.random_spinor(T * L ** 3, 8)
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        ref, _ = lat.inv_tmQ2_cg(KAPPA, MU, src, 100000, 1e-22)
        for prec in ("single", "half"):
            for v in (0, 3, 4, 5, 6, 7):
                lat.set_tuning("hop_cfg_" + prec, v)
                sol, st = lat.inv_tmQ2_cg(KAPPA, MU, src, 100000, 1e-20, precision=prec)
                assert rel(sol, ref) < 1e-8, (prec, v)


def test_shape_range_checked(cuda_device):
    with Lattice(4, 4) as lat:
        with pytest.raises(TmError):
            lat.set_tuning("hop_cfg_double", 3)
        with pytest.raises(TmError):
            lat.set_tuning("hop_cfg_single", 8)
        lat.set_tuning("hop_cfg_half", 4)
        lat.set_tuning("hop_cfg_half", 7)
        assert lat.get_tuning("hop_cfg_half") == 7 and lat.get_tuning("hop_cfg_single") == 1
        assert lat.get_tuning("tma_rows") == 0 and lat.get_tuning("reliable_delta_half") == 0.005
        with pytest.raises(TmError):
            lat.get_tuning("no_such_knob")


def test_autotune_on_device(cuda_device, tmp_path):
    """The autotuner times real kernels, applies a valid choice and reuses its cache;
    a solve under the tuned choice still reaches the target."""
    from nissa_b200 import tune
    T, L = 8, 4
    conf = wl.gauge_conf(T, L, 0.35, seed=33)
    src = wl.random_spinor(T * L ** 3 // 2, 9)
    cache = str(tmp_path / "tune.json")
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        r = tune.autotune(lat, "half", cache=cache)
        assert not r["cached"] and r["settings"]["hop_cfg_half"] in tune.HOP_SHAPES["half"]
        rb = tune.autotune(lat, "half", nrhs=8, cache=cache)
        assert rb["settings"]["mrhs_per_thread"] in tune.MRHS_CHOICES
        assert tune.autotune(lat, "half", cache=cache)["cached"]
        sol, st = lat.inv_tmDkern_eoprec_square_eos_cg(KAPPA, MU, src, 100000, 1e-20, precision="half")
        assert st["true_rel_res2"] < 1e-20


def test_stream_priority_keeps_results(cuda_device):
    """The context's stream recreated at a raised priority: the same solve
    gives the same bits; priorities outside the device's range are refused."""
    conf = wl.gauge_conf(8, 4, 0.35, seed=91)
    src = wl.random_spinor(8 * 4 ** 3, 92)
    with Lattice(8, 4) as lat:
        lat.upload_conf(conf)
        ref, _ = lat.inv_tmD_cg_eoprec(0.16, 0.01, src, 100000, 1e-20, precision="half")
        lat.set_tuning("stream_priority", -1)
        sol, _ = lat.inv_tmD_cg_eoprec(0.16, 0.01, src, 100000, 1e-20, precision="half")
        assert np.array_equal(sol, ref)
        for bad in (1, -1000, -0.5):
            with pytest.raises(TmError):
                lat.set_tuning("stream_priority", bad)
