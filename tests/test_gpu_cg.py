"""CUDA solvers (through the C ABI) against the reference's fixtures and the
oracle.  FP64 solutions must agree to 1e-9 relative at a 1e-12 target
(|r|/|b|, i.e. residue 1e-24 in the reference's squared convention); mixed
precision solutions are reported against the FP64 oracle and must reach the
target true residual."""
import numpy as np
import pytest

import oracle
from nissa_b200 import Lattice, TmError
from nissa_b200 import workload as wl
from conftest import rel

pytestmark = pytest.mark.gpu


def test_cg_square_matches_reference_fixture(cuda_device, golden_small):
    g = golden_small
    T, L = int(g["T"]), int(g["L"])
    with Lattice(T, L) as lat:
        lat.upload_conf(g["conf"])
        sol, st = lat.inv_tmDkern_eoprec_square_eos_cg(float(g["kappa"]), float(g["mu"]), g["in_odd"], 10000, 1e-24)
        assert abs(st["iterations"] - int(g["cg_iters"])) <= 1
        assert rel(sol, g["cg"]) < 1e-9
        assert st["true_rel_res2"] < 2e-24


def test_full_solve_matches_reference_fixture(cuda_device, golden_small):
    g = golden_small
    T, L = int(g["T"]), int(g["L"])
    with Lattice(T, L) as lat:
        lat.upload_conf(g["conf"])
        sol, st = lat.inv_tmD_cg_eoprec(float(g["kappa"]), float(g["mu"]), g["in_lx"], 10000, 1e-24)
        assert abs(st["iterations"] - int(g["cgfull_iters"])) <= 1
        assert rel(sol, g["cgfull"]) < 1e-9
        assert st["lx_rel_res2"] < 1e-22


def test_config1_plain_fp64_cg(cuda_device, golden_cg):
    """8^3x16, kappa 0.16, mu 0.01, eps 0.4, point source, |r|/|b| <= 1e-12."""
    g = golden_cg
    T, L = int(g["T"]), int(g["L"])
    conf = wl.gauge_conf(T, L, float(g["eps"]), int(g["seed"]))
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        sol, st = lat.inv_tmD_cg_eoprec(float(g["kappa"]), float(g["mu"]), wl.point_source(T, L), 100000,
                                        float(g["residue"]))
        assert abs(st["iterations"] - int(g["iters"])) <= 2
        assert rel(sol[::8], g["sol_every8"]) < 1e-9
        assert st["lx_rel_res2"] < 1e-22


@pytest.mark.parametrize("precision", ["single", "half"])
def test_mixed_precision_reaches_target(cuda_device, precision):
    T, L = 16, 8
    kappa, mu = 0.1610, 0.005
    conf = wl.gauge_conf(T, L, 0.35, seed=21)
    geo = oracle.Geom(T, L)
    ceo = geo.split(wl.apply_time_bc(conf, T, L))
    src = wl.random_spinor(geo.Vh, 9)
    ref, _, _ = geo.cg_eos(ceo, kappa, mu, src, 100000, 1e-26)
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        sol, st = lat.inv_tmDkern_eoprec_square_eos_cg(kappa, mu, src, 100000, 1e-20, precision=precision)
        assert st["true_rel_res2"] < 1e-20
        assert st["reliable_updates"] >= 1
        err = rel(sol, ref)
        assert err < 1e-8, err


def test_guess_is_used(cuda_device, golden_small):
    g = golden_small
    T, L = int(g["T"]), int(g["L"])
    with Lattice(T, L) as lat:
        lat.upload_conf(g["conf"])
        sol, st = lat.inv_tmDkern_eoprec_square_eos_cg(float(g["kappa"]), float(g["mu"]), g["in_odd"], 10000, 1e-24,
                                                       guess=g["cg"])
        assert st["iterations"] <= 2
        assert rel(sol, g["cg"]) < 1e-9


def test_solver_error_paths(cuda_device):
    T, L = 4, 4
    with Lattice(T, L) as lat:
        lat.upload_conf(wl.gauge_conf(T, L, 0.4, 2))
        z = np.zeros((lat.Vh, 4, 3, 2))
        with pytest.raises(TmError) as e:
            lat.inv_tmDkern_eoprec_square_eos_cg(0.16, 0.01, z, 100, 1e-20)
        assert e.value.status == 8  # invalid source norm
        x = wl.random_spinor(lat.Vh, 1)
        with pytest.raises(TmError) as e:
            lat.inv_tmDkern_eoprec_square_eos_cg(0.16, 0.01, x, 3, 1e-24)
        assert e.value.status == 1  # not converged
        assert e.value.stats["iterations"] >= 3
        xn = x.copy()
        xn[3, 1, 2, 0] = np.nan
        with pytest.raises(TmError) as e:
            lat.inv_tmDkern_eoprec_square_eos_cg(0.16, 0.01, xn, 100, 1e-20)
        assert e.value.status in (2, 8)
        for prec in ("single", "half"):
            with pytest.raises(TmError) as e:
                lat.inv_tmDkern_eoprec_square_eos_cg(0.16, 0.01, x, 3, 1e-24, precision=prec)
            assert e.value.status == 1


def test_precision_switching_same_lattice(cuda_device):
    """single -> half -> single -> double on one context: graphs are rebuilt
    when the inner fields change precision."""
    T, L = 8, 4
    conf = wl.gauge_conf(T, L, 0.35, seed=4)
    src = wl.random_spinor(T * L ** 3 // 2, 5)
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        sols = []
        for prec in ("single", "half", "single", "double"):
            sol, st = lat.inv_tmDkern_eoprec_square_eos_cg(0.16, 0.01, src, 10000, 1e-20, precision=prec)
            assert st["true_rel_res2"] < 1e-20
            sols.append(sol)
        for s in sols[:3]:
            assert rel(s, sols[3]) < 1e-8
        n0 = lat.launch_count
        lat.inv_tmDkern_eoprec_square_eos_cg(0.16, 0.01, src, 10000, 1e-20, precision="single")
        assert lat.launch_count - n0 >= 5 * 10


@pytest.mark.parametrize("precision", ["double", "single", "half"])
def test_full_solve_point_source_all_precisions(cuda_device, golden_cg, precision):
    """The 8^3x16 point-source solve in every precision: a point source leaves
    most sites at (or near) zero for many iterations, which the FP16 per-site
    scale must survive."""
    g = golden_cg
    T, L = int(g["T"]), int(g["L"])
    conf = wl.gauge_conf(T, L, float(g["eps"]), int(g["seed"]))
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        sol, st = lat.inv_tmD_cg_eoprec(float(g["kappa"]), float(g["mu"]), wl.point_source(T, L), 100000, 1e-24,
                                        precision=precision)
        assert st["true_rel_res2"] < 1e-24
        assert rel(sol[::8], g["sol_every8"]) < 1e-9


@pytest.mark.parametrize("mode", ["numpy", "pinned", "device"])
def test_columns_equal_single_solves(cuda_device, golden_cg, mode):
    """tms_cg_eoprec_columns runs the same solve per column as tms_cg_eoprec:
    the solutions are bit-identical whether the buffers are pageable host,
    page-locked host (copies overlapping the neighbouring solves) or device
    memory, and the point-source column matches the reference's solution."""
    import torch
    g = golden_cg
    T, L = int(g["T"]), int(g["L"])
    V = T * L ** 3
    kappa, mu = float(g["kappa"]), float(g["mu"])
    srcs = [wl.point_source(T, L)] + [wl.random_spinor(V, 70 + k) for k in range(4)]
    with Lattice(T, L) as lat:
        lat.upload_conf(wl.gauge_conf(T, L, float(g["eps"]), int(g["seed"])))
        singles = [lat.inv_tmD_cg_eoprec(kappa, mu, s, 100000, 1e-24, precision="half")[0] for s in srcs]
        outs = None
        if mode == "numpy":
            ins = srcs
        elif mode == "pinned":
            ins = [torch.from_numpy(s).pin_memory() for s in srcs]
            outs = [torch.empty((V, 4, 3, 2), dtype=torch.float64).pin_memory() for _ in srcs]
        else:
            ins = [torch.from_numpy(s).to("cuda:0") for s in srcs]
        sols, sts = lat.inv_tmD_cg_eoprec_columns(kappa, mu, ins, 100000, 1e-24, precision="half", out=outs)
        assert len(sts) == len(srcs)
        for k in range(len(srcs)):
            got = sols[k].cpu().numpy() if mode != "numpy" else sols[k]
            assert np.array_equal(got, singles[k])
            assert sts[k]["status"] == 0 and sts[k]["lx_rel_res2"] < 1e-23
        first = sols[0].cpu().numpy() if mode != "numpy" else sols[0]
        assert rel(first[::8], g["sol_every8"]) < 1e-9
        # a column count of zero is refused before any work
        import ctypes
        st = lat.lib.tms_cg_eoprec_columns(lat.h, 0, None, None, kappa, 0, 1.0, mu, 100, 1e-20, 0, None)
        assert st == 3


def test_device_buffers_need_only_8_byte_alignment(cuda_device, golden_cg):
    """Device pointers need only the alignment of a double: a conf, an operator
    input/output and a full solve on buffers offset by one double give the same
    bits as on 16-byte aligned ones."""
    import torch
    g = golden_cg
    T, L = int(g["T"]), int(g["L"])
    V = T * L ** 3
    kappa, mu = float(g["kappa"]), float(g["mu"])
    conf = torch.from_numpy(wl.gauge_conf(T, L, float(g["eps"]), int(g["seed"])))

    def offset(a):
        big = torch.zeros(a.numel() + 1, dtype=torch.float64, device="cuda:0")
        v = big[1:].view(a.shape)
        v.copy_(a)
        assert v.data_ptr() % 16 == 8
        return v

    src = torch.from_numpy(wl.random_spinor(V, 81))
    x = torch.from_numpy(wl.random_spinor(V // 2, 82))
    with Lattice(T, L) as lat:
        lat.upload_conf(conf.to("cuda:0"))
        hop = lat.tmn2Deo_or_tmn2Doe_eos(1, x.to("cuda:0"))
        sol, _ = lat.inv_tmD_cg_eoprec(kappa, mu, src.to("cuda:0"), 100000, 1e-22, precision="half")
    with Lattice(T, L) as lat:
        lat.upload_conf(offset(conf))
        hop_o = lat.tmn2Deo_or_tmn2Doe_eos(1, offset(x), out=offset(torch.zeros_like(x)))
        out = offset(torch.zeros_like(src))
        lat.inv_tmD_cg_eoprec(kappa, mu, offset(src), 100000, 1e-22, precision="half", out=out)
        assert torch.equal(hop_o, hop)
        assert torch.equal(out, sol)


@pytest.mark.parametrize("precision", ["single", "half"])
def test_paired_x_updates_match_unpaired(cuda_device, precision):
    """An even CUDA-graph length makes the mixed e/o solver add the steps to x
    every other iteration (two directions kept, the pending step flushed when
    a reliable update cuts a replay); an odd length keeps the per-iteration
    update.  Both reach the target with the same iteration count, and their
    solutions agree to the solver's accuracy."""
    T, L = 16, 8
    conf = wl.gauge_conf(T, L, 0.35, seed=61)
    src = wl.random_spinor(T * L ** 3, 62)
    sols, its = [], []
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        for gi in (8, 7, 2):
            lat.set_tuning("graph_iters", gi)
            sol, st = lat.inv_tmD_cg_eoprec(0.1610, 0.005, src, 100000, 1e-20, precision=precision)
            assert st["reliable_updates"] >= 2 and st["lx_rel_res2"] < 1e-19
            sols.append(sol)
            its.append(st["iterations"])
    assert max(its) - min(its) <= 1
    assert rel(sols[0], sols[1]) < 1e-8 and rel(sols[2], sols[1]) < 1e-8


def test_full_solve_from_guess(cuda_device, golden_cg):
    """inv_tmD_cg_eoprec's optional guess_Koo: the Eq. (9) CG started from the
    exact Koo solution (the square solve of the oracle's Eq. 8 source) needs no
    iteration in any precision, and a zero guess behaves as none."""
    g = golden_cg
    T, L = int(g["T"]), int(g["L"])
    V, Vh = T * L ** 3, T * L ** 3 // 2
    kappa, mu = float(g["kappa"]), float(g["mu"])
    conf = wl.gauge_conf(T, L, float(g["eps"]), int(g["seed"]))
    geo = oracle.Geom(T, L)
    ceo = geo.split(wl.apply_time_bc(conf, T, L, -1.0))
    src = wl.random_spinor(V, 71)
    eta = geo.split(src.reshape(V, -1)).reshape(2, Vh, 4, 3, 2)
    varphi = eta[1] + 0.5 * geo.hop(ceo, 1, geo.inv_tmDee(kappa, mu, eta[0])).reshape(Vh, 4, 3, 2)
    varphi[:, 2:] *= -1.0
    with Lattice(T, L) as lat:
        lat.upload_conf(conf)
        y, _ = lat.inv_tmDkern_eoprec_square_eos_cg(kappa, mu, np.ascontiguousarray(varphi), 100000, 1e-28)
        ref, st0 = lat.inv_tmD_cg_eoprec(kappa, mu, src, 100000, 1e-22)
        assert st0["iterations"] > 10
        sol, st1 = lat.inv_tmD_cg_eoprec(kappa, mu, src, 100000, 1e-22, guess_Koo=y)
        assert st1["iterations"] <= 1 and rel(sol, ref) < 1e-9
        z, st2 = lat.inv_tmD_cg_eoprec(kappa, mu, src, 100000, 1e-22, guess_Koo=np.zeros((Vh, 4, 3, 2)))
        assert abs(st2["iterations"] - st0["iterations"]) <= 1 and rel(z, ref) < 1e-10
        for prec in ("single", "half"):
            s, st = lat.inv_tmD_cg_eoprec(kappa, mu, src, 100000, 1e-20, precision=prec, guess_Koo=y)
            assert st["iterations"] <= 1 and rel(s, ref) < 1e-8


def test_columns_error_leaves_context_usable(cuda_device):
    """A column whose source is zero stops tms_cg_eoprec_columns with the
    reference's invalid-norm error (host buffers: no copy is left running),
    and the context solves normally afterwards."""
    T, L = 8, 4
    V = T * L ** 3
    srcs = [wl.random_spinor(V, 91), np.zeros((V, 4, 3, 2)), wl.random_spinor(V, 92)]
    with Lattice(T, L) as lat:
        lat.upload_conf(wl.gauge_conf(T, L, 0.35, seed=90))
        with pytest.raises(TmError) as e:
            lat.inv_tmD_cg_eoprec_columns(0.16, 0.01, srcs, 100000, 1e-20, precision="half")
        assert e.value.status == 8
        sols, sts = lat.inv_tmD_cg_eoprec_columns(0.16, 0.01, [srcs[0], srcs[2]], 100000, 1e-20, precision="half")
        ref, _ = lat.inv_tmD_cg_eoprec(0.16, 0.01, srcs[2], 100000, 1e-20, precision="half")
        assert np.array_equal(sols[1], ref) and all(s["status"] == 0 for s in sts)
