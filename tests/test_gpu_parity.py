"""Parity of the CUDA path (through the C ABI) with the oracle and the golden fixtures.

Bar: sort order, gridbox indices, multiplicities and ids bit-exact; radius, solute mass,
coordinates and gridbox state within 1e-12 relative in FP64 (the only differences allowed come
from CUDA's vs the host libm's pow/exp and from the order of per-gridbox FP64 sums).
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

import checkers as K
from cleo_b200 import abi, workloads as W
from cleo_b200.config import Rho_l, make_params
from cleo_b200.sdm import CleoError, make_sdm
from test_oracle import ERRS, VARIANTS, _err_case, golovin_l1

pytestmark = pytest.mark.gpu

RTOL = 1e-12


def budget_close(got, exp, what=""):
    """The cumulative condensed mass per gridbox is a sum of differences of nearly equal masses
    (and keeps the contributions of droplets that have since left), so it is compared relative to
    the largest budget of the domain, not element-wise."""
    scale = float(np.max(np.abs(exp))) if len(exp) else 0.0
    err = np.abs(got - exp)
    assert np.all(err <= 1e-12 * scale + 1e-300), (what, float(np.max(err)) / max(scale, 1e-300))


MODES = [abi.EXEC_PLAIN, abi.EXEC_BATCHED]
MODE_IDS = ["plain", "batched"]


def with_mode(w, mode):
    w["params"].exec_mode = mode
    return w


@pytest.fixture(scope="module")
def lib():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return abi.load_library()


def run_pair(lib, w, nsteps):
    g = make_sdm(w, lib=lib)
    o = make_sdm(w, lib=K.oracle_lib(), prefix="oc")
    ts = w["tstep"]
    for s in range(nsteps):
        g.run_step(s * ts, (s + 1) * ts)
        o.run_step(s * ts, (s + 1) * ts)
    g.check()
    return g, o


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("fname", K.step_fixtures())
def test_gpu_matches_golden(lib, fname, mode):
    w, exp = K.load_step_fixture(os.path.join(K.GOLDEN, fname))
    with_mode(w, mode)
    g = make_sdm(w, lib=lib)
    for s in range(exp["nsteps"]):
        g.run_step(s * w["tstep"], (s + 1) * w["tstep"])
    g.check()
    K.assert_same_domain(g.download_supers(), exp["supers"], rtol=RTOL, what=fname)
    st = g.download_state()
    for f in abi.STATE_FIELDS:
        assert K.max_rel(st[f], exp["state"][f]) <= RTOL, (fname, f)
    budget_close(g.download_budgets()[0], exp["cond_mass"], fname)


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("name,build,nsteps", VARIANTS, ids=[v[0] for v in VARIANTS])
def test_gpu_matches_oracle_variants(lib, name, build, nsteps, mode):
    w = with_mode(build(), mode)
    g, o = run_pair(lib, w, nsteps)
    K.assert_same_domain(g.download_supers(), o.download_supers(), rtol=RTOL, what=name)
    sg, so = g.download_state(), o.download_state()
    for f in abi.STATE_FIELDS:
        assert K.max_rel(sg[f], so[f]) <= RTOL, (name, f)
    cg, ig = g.download_budgets()
    co, io = o.download_budgets()
    budget_close(cg, co, name)
    assert np.array_equal(ig, io), (name, "newton iteration counts")


@pytest.mark.parametrize("tol", [(50, 0.0, 0.01), (200, 0.0, 1e-10)])
def test_gpu_condensation_solve(lib, tol):
    import torch
    mx, rt, at = tol
    p = make_params(condtstep=1.0, maxniters=mx, rtol=rt, atol=at)
    w = W.condsolve(50000, seed=13)
    rc_o, ro, io = K.condsolve(K.oracle_lib(), "oc", p, w)
    grid = W.cartesian_grid((1, 1, 1), (1.0, 1.0, 1.0), nspacedims=0)
    from cleo_b200.sdm import SDM
    s = SDM(p, grid, 1, lib=lib)
    dev = {k: torch.tensor(w[k], dtype=torch.float64, device="cuda")
           for k in ("radius", "msol", "temp", "press", "s_ratio", "delt")}
    out = torch.empty_like(dev["radius"])
    nit = torch.empty(len(w["radius"]), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = lib.cleo_b200_condensation_solve(
        s.ctx, len(w["radius"]), *[C.c_void_p(dev[k].data_ptr()) for k in
                                   ("radius", "msol", "temp", "press", "s_ratio", "delt")],
        C.c_void_p(out.data_ptr()), C.c_void_p(nit.data_ptr()))
    assert rc == 0
    err = s.status()
    assert err.code == rc_o, (err.code, rc_o)  # same abort site (e.g. NR non-convergence)
    rg = out.cpu().numpy()
    assert K.max_rel(rg, ro) <= RTOL
    assert np.array_equal(nit.cpu().numpy().astype(np.uint32), io)


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("name,pov,sov,dov,code", ERRS, ids=[e[0] for e in ERRS])
def test_gpu_error_codes(lib, name, pov, sov, dov, code, mode):
    w = with_mode(_err_case(pov, sov, dov), mode)
    s = make_sdm(w, lib=lib)
    with pytest.raises(CleoError) as ei:
        for k in range(3):
            s.run_step(k * 100, (k + 1) * 100)
        s.check()
    assert ei.value.name == code
    # the context stays usable after a reported failure
    s.download_supers()


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_gpu_rainshaft_config(lib, mode):
    """1-D rain shaft at full size (256 boxes x 256 superdroplets), 10 steps."""
    w = with_mode(W.rainshaft(), mode)
    g, o = run_pair(lib, w, 10)
    K.assert_same_domain(g.download_supers(), o.download_supers(), rtol=RTOL, what="rainshaft")


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_gpu_uneven3d_medium(lib, mode):
    """3-D uneven counts on 32x32x16 boxes (~0.6 M superdroplets), 4 steps."""
    w = with_mode(W.uneven3d(ndims=(16, 32, 32), seed=8), mode)
    g, o = run_pair(lib, w, 4)
    K.assert_same_domain(g.download_supers(), o.download_supers(), rtol=RTOL, what="uneven3d")


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_gpu_deterministic(lib, mode):
    w = with_mode(W.bubble3d(ndims=(8, 16, 8), seed=9), mode)
    runs = []
    for _ in range(2):
        g = make_sdm(w, lib=lib)
        for s in range(5):
            g.run_step(s * 100, (s + 1) * 100)
        d = g.download_supers()
        runs.append(d)
    for k in ("sdid", "xi", "radius", "coord3", "coord1"):
        assert np.array_equal(runs[0][k], runs[1][k]), k


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_gpu_all_bucket_sizes(lib, mode):
    """Gridboxes of 0 .. 3000 superdroplets (every size bucket of the batched schedule)."""
    w = W.uneven3d(ndims=(4, 4, 4), seed=12)
    rng = np.random.default_rng(12)
    counts = rng.integers(0, 80, 64)
    counts[[3, 17, 40]] = (300, 1024, 3000)
    counts[[5, 6]] = (0, 1)
    sd = W.populate(w["grid"], counts, rng, temp=w["state"]["temp"],
                    s_ratio=np.full(64, 0.99))
    w["supers"] = sd
    w["n_sd"] = int(counts.sum())
    w["params"].exec_mode = mode
    g, o = run_pair(lib, w, 6)
    K.assert_same_domain(g.download_supers(), o.download_supers(), rtol=RTOL, what="buckets")
    budget_close(g.download_budgets()[0], o.download_budgets()[0], "buckets")


def test_gpu_golovin_analytic(lib):
    """The box model reproduces the Golovin analytic spectrum on the GPU (statistical)."""
    errs = []
    for seed in range(3):
        w = W.box_golovin(8192, seed=200 + seed)
        g = make_sdm(w, lib=lib)
        for t in range(1200):
            g.run_step(t * 100, (t + 1) * 100)
        errs.append(golovin_l1(g.download_supers(), 1200))
    assert np.mean(errs) < 0.12, errs


@pytest.mark.parametrize("ndims", [(16, 32, 32), (32, 64, 64)])
def test_gpu_mid_size_domains_tuned_config(lib, ndims):
    """Domains of 16,384 and 131,072 gridboxes (0.6 M and 5 M superdroplets) with the launch
    configuration the autotuner picks on the 40 M-superdroplet workload: the qcond kernel takes 2
    and 14 gridboxes per warp here (one on the smaller test domains), the warp collision kernel's
    64-slot variant runs at 3 CTAs per SM and its 128-slot variant at 2. One step from identical
    states: the per-gridbox sums' order differs from the oracle's in the last bits, which later
    steps' condensation near activation could amplify in a rare droplet of a population this
    large."""
    w = W.uneven3d(ndims=ndims, seed=29)
    w["params"].exec_mode = abi.EXEC_BATCHED
    g = make_sdm(w, lib=lib)
    cfg = (C.c_int32 * 4)(256, 5, 128, 3)
    assert lib.cleo_b200_set_launch_config(g.ctx, cfg) == 0
    o = make_sdm(w, lib=K.oracle_lib(), prefix="oc")
    ts = w["tstep"]
    g.run_step(0, ts)
    o.run_step(0, ts)
    g.check()
    K.assert_same_domain(g.download_supers(), o.download_supers(), rtol=RTOL, what=str(ndims))
    sg, so = g.download_state(), o.download_state()
    for k in ("qcond", "qvap", "temp"):
        assert K.max_rel(sg[k], so[k]) < RTOL, k
    budget_close(g.download_budgets()[0], o.download_budgets()[0], str(ndims))
    g.close()
