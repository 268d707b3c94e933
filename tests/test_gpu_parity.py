"""Parity of the CUDA path (through the C ABI) with the oracle and the golden fixtures.

Two bars, one per oracle build:
* against liboracle_cr.so (the restatement with correctly rounded pow and exp, the arithmetic
  the CUDA path computes): every superdroplet field, gridbox state and budget bit for bit, order
  included, over runs of the configurations' own lengths and at their sizes;
* against liboracle.so (host libm, pinned bit for bit to CLEO's own sources) and the golden
  fixtures made by CLEO's own sources: order, gridbox indices, multiplicities and ids bit-exact;
  radius, solute mass, coordinates and gridbox state within 1e-12 relative (the host libm's rare
  misroundings of pow and exp are the only difference left).
"""
import ctypes as C
import os

import numpy as np
import pytest

import checkers as K
from cleo_b200 import abi, workloads as W
from cleo_b200.config import make_params
from cleo_b200.sdm import CleoError, make_sdm
from test_oracle import ERRS, GOLOVIN_L1_BOUND, VARIANTS, _err_case, golovin_l1

pytestmark = pytest.mark.gpu

RTOL = 1e-12
TUNED = (256, 5, 128, 3)  # the launch configuration the autotuner picks on the 40 M workload


def budget_close(got, exp, what=""):
    """The cumulative condensed mass per gridbox is a sum of differences of nearly equal masses
    (and keeps the contributions of droplets that have since left), so against the host-libm
    oracle it is compared relative to the largest budget of the domain, not element-wise."""
    scale = float(np.max(np.abs(exp))) if len(exp) else 0.0
    err = np.abs(got - exp)
    assert np.all(err <= 1e-12 * scale + 1e-300), (what, float(np.max(err)) / max(scale, 1e-300))


# the batched schedule with the page re-sort after every motion step, whatever the domain's size
# and the movers' share (the default policy takes the full sort on domains of fewer pages than the
# GPU has SMs, which the small workloads here are)
PAGES = 2
MODES = [abi.EXEC_PLAIN, abi.EXEC_BATCHED, PAGES]
MODE_IDS = ["plain", "batched", "pages"]


def with_mode(w, mode):
    w["params"].exec_mode = abi.EXEC_BATCHED if mode == PAGES else mode
    w["resort"] = abi.RESORT_PAGES if mode == PAGES else abi.RESORT_AUTO
    return w


def make_gpu(w, lib):
    """The workload on the GPU, with the re-sort policy with_mode chose."""
    g = make_sdm(w, lib=lib)
    assert lib.cleo_b200_set_resort_policy(g.ctx, w.get("resort", abi.RESORT_AUTO)) == 0
    return g


@pytest.fixture(scope="module")
def lib():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return abi.load_library()


def cr_oracle(w):
    """The correctly rounded oracle on every host core (its results do not depend on them)."""
    lib = K.oracle_lib(cr=True)
    K.oracle_threads(lib)
    return make_sdm(w, lib=lib, prefix="oc")


def run_pair(lib, w, nsteps, cfg=None, oracle=None):
    g = make_gpu(w, lib)
    if cfg is not None:
        assert lib.cleo_b200_set_launch_config(g.ctx, (C.c_int32 * 4)(*cfg)) == 0
    o = oracle(w) if oracle else cr_oracle(w)
    ts = w["tstep"]
    for s in range(nsteps):
        g.run_step(s * ts, (s + 1) * ts)
        o.run_step(s * ts, (s + 1) * ts)
    g.check()
    o.check()
    return g, o


def within_bar(g, o, what):
    """The bar against the host-libm oracle (or CLEO's fixtures)."""
    K.assert_same_domain(g.download_supers(), o.download_supers(), rtol=RTOL, what=what)
    sg, so = g.download_state(), o.download_state()
    for f in abi.STATE_FIELDS:
        assert K.max_rel(sg[f], so[f]) <= RTOL, (what, f)
    budget_close(g.download_budgets()[0], o.download_budgets()[0], what)


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("fname", K.step_fixtures())
def test_gpu_matches_golden(lib, fname, mode):
    w, exp = K.load_step_fixture(os.path.join(K.GOLDEN, fname))
    with_mode(w, mode)
    g = make_gpu(w, lib)
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
    K.assert_identical_run(g, o, name)
    o2 = make_sdm(w, lib=K.oracle_lib(), prefix="oc")
    for s in range(nsteps):
        o2.run_step(s * w["tstep"], (s + 1) * w["tstep"])
    within_bar(g, o2, name)


@pytest.mark.parametrize("tol", [(50, 0.0, 0.01), (200, 0.0, 1e-8)])
@pytest.mark.parametrize("mode", MODES[:2], ids=MODE_IDS[:2])
def test_gpu_condensation_solve(lib, tol, mode):
    """2^21 independent droplets at the reference's and at the tight tolerance: radii and Newton
    iteration counts bit for bit, including the marks (NITERS_FAILED) of the few droplets that
    the reference itself cannot converge (about two per million; its abort,
    impliciteuler.cpp:213-217): the correctly rounded oracle marks exactly the same ones. (With
    the host libm a borderline droplet at the tight tolerance can fail too: whether its last
    Newton step passes atol = 1e-8 depends on the rounding of pow.)"""
    import torch
    mx, rt, at = tol
    p = make_params(condtstep=1.0, maxniters=mx, rtol=rt, atol=at)
    p.exec_mode = mode
    w = W.condsolve(1 << 21, seed=2026)
    for cr in (True, False):
        K.oracle_threads(K.oracle_lib(cr=cr))
    rc_c, rc_r, itc = K.condsolve(K.oracle_lib(cr=True), "oc", p, w)
    rc_o, ro, ito = K.condsolve(K.oracle_lib(), "oc", p, w)
    failed = (itc & abi.NITERS_FAILED) != 0
    failed_libm = (ito & abi.NITERS_FAILED) != 0
    assert failed.sum() > 0 and np.all(failed_libm[failed])
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
    assert err.code == rc_c == rc_o, (err.code, rc_c, rc_o)  # same abort site
    rg = out.cpu().numpy()
    assert np.array_equal(rg.view(np.uint64), rc_r.view(np.uint64)), K.max_rel(rg, rc_r)
    assert np.array_equal(nit.cpu().numpy().astype(np.uint32), itc)
    ok = ~(failed | failed_libm)
    assert K.max_rel(rg[ok], ro[ok]) <= RTOL


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
@pytest.mark.parametrize("name,pov,sov,dov,code", ERRS, ids=[e[0] for e in ERRS])
def test_gpu_error_codes(lib, name, pov, sov, dov, code, mode):
    w = with_mode(_err_case(pov, sov, dov), mode)
    s = make_gpu(w, lib)
    with pytest.raises(CleoError) as ei:
        for k in range(3):
            s.run_step(k * 100, (k + 1) * 100)
        s.check()
    assert ei.value.name == code
    # the context stays usable after a reported failure
    s.download_supers()


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_gpu_rainshaft_config_full_length(lib, mode):
    """The 1-D rain shaft configuration at its size (256 boxes x 256 superdroplets) and length
    (1800 steps of 1 s), compared bit for bit after 10, 600 and 1800 steps."""
    w = with_mode(W.rainshaft(), mode)
    g = make_gpu(w, lib)
    o = cr_oracle(w)
    ts = w["tstep"]
    t = 0
    for t_check in (10, 600, 1800):
        while t < t_check:
            g.run_step(t * ts, (t + 1) * ts)
            o.run_step(t * ts, (t + 1) * ts)
            t += 1
        g.check()
        o.check()
        K.assert_identical_run(g, o, f"rainshaft t={t}")


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_gpu_uneven3d_medium(lib, mode):
    """3-D uneven counts on 32x32x16 boxes (~0.6 M superdroplets), 4 steps."""
    w = with_mode(W.uneven3d(ndims=(16, 32, 32), seed=8), mode)
    g, o = run_pair(lib, w, 4)
    K.assert_identical_run(g, o, "uneven3d")


@pytest.mark.parametrize("mode", MODES, ids=MODE_IDS)
def test_gpu_deterministic(lib, mode):
    w = with_mode(W.bubble3d(ndims=(8, 16, 8), seed=9), mode)
    runs = []
    for _ in range(2):
        g = make_gpu(w, lib)
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
    with_mode(w, mode)
    g, o = run_pair(lib, w, 6)
    K.assert_identical_run(g, o, "buckets")


@pytest.mark.parametrize("small_xi", [False, True], ids=["golovin", "golovin_nulls"])
def test_gpu_one_box_large_store(lib, small_xi):
    """A one-gridbox domain whose store is too large for the one-block front kernel (more than
    16 000 slots): the draws, counting sort and chain walks as separate kernels over the GPU, the
    scans in several tiles; with small multiplicities collisions leave nulls, which the flags'
    scan moves behind the valid superdroplets. Bit for bit against the oracle."""
    w = W.box_golovin(20000, seed=31)
    if small_xi:
        rng = np.random.default_rng(31)
        w["supers"]["xi"][:] = rng.integers(1, 4, 20000).astype(np.uint64)
        w["state"]["volume"][:] = 1e-13  # large probabilities: about a third become null
    with_mode(w, abi.EXEC_BATCHED)
    g, o = run_pair(lib, w, 12)
    K.assert_identical_run(g, o, "one box, large store")
    if small_xi:
        d = g.download_supers()
        assert d["n_total"] > d["n_domain"]  # nulls left the domain


def test_gpu_golovin_analytic(lib):
    """The box model (8192 superdroplets, Golovin kernel, 3600 steps of 1 s) reproduces the
    Golovin analytic spectrum on the GPU: mean over 8 seeds of the relative L1 distance of
    g(ln R) at t = 1200, 2400 and 3600 s within the bounds calibrated on the oracle, and total
    water conserved to 1e-12; the first seed's run is the oracle's bit for bit at 3600 s."""
    errs = {t: [] for t in GOLOVIN_L1_BOUND}
    for seed in range(8):
        w = W.box_golovin(8192, seed=200 + seed)
        g = make_sdm(w, lib=lib)
        o = cr_oracle(w) if seed == 0 else None
        t = 0
        for t_out in sorted(GOLOVIN_L1_BOUND):
            while t < t_out:
                g.run_step(t * 100, (t + 1) * 100)
                if o is not None:
                    o.run_step(t * 100, (t + 1) * 100)
                t += 1
            errs[t_out].append(golovin_l1(g.download_supers(), t_out))
        g.check()
        d = g.download_supers()
        nd = d["n_domain"]
        tot0 = float(np.sum(w["supers"]["xi"].astype(np.float64) * w["supers"]["radius"] ** 3))
        tot1 = float(np.sum(d["xi"][:nd].astype(np.float64) * d["radius"][:nd] ** 3))
        assert abs(tot1 - tot0) / tot0 < 1e-12, seed
        if o is not None:
            K.assert_identical_run(g, o, "golovin 3600 s")
    for t_out, bound in GOLOVIN_L1_BOUND.items():
        assert np.mean(errs[t_out]) < bound, (t_out, errs[t_out])


@pytest.mark.parametrize("ndims", [(16, 32, 32), (32, 64, 64)])
def test_gpu_mid_size_domains_tuned_config(lib, ndims):
    """Domains of 16,384 and 131,072 gridboxes (0.6 M and 5 M superdroplets), 10 steps, with the
    launch configuration the autotuner picks on the 40 M-superdroplet workload (the warp
    collision kernel's 64-slot variant at 3 CTAs per SM, its 128-slot variant at 2)."""
    w = W.uneven3d(ndims=ndims, seed=29)
    w["params"].exec_mode = abi.EXEC_BATCHED
    g, o = run_pair(lib, w, 10, cfg=TUNED)
    K.assert_identical_run(g, o, str(ndims))
    g.close()


def test_gpu_uneven3d_full_grid(lib):
    """The 3-D uneven-count configuration at its full size (64 x 128 x 128 gridboxes, ~40 M
    superdroplets), 5 steps at the tuned launch configuration, bit for bit."""
    w = W.uneven3d(ndims=(64, 128, 128), seed=3)
    w["params"].exec_mode = abi.EXEC_BATCHED
    g, o = run_pair(lib, w, 5, cfg=TUNED)
    K.assert_identical_run(g, o, "uneven3d 64x128x128")
    g.close()
    o.close()


def test_gpu_bubble_flow_1m(lib):
    """The coupled-bubble shape (prescribed 2-D flow, lognormal counts of median 16) on
    32 x 64 x 32 gridboxes (~1.6 M superdroplets), 10 steps: about 40% of the superdroplets
    change gridbox every step, so the re-sort takes its full form; bit for bit."""
    w = W.bubble3d(ndims=(32, 64, 32), seed=31)
    w["params"].exec_mode = abi.EXEC_BATCHED
    assert w["n_sd"] > 1_000_000
    g, o = run_pair(lib, w, 10, cfg=TUNED)
    K.assert_identical_run(g, o, "bubble3d 32x64x32")
    g.close()


def test_gpu_resort_policy_and_stats(lib):
    """The re-sort policies give the same run (the page re-sort, the full sort, the automatic
    choice), and cleo_b200_resort_stats reports which re-sort ran and how much it rewrote."""
    runs = {}
    for policy in (abi.RESORT_AUTO, abi.RESORT_PAGES, abi.RESORT_FULL):
        w = W.bubble3d(ndims=(8, 16, 8), seed=21)
        w["params"].exec_mode = abi.EXEC_BATCHED
        g = make_sdm(w, lib=lib)
        assert lib.cleo_b200_set_resort_policy(g.ctx, policy) == 0
        for s in range(4):
            g.run_step(s * w["tstep"], (s + 1) * w["tstep"])
        g.check()
        st = (C.c_uint64 * 4)()
        assert lib.cleo_b200_resort_stats(g.ctx, st) == 0
        movers, rewritten, how, pages = (int(v) for v in st)
        assert pages == (w["grid"]["ngbxs"] + 63) // 64 and movers > 0
        assert rewritten <= pages
        if policy == abi.RESORT_PAGES:
            assert how in (0, 1)  # in place, or every page repacked
        else:  # 16 pages, fewer than the GPU's SMs: the automatic choice is the full sort too
            assert how == 2
        runs[policy] = g.download_supers()
    for policy in (abi.RESORT_PAGES, abi.RESORT_FULL):
        K.assert_same_domain(runs[policy], runs[abi.RESORT_AUTO], rtol=0.0, what=f"policy {policy}")
    assert lib.cleo_b200_set_resort_policy(None, 0) != 0
