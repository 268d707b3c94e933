"""CPU tests of the checkers: the oracle (C restatement) pinned to CLEO's own sources.

Tests that need the reference build (oracle/_ref/libcleo_ref.so, compiled from CLEO's sources
against the Kokkos-API shim) skip where it is absent; the golden fixtures in tests/golden pin the
oracle everywhere else (see test_golden.py).
"""
import ctypes as C
import math

import numpy as np
import pytest

import checkers as K
from cleo_b200 import abi, workloads as W
from cleo_b200.config import cartesian_grid, make_params
from cleo_b200.sdm import CleoError, make_sdm

needs_ref = pytest.mark.skipif(not K.ref_available(), reason="reference build absent")

MASK = (1 << 64) - 1


def py_mix64(z):
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
    return z ^ (z >> 31)


def py_rng(seed, t, g, slot):
    k = py_mix64((seed + 0x9E3779B97F4A7C15) & MASK)
    k = py_mix64(k ^ ((t << 32) | g))
    return py_mix64((k + (slot + 1) * 0x9E3779B97F4A7C15) & MASK)


def test_rng_contract():
    lib = K.oracle_lib()
    for seed, t, g, slot in [(0, 0, 0, 0), (7, 100, 3, 5), (2**63 + 11, 4294967295, 4294967295, 2**40)]:
        u = py_rng(seed, t, g, slot)
        assert lib.oc_rng_u64(seed, t, g, slot) == u
        assert lib.oc_rng_drand(seed, t, g, slot) == (u >> 11) * 2.0**-53
        for hi in (1, 2, 7, 1000, 2**33):
            assert lib.oc_rng_urand(seed, t, g, slot, 0, hi) == (u * hi) >> 64


def test_rng_uniformity():
    lib = K.oracle_lib()
    x = np.array([lib.oc_rng_drand(5, 100, 7, s) for s in range(20000)])
    assert abs(x.mean() - 0.5) < 0.01 and abs(x.var() - 1 / 12) < 0.005
    j = np.array([lib.oc_rng_urand(5, 100, 7, s, 0, 10) for s in range(20000)])
    counts = np.bincount(j, minlength=10)
    assert counts.min() > 1800 and counts.max() < 2200


@needs_ref
def test_grid_neighbours_match_reference():
    ref = K.ref_lib()
    ndims = (5, 4, 3)
    g = cartesian_grid(ndims, (1.0, 1.0, 1.0), nspacedims=3)
    nd = (C.c_uint32 * 3)(*ndims)
    out = (C.c_uint32 * 6)()
    for idx in range(g["ngbxs"]):
        ref.ref_cartesian_neighbours(nd, idx, out)
        mine = [g[k][idx] for k in ("back3", "fwd3", "back1", "fwd1", "back2", "fwd2")]
        assert list(out) == mine, (idx, list(out), mine)


@needs_ref
@pytest.mark.parametrize("kind", [abi.TV_NULL, abi.TV_SIMMEL, abi.TV_ROGERSYAU, abi.TV_ROGERSGK])
def test_terminal_velocity_matches_reference(kind):
    orc, ref = K.oracle_lib(), K.ref_lib()
    for r in np.exp(np.linspace(math.log(1e-3), math.log(5e4), 400)):
        assert orc.oc_terminal_velocity(kind, r) == ref.ref_terminal_velocity(kind, r)


@needs_ref
@pytest.mark.parametrize("prob", [abi.PROB_GOLOVIN, abi.PROB_LONG, abi.PROB_CONST])
def test_pair_probability_matches_reference(prob):
    orc, ref = K.oracle_lib(), K.ref_lib()
    p = make_params(colltstep=1.0, coll_prob=prob, coaleff=0.8, const_kernel=3.5e-9)
    rng = np.random.default_rng(0)
    for _ in range(300):
        r1, r2 = np.exp(rng.uniform(-3, 8, 2))
        a = orc.oc_pair_probability(C.byref(p), r1, 10, 1e-3, r2, 5, 2e-3, 5e-8)
        b = ref.ref_pair_probability(C.byref(p), r1, 10, 1e-3, r2, 5, 2e-3, 5e-8)
        assert a == b


@needs_ref
@pytest.mark.parametrize("tol", [(50, 0.0, 0.01), (200, 0.0, 1e-10)])
def test_condensation_solve_matches_reference(tol):
    orc, ref = K.oracle_lib(), K.ref_lib()
    maxniters, rtol, atol = tol
    p = make_params(condtstep=1.0, maxniters=maxniters, rtol=rtol, atol=atol)
    w = W.condsolve(20000, seed=11)
    rc_a, ra, it = K.condsolve(orc, "oc", p, w)
    rc_b, rb, _ = K.condsolve(ref, "ref", p, w)
    assert rc_a == rc_b == 0
    assert np.array_equal(ra, rb), K.max_rel(ra, rb)
    assert it.min() >= 2


def _variants():
    """(name, workload builder, param overrides, nsteps) covering every plug-in and edge case."""
    v = []
    # box models: Golovin with small xi -> twins and null superdroplets
    def box_small_xi():
        w = W.box_golovin(512, seed=21)
        w["supers"]["xi"][:] = np.random.default_rng(1).integers(1, 4, 512).astype(np.uint64)
        w["params"] = make_params(colltstep=1.0, coll_prob=abi.PROB_GOLOVIN, seed=21)
        w["state"]["volume"][:] = 1e-19  # tiny volume -> large probabilities -> many gammas > 1
        return w
    v.append(("box_golovin_nulls", box_small_xi, 30))
    v.append(("box_golovin", lambda: W.box_golovin(1024, seed=22), 60))

    def box_with(enact, **kw):
        def f():
            w = W.box_golovin(700, seed=23)
            w["supers"]["xi"][:] = np.random.default_rng(2).integers(1, 50, 700).astype(np.uint64)
            w["supers"]["radius"][:] = np.exp(np.random.default_rng(3).uniform(1, 7.5, 700))
            w["params"] = make_params(colltstep=1.0, coll_prob=abi.PROB_LONG, coll_enact=enact,
                                      seed=23, **kw)
            w["state"]["volume"][:] = 1e-9
            return w
        return f
    v.append(("box_breakup_const", box_with(abi.ENACT_BREAKUP, nfrags=5.0), 20))
    v.append(("box_coalbure_straub", box_with(abi.ENACT_COALBURE, flag_kind=abi.FLAG_STRAUB), 20))
    v.append(("box_coalbure_cke", box_with(abi.ENACT_COALBURE, nfrags_kind=abi.NFRAGS_CKE,
                                           flag_kind=abi.FLAG_STRAUB), 20))
    v.append(("box_coalbure_ts", box_with(abi.ENACT_COALBURE, nfrags_kind=abi.NFRAGS_CKE,
                                          flag_kind=abi.FLAG_TESTIKSTRAUB), 20))
    v.append(("box_coalbure_su", box_with(abi.ENACT_COALBURE, flag_kind=abi.FLAG_SZAKALLURBICH), 20))
    v.append(("box_coalbure_const", box_with(abi.ENACT_COALBURE, flag_kind=abi.FLAG_CONST,
                                             flag_coaleff=0.4), 20))
    v.append(("box_const_kernel", box_with(abi.ENACT_COALESCENCE), 20))

    def rain_big():
        w = W.rainshaft(nz=12, per_gbx=24, seed=24)
        rng = np.random.default_rng(4)
        big = rng.random(w["n_sd"]) < 0.3
        w["supers"]["radius"][big] = np.exp(rng.uniform(math.log(50), math.log(1500), big.sum()))
        return w
    v.append(("rain_sediment_out", rain_big, 40))

    def rain_alter():
        w = W.rainshaft(nz=8, per_gbx=20, seed=25)
        w["params"].do_alter_thermo = 1
        w["state"]["qvap"][:] *= 1.02  # supersaturated -> activation and sub-stepping
        return w
    v.append(("rain_alter_thermo", rain_alter, 25))

    def bubble():
        return W.bubble3d(ndims=(6, 8, 4), seed=26)  # 2 m/s flow: drops cross boxes and wrap
    v.append(("bubble_flow_wrap", bubble, 20))

    def uneven_v():
        w = W.uneven3d(ndims=(5, 6, 5), seed=27)
        w["state"]["vvel_lo"][:] = -0.9
        w["state"]["vvel_hi"][:] = 1.1
        w["state"]["uvel_lo"][:] = 0.4
        w["state"]["uvel_hi"][:] = -0.3
        w["state"]["wvel_lo"][:] = 0.5
        w["state"]["wvel_hi"][:] = -0.2
        return w
    v.append(("uneven3d_xyz_winds", uneven_v, 20))
    return v


VARIANTS = _variants()


@needs_ref
@pytest.mark.parametrize("name,build,nsteps", VARIANTS, ids=[v[0] for v in VARIANTS])
def test_sdm_step_matches_reference(name, build, nsteps):
    orc, ref = K.oracle_lib(), K.ref_lib()
    w = build()
    a = make_sdm(w, lib=orc, prefix="oc")
    b = make_sdm(w, lib=ref, prefix="ref")
    ts = w["tstep"]
    for s in range(nsteps):
        a.run_step(s * ts, (s + 1) * ts)
        b.run_step(s * ts, (s + 1) * ts)
    da, db = a.download_supers(), b.download_supers()
    K.assert_same_domain(da, db, rtol=0.0, what=name)
    sa, sb = a.download_state(), b.download_state()
    for f in abi.STATE_FIELDS:
        assert np.array_equal(sa[f], sb[f]), (name, f)
    assert np.array_equal(a.download_budgets()[0], b.download_budgets()[0])


@needs_ref
def test_variants_exercise_edge_cases():
    """The step variants really produce nulls, breakup, out-of-domain and wrapped drops."""
    orc = K.oracle_lib()
    seen = {}
    for name, build, nsteps in VARIANTS:
        w = build()
        a = make_sdm(w, lib=orc, prefix="oc")
        for s in range(nsteps):
            a.run_step(s * w["tstep"], (s + 1) * w["tstep"])
        d = a.download_supers()
        seen[name] = (d["n_total"] - d["n_domain"],
                      int(d["xi"][: d["n_domain"]].sum()) - int(w["supers"]["xi"].sum()))
    assert seen["box_golovin_nulls"][0] > 0          # nulls removed from the domain
    assert seen["box_breakup_const"][1] > 0          # breakup increases total multiplicity
    assert seen["rain_sediment_out"][0] > 0          # drops left through the bottom
    assert seen["bubble_flow_wrap"][0] >= 0


def _err_case(p_over, state_over=None, supers_over=None):
    w = W.rainshaft(nz=4, per_gbx=8, seed=31)
    for k, v in p_over.items():
        setattr(w["params"], k, v)
    if state_over:
        for k, v in state_over.items():
            w["state"][k][:] = v
    if supers_over:
        for k, v in supers_over.items():
            w["supers"][k][:] = v
    return w


ERRS = [
    ("cfl", dict(), dict(wvel_lo=50.0, wvel_hi=50.0), None, "CLEO_ERR_CFL"),
    ("nr_noconverge", dict(maxniters=1, atol=1e-300, rtol=0.0), dict(qvap=0.05), None,
     "CLEO_ERR_NR_NOCONVERGE"),
    ("temperature", dict(), dict(temp=-1.0), None, "CLEO_ERR_TEMPERATURE"),
]


@needs_ref
@pytest.mark.parametrize("name,pov,sov,dov,code", ERRS, ids=[e[0] for e in ERRS])
def test_error_codes_match_reference(name, pov, sov, dov, code):
    orc, ref = K.oracle_lib(), K.ref_lib()
    w = _err_case(pov, sov, dov)
    for lib, prefix in ((orc, "oc"), (ref, "ref")):
        s = make_sdm(w, lib=lib, prefix=prefix)
        with pytest.raises(CleoError) as ei:
            for k in range(3):
                s.run_step(k * 100, (k + 1) * 100)
        assert ei.value.name == code, (prefix, ei.value.name)


def test_subdelt_rejected_at_create():
    w = W.rainshaft(nz=2, per_gbx=2)
    w["params"].cond_minsubdelt = 1.0
    with pytest.raises(CleoError) as ei:
        make_sdm(w, lib=K.oracle_lib(), prefix="oc")
    assert ei.value.name == "CLEO_ERR_SUBDELT"


# ------------------------------------------------------------------------------------------
# the reference's one known answer: the Golovin analytic spectrum (shima2009fig.py:123-151)
# ------------------------------------------------------------------------------------------

def golovin_massdens(r_um, t, n_a=2 ** 23, r_a_um=30.531, b=1500.0, rho_l=998.203):
    """g(lnR) [g m^-3 per unit lnR] of the Golovin solution (restated from shima2009fig.py)."""
    from scipy.special import ive
    r = r_um * 1e-6
    vol_a = 4 / 3 * np.pi * (r_a_um * 1e-6) ** 3
    x = 4 / 3 * np.pi * r ** 3 / vol_a
    tau = 1 - np.exp(-b * n_a * vol_a * t)
    z = 2 * x * np.sqrt(tau)
    bsl_exp = ive(1, z) * np.exp(z - (1 + tau) * x)  # iv(1,z) exp(-(1+tau)x), overflow-safe
    phi = (1 - tau) / (x * np.sqrt(tau)) * bsl_exp
    n = n_a / vol_a * phi
    dv_dlnR = 3 * (4 / 3 * np.pi * r ** 3)
    return n * rho_l * (4 / 3 * np.pi * r ** 3) * dv_dlnR * 1000


def massdens_from_supers(radius_um, xi, volume_m3, edges_ln, rho_l=998.203, smooth=0.2):
    m_g = rho_l * 4 / 3 * np.pi * (radius_um * 1e-6) ** 3 * 1000
    hist, _ = np.histogram(np.log(radius_um), bins=edges_ln, weights=xi * m_g)
    hist = hist / volume_m3 / np.diff(edges_ln)
    cen = 0.5 * (edges_ln[1:] + edges_ln[:-1])
    k = np.exp(-((cen[:, None] - cen[None, :]) ** 2) / (2 * smooth ** 2))
    k /= k.sum(axis=1, keepdims=True)
    return k @ hist, np.exp(cen)


def golovin_l1(d, t_s, volume_m3=1e6):
    nd = d["n_domain"]
    edges = np.linspace(np.log(10.0), np.log(5000.0), 101)
    g_sim, rc = massdens_from_supers(d["radius"][:nd], d["xi"][:nd].astype(np.float64),
                                     volume_m3, edges)
    g_ana = golovin_massdens(rc, t_s)
    dl = np.diff(edges)
    return float(np.sum(np.abs(g_sim - g_ana) * dl) / np.sum(g_ana * dl))


# Relative L1 distance between the simulated and analytic g(lnR), averaged over seeds; bound
# calibrated on the oracle (N = 8192, 100 ln-bins over 10-5000 um, 0.2 lnR Gaussian smoothing).
GOLOVIN_L1_BOUND = {1200: 0.12, 2400: 0.15, 3600: 0.15}


@pytest.mark.slow
def test_golovin_analytic_spectrum_oracle():
    orc = K.oracle_lib()
    errs = {t: [] for t in GOLOVIN_L1_BOUND}
    for seed in range(4):
        w = W.box_golovin(8192, seed=100 + seed)
        a = make_sdm(w, lib=orc, prefix="oc")
        t = 0
        for t_out in sorted(GOLOVIN_L1_BOUND):
            while t < t_out:
                a.run_step(t * 100, (t + 1) * 100)
                t += 1
            errs[t_out].append(golovin_l1(a.download_supers(), t_out))
        tot0 = float(np.sum(w["supers"]["xi"].astype(np.float64) * w["supers"]["radius"] ** 3))
        d = a.download_supers()
        nd = d["n_domain"]
        tot1 = float(np.sum(d["xi"][:nd].astype(np.float64) * d["radius"][:nd] ** 3))
        assert abs(tot1 - tot0) / tot0 < 1e-12  # water mass conserved
    for t_out, bound in GOLOVIN_L1_BOUND.items():
        assert np.mean(errs[t_out]) < bound, (t_out, errs[t_out])
