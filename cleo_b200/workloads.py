"""Seeded synthetic superdroplet populations with the shapes of the benchmark configurations.

There is no public dataset for this path; populations are drawn from the distributions that the
configurations name (and that cleopy's generators use: volume-exponential radii,
attrgens_shima2009.py:22-76; lognormal dry radii, initsuperdropsbinary_src/probdists.py:125-177;
divergence-free 2-D flow, thermobinary_src/windsgen.py:57-73). All arrays are SoA numpy arrays
in CLEO's non-dimensional units, keyed like ``abi.SUPERS_FIELDS`` / ``abi.STATE_FIELDS``.

Workloads:
  box_golovin   1 gridbox of 1e6 m^3, N superdroplets, equal xi, Golovin coalescence.
  rainshaft     1 x 1 x nz column of 20 m boxes, condensation + Long collisions + sedimentation.
  uneven3d      nz x nx x ny boxes of 50 m^3, lognormal counts (median 32, clip 0..2048),
                condensation + Long CoalBuRe (ConstNFrags 5, Straub flag) + sedimentation.
  bubble3d      nz x nx x ny boxes of 25 m^3, lognormal counts (median 16, mean 24), prescribed
                2-D divergence-free flow (w_max = 2 m/s) + condensation + CoalBuRe.
  condsolve     independent droplets for the batched condensation solve.
"""
from __future__ import annotations

import math

import numpy as np

from . import abi
from .config import (COORD0, LLIM, Mr_ratio, P0, R0, RHO0, Rho_sol, TEMP0, VOL0, Mr_sol,
                     cartesian_grid, make_params)

# ---------------------------------------------------------------------------------------------
# thermodynamics used only to generate inputs (numpy restatement of
# thermodynamic_equations.cpp:38-52 and thermodynamic_equations.hpp:95-107)
# ---------------------------------------------------------------------------------------------


def psat_dimless(temp_dimless):
    T = temp_dimless * TEMP0
    return (611.655 * np.exp(17.4146 * (T - 273.16) / (T - 33.639))) / P0


def kohler_ab(msol, temp_dimless):
    akoh = (3.3e-7 / (TEMP0 * R0)) / temp_dimless
    bkoh = (4.3e-6 * RHO0 / 0.028966216) * msol * 2.0 / Mr_sol
    return akoh, bkoh


def msol_from_dryradius(rdry):
    """msol such that SuperdropAttrs::dryradius() == rdry (superdrop_attrs.hpp:227-231)."""
    return rdry ** 3 * (4.0 * math.pi / 3.0) * Rho_sol


def equilibrium_radius(rdry, msol, s_ratio, temp, iters=44):
    """Stable Kohler equilibrium radius below the critical radius for saturation ratio s.

    Solves s - 1 - a/r + b/r^3 = 0 on (r_dry, r_crit] by bisection; supersaturations above the
    critical one are capped just below it, so every droplet starts unactivated.
    """
    a, b = kohler_ab(msol, temp)
    a = np.broadcast_to(a, rdry.shape)
    rcrit = np.sqrt(3.0 * b / a)
    scrit = 1.0 + np.sqrt(4.0 * a ** 3 / (27.0 * b))
    sm1 = np.minimum(s_ratio, 1.0 + 0.999 * (scrit - 1.0)) - 1.0
    lo = np.maximum(rdry * (1.0 + 1e-9), 1e-12)
    hi = np.maximum(rcrit, lo)
    if lo.size > 1_000_000:
        try:  # same IEEE element-wise arithmetic, on the GPU when there is one, else host cores
            import torch
            dev = "cuda" if torch.cuda.is_available() else "cpu"
            T = {k: torch.from_numpy(np.array(v, dtype=np.float64, copy=True)).to(dev)
                 for k, v in (("a", a), ("b", np.broadcast_to(b, lo.shape)), ("sm1", sm1),
                              ("lo", lo), ("hi", hi))}
            lo_t, hi_t = T["lo"].clone(), T["hi"].clone()
            for _ in range(iters):
                mid = (lo_t + hi_t) * 0.5
                f = (T["b"] / (mid * mid * mid) - T["a"] / mid) + T["sm1"]
                up = f > 0.0
                lo_t = torch.where(up, mid, lo_t)
                hi_t = torch.where(up, hi_t, mid)
            return np.maximum(((lo_t + hi_t) * 0.5).cpu().numpy(), rdry)
        except ImportError:
            pass
    mid = np.empty_like(lo)
    f = np.empty_like(lo)
    tmp = np.empty_like(lo)
    up = np.empty(lo.shape, dtype=bool)
    for _ in range(iters):
        np.add(lo, hi, out=mid)
        mid *= 0.5
        np.divide(a, mid, out=f)          # a/r
        np.multiply(mid, mid, out=tmp)
        tmp *= mid                        # r^3
        np.divide(b, tmp, out=tmp)        # b/r^3
        np.subtract(tmp, f, out=f)
        f += sm1                          # f = s - 1 - a/r + b/r^3, decreasing on (r_dry, r_crit)
        np.greater(f, 0.0, out=up)
        np.copyto(lo, mid, where=up)
        np.logical_not(up, out=up)
        np.copyto(hi, mid, where=up)
    r = 0.5 * (lo + hi)
    return np.maximum(r, rdry)


def qvap_from_s(s_ratio, press, psat):
    """Inverse of supersaturation_ratio (thermodynamic_equations.hpp:78-81)."""
    return s_ratio * Mr_ratio * psat / (press - s_ratio * psat)


def column_thermo(zc_m, rng, rh_lo=0.95, rh_hi=1.01, t_bottom=300.0, lapse_per_m=30.0 / 5120.0):
    """Linear T profile from 300 K, hydrostatic p from 1000 hPa, per-box RH in [rh_lo, rh_hi]."""
    T = t_bottom - lapse_per_m * zc_m
    Hs = 287.04 * 0.5 * (t_bottom + T) / 9.80665
    p = 100000.0 * np.exp(-zc_m / Hs)
    rh = rng.uniform(rh_lo, rh_hi, size=zc_m.shape)
    temp = T / TEMP0
    press = p / P0
    qvap = qvap_from_s(rh, press, psat_dimless(temp))
    return temp, press, qvap, rh


def make_state(ngbxs, volume_dimless, temp, press, qvap, w=None, u=None, v=None):
    st = {f: np.zeros(ngbxs, dtype=np.float64) for f in abi.STATE_FIELDS}
    st["volume"][:] = volume_dimless
    st["temp"][:] = temp
    st["press"][:] = press
    st["qvap"][:] = qvap
    for key, val in (("wvel", w), ("uvel", u), ("vvel", v)):
        if val is not None:
            st[key + "_lo"][:] = val[0]
            st[key + "_hi"][:] = val[1]
    return st


def _supers_empty(n):
    return {name: np.zeros(n, dtype=dt) for name, dt in abi.SUPERS_FIELDS}


def populate(grid, counts, rng, *, rdry_geomean_um=0.02, rdry_sigma=1.5, numconc_m3=1.325e9,
             temp=None, s_ratio=None):
    """Superdroplets with lognormal NaCl dry radii and Kohler-equilibrium wet radii per gridbox.

    ``counts[g]`` superdroplets in gridbox g, sorted by gridbox, uniform positions inside it;
    xi from the number concentration split evenly among the gridbox's superdroplets.
    """
    counts = np.asarray(counts, dtype=np.int64)
    n = int(counts.sum())
    sd = _supers_empty(n)
    gbx = np.repeat(np.arange(grid["ngbxs"], dtype=np.uint32), counts)
    sd["sdgbxindex"][:] = gbx
    sd["sdid"][:] = np.arange(n, dtype=np.uint64)
    for c in ("coord3", "coord1", "coord2"):
        lo = grid[c + "lo"][gbx]
        hi = grid[c + "hi"][gbx]
        null = (lo == LLIM)
        u = rng.random(n)
        with np.errstate(over="ignore", invalid="ignore"):
            sd[c][:] = np.where(null, 0.0, lo + u * (hi - lo))
        # keep strictly inside [lo, hi)
        sd[c][:] = np.where(null, 0.0, np.minimum(sd[c], np.nextafter(hi, lo)))
    rdry = np.exp(rng.normal(math.log(rdry_geomean_um), math.log(rdry_sigma), size=n))
    rdry = np.clip(rdry, 1e-3, 10.0)
    msol = msol_from_dryradius(rdry)
    sd["msol"][:] = msol
    if temp is None:
        sd["radius"][:] = rdry * 2.0
    else:
        sd["radius"][:] = equilibrium_radius(rdry, msol, s_ratio[gbx], temp[gbx])
    vol_m3 = grid["volume_m3"]
    xi_box = np.maximum(1, np.round(numconc_m3 * vol_m3 / np.maximum(counts, 1))).astype(np.uint64)
    sd["xi"][:] = xi_box[gbx]
    return sd


# ---------------------------------------------------------------------------------------------
# configurations
# ---------------------------------------------------------------------------------------------

def box_golovin(n_sd=8192, seed=1, volume_m3=1e6, numconc=2 ** 23, r0_um=30.531):
    """Golovin box model: 0-D gridbox, equal xi = numconc*V/N, volume-exponential radii."""
    rng = np.random.default_rng(seed)
    grid = cartesian_grid((1, 1, 1), (100.0, 100.0, 100.0), nspacedims=0)
    grid["volume_m3"] = volume_m3
    sd = _supers_empty(n_sd)
    sd["sdid"][:] = np.arange(n_sd, dtype=np.uint64)
    vmean = 4.0 / 3.0 * math.pi * r0_um ** 3
    r = np.empty(0)
    while r.size < n_sd:  # volume-exponential, truncated to [0.62 um, 6.34 cm] like the config
        v = rng.exponential(vmean, size=2 * n_sd)
        rr = (3.0 * v / (4.0 * math.pi)) ** (1.0 / 3.0)
        r = np.concatenate([r, rr[(rr >= 0.62) & (rr <= 6.34e4)]])
    sd["radius"][:] = r[:n_sd]
    sd["msol"][:] = msol_from_dryradius(1e-16 / R0)
    sd["xi"][:] = np.uint64(int(numconc * volume_m3) // n_sd)
    st = make_state(1, volume_m3 / VOL0, 300.0 / TEMP0, 1.0, 0.01)
    params = make_params(colltstep=1.0, coll_prob=abi.PROB_GOLOVIN,
                         coll_enact=abi.ENACT_COALESCENCE, seed=seed)
    return dict(name="box_golovin", grid=grid, state=st, supers=sd, params=params,
                tstep=100, n_sd=n_sd)


def rainshaft(nz=256, per_gbx=256, seed=2, dz=20.0, coll=True, cond=True, motion=True):
    """1-D rain shaft: 1 x 1 x nz column of dz boxes, per_gbx superdroplets each."""
    rng = np.random.default_rng(seed)
    grid = cartesian_grid((nz, 1, 1), (dz, dz, dz), nspacedims=1)
    zc = (np.arange(nz) + 0.5) * dz
    temp, press, qvap, rh = column_thermo(zc, rng)
    st = make_state(nz, grid["volume_m3"] / VOL0, temp, press, qvap)
    psat = psat_dimless(temp)
    s_ratio = press * qvap / ((Mr_ratio + qvap) * psat)
    counts = np.full(nz, per_gbx)
    sd = populate(grid, counts, rng, temp=temp, s_ratio=s_ratio)
    params = make_params(condtstep=1.0 if cond else None, colltstep=1.0 if coll else None,
                         motiontstep=1.0 if motion else None, maxniters=50, rtol=0.0, atol=0.01,
                         minsubtstep=0.001, coll_prob=abi.PROB_LONG,
                         coll_enact=abi.ENACT_COALESCENCE, coaleff=1.0, seed=seed,
                         motion_tv=abi.TV_ROGERSGK)
    return dict(name="rainshaft", grid=grid, state=st, supers=sd, params=params, tstep=100,
                n_sd=int(counts.sum()))


def lognormal_counts(ngbxs, rng, median, sigma, cap=2048):
    c = np.round(np.exp(rng.normal(math.log(median), sigma, size=ngbxs)))
    return np.clip(c, 0, cap).astype(np.int64)


def uneven3d(ndims=(64, 128, 128), seed=3, volume_m3=50.0, median=32.0, sigma=0.586,
             cond=True, coll=True, motion=True, nfrags=5.0):
    """3-D uneven counts: boxes of volume_m3, lognormal per-box count (median, sigma)."""
    rng = np.random.default_rng(seed)
    d = volume_m3 ** (1.0 / 3.0)
    grid = cartesian_grid(ndims, (d, d, d), nspacedims=3)
    grid["volume_m3"] = volume_m3
    ngbxs = grid["ngbxs"]
    zc = 0.5 * (grid["coord3lo"] + grid["coord3hi"]) * COORD0
    temp, press, qvap, rh = column_thermo(zc, rng)
    st = make_state(ngbxs, volume_m3 / VOL0, temp, press, qvap)
    psat = psat_dimless(temp)
    s_ratio = press * qvap / ((Mr_ratio + qvap) * psat)
    counts = lognormal_counts(ngbxs, rng, median, sigma)
    sd = populate(grid, counts, rng, temp=temp, s_ratio=s_ratio)
    params = make_params(condtstep=1.0 if cond else None, colltstep=1.0 if coll else None,
                         motiontstep=1.0 if motion else None, maxniters=50, rtol=0.0, atol=0.01,
                         minsubtstep=0.001, coll_prob=abi.PROB_LONG,
                         coll_enact=abi.ENACT_COALBURE, coaleff=1.0,
                         nfrags_kind=abi.NFRAGS_CONST, nfrags=nfrags,
                         flag_kind=abi.FLAG_STRAUB, flag_tv=abi.TV_ROGERSGK, seed=seed,
                         motion_tv=abi.TV_ROGERSGK)
    return dict(name="uneven3d", grid=grid, state=st, supers=sd, params=params, tstep=100,
                n_sd=int(counts.sum()), counts=counts)


def divfree_flow(grid, wmax=2.0):
    """Face winds of a steady divergence-free 2-D (z, x) flow (windsgen.py:57-73), dimensionless.

    W = wamp sin(z/zt) sin(x/xt), U = wamp (xt/zt) cos(z/zt) cos(x/xt), zt = Lz/pi,
    xt = Lx/(2 pi), density factor 1. windsgen.py uses wamp = 2*WMAX; here wamp = wmax so that
    the peak vertical wind is w_max (2 m/s keeps the 1 s motion step within CFL for ~3 m boxes,
    where 4 m/s would make the reference abort in cfl_criteria.hpp:52-54).
    """
    nz, nx, ny = grid["ndims"]
    Lz = (grid["coord3hi"].max() - grid["coord3lo"].min()) * COORD0
    Lx = (grid["coord1hi"].max() - grid["coord1lo"].min()) * COORD0
    zt, xt = Lz / math.pi, Lx / (2.0 * math.pi)
    z0, z1 = grid["coord3lo"] * COORD0, grid["coord3hi"] * COORD0
    x0, x1 = grid["coord1lo"] * COORD0, grid["coord1hi"] * COORD0
    xc = 0.5 * (x0 + x1)
    zc = 0.5 * (z0 + z1)
    W = lambda z, x: wmax * np.sin(z / zt) * np.sin(x / xt)
    U = lambda z, x: wmax * (xt / zt) * np.cos(z / zt) * np.cos(x / xt)
    w = (W(z0, xc), W(z1, xc))
    u = (U(zc, x0), U(zc, x1))
    return w, u


def bubble3d(ndims=(128, 256, 256), seed=5, volume_m3=25.0, median=16.0, sigma=0.9005):
    """Coupled 3-D bubble shape: lognormal counts (median 16, mean 24), prescribed 2-D flow."""
    wl = uneven3d(ndims=ndims, seed=seed, volume_m3=volume_m3, median=median, sigma=sigma)
    w, u = divfree_flow(wl["grid"])
    for k, val in (("wvel", w), ("uvel", u)):
        wl["state"][k + "_lo"][:] = val[0]
        wl["state"][k + "_hi"][:] = val[1]
    wl["name"] = "bubble3d"
    return wl


def condsolve(n, seed=4):
    """Independent droplets for batched condensation solves (dimensionless inputs).

    Dry radius lognormal (0.02 um, 1.5); wet radius log-uniform in [0.01, 100] um resampled to
    r >= r_dry; supersaturation s-1 uniform in [-0.05, 0.02]; T uniform [250, 305] K; p uniform
    [50, 101] kPa; dt in {0.5, 1, 2} s.
    """
    rng = np.random.default_rng(seed)
    rdry = np.clip(np.exp(rng.normal(math.log(0.02), math.log(1.5), size=n)), 1e-3, 10.0)
    msol = msol_from_dryradius(rdry)
    r = np.exp(rng.uniform(math.log(0.01), math.log(100.0), size=n))
    bad = r < rdry
    while bad.any():
        r[bad] = np.exp(rng.uniform(math.log(0.01), math.log(100.0), size=int(bad.sum())))
        bad = r < rdry
    s = 1.0 + rng.uniform(-0.05, 0.02, size=n)
    temp = rng.uniform(250.0, 305.0, size=n) / TEMP0
    press = rng.uniform(50e3, 101e3, size=n) / P0
    delt = rng.choice(np.array([0.5, 1.0, 2.0]), size=n) / 1000.0
    return dict(radius=r, msol=msol, temp=temp, press=press, s_ratio=s, delt=delt, rdry=rdry)
