"""Host-side construction of parameters and Cartesian gridbox maps, mirroring the reference.

* Timestep conversions follow libs/initialise/timesteps.hpp:34-59 (model_step = 1e-5 TIME0 =
  0.01 s, std::chrono double conversions).
* :func:`make_params` fills ``cleo_b200_params`` with the arguments the reference factories take
  (Condensation, condensation.hpp:242-253; CollCoal / CoalBuRe / CollBu, coalescence.hpp:133-160,
  coalbure.hpp:156-185, breakup.hpp:97-123; CartesianMotion, cartesian_motion.hpp:60-66).
* :func:`cartesian_grid` builds the content of CartesianMaps for an undecomposed domain
  (createcartesianmaps.cpp:143-285): per-gridbox bounds, finite z / periodic x,y neighbours
  (doubly_periodic_domain.hpp:41-101, domainboundaries.hpp:34-88) and null maps for directions a
  model does not resolve.
"""
from __future__ import annotations

import numpy as np

from .abi import (ENACT_COALBURE, ENACT_COALESCENCE, FLAG_STRAUB, NFRAGS_CONST, NRSEED_REFERENCE,
                  OOB, PROB_GOLOVIN, STEP_OFF, TV_NULL, TV_ROGERSGK, Params)

# libs/cleoconstants.hpp
TIME0 = 1000.0
COORD0 = 1000.0
VOL0 = COORD0 * COORD0 * COORD0
R0 = 1e-6
P0 = 100000.0
TEMP0 = 273.15
CP0 = 1004.64
RHO0 = P0 / (CP0 * TEMP0)
MR0 = 0.028966216
RHO_SOL = 2016.5
RHO_L = 998.203
Rho_sol = RHO_SOL / RHO0
Rho_l = RHO_L / RHO0
Mr_sol = 0.05844277 / MR0
Mr_ratio = 0.01801528 / 0.028966216
LLIM = -np.finfo(np.float64).max
ULIM = np.finfo(np.float64).max
MODEL_STEP_DEN = 100000  # model_step = duration<int, ratio<1, 100000>>


def realtime2step(tstep_s: float) -> int:
    """timesteps.hpp:40-43: round(TSTEP / TIME0 in model_step units)."""
    return int(round((tstep_s / TIME0) * MODEL_STEP_DEN))


def step2dimlesstime(mdlstep: int) -> float:
    """timesteps.hpp:55-58: secd{model_step{mdlstep}}.count() = mdlstep / 100000."""
    return float(mdlstep) / float(MODEL_STEP_DEN)


def step2realtime(mdlstep: int) -> float:
    """timesteps.hpp:49-52."""
    return step2dimlesstime(mdlstep) * TIME0


def realtime2dimless(tstep_s: float) -> float:
    """timesteps.hpp:46-47."""
    return tstep_s / TIME0


def make_params(*, condtstep: float | None = None, colltstep: float | None = None,
                motiontstep: float | None = None, do_alter_thermo: bool = False,
                maxniters: int = 50, rtol: float = 0.0, atol: float = 0.01,
                minsubtstep: float = 0.001, coll_prob: int = PROB_GOLOVIN,
                coll_enact: int = ENACT_COALESCENCE, coaleff: float = 1.0,
                const_kernel: float = 1.0, nfrags_kind: int = NFRAGS_CONST, nfrags: float = 5.0,
                nfrags_tv: int = TV_ROGERSGK, flag_kind: int = FLAG_STRAUB,
                flag_tv: int = TV_ROGERSGK, flag_coaleff: float = 1.0, seed: int = 0,
                motion_tv: int = TV_NULL, nr_seed: int = NRSEED_REFERENCE,
                exec_mode: int = 1, monitors: int = 0) -> Params:
    """Parameters of one SDM configuration. A timestep of None switches that process off."""
    p = Params()
    p.condstep = STEP_OFF if condtstep is None else realtime2step(condtstep)
    p.collstep = STEP_OFF if colltstep is None else realtime2step(colltstep)
    p.motionstep = STEP_OFF if motiontstep is None else realtime2step(motiontstep)
    # a switched-off condensation still gets a delt >= minsubdelt (ImplicitEuler ctor check)
    p.cond_delt = step2dimlesstime(p.condstep if condtstep is not None else 1)
    p.cond_minsubdelt = realtime2dimless(minsubtstep)
    if condtstep is None:
        p.cond_delt = max(p.cond_delt, p.cond_minsubdelt)
    p.coll_delt = step2realtime(p.collstep) if colltstep is not None else 0.0
    p.motion_delt = step2dimlesstime(p.motionstep) if motiontstep is not None else 0.0
    p.do_alter_thermo = int(bool(do_alter_thermo))
    p.maxniters = int(maxniters)
    p.rtol = float(rtol)
    p.atol = float(atol)
    p.coll_prob = int(coll_prob)
    p.coll_enact = int(coll_enact)
    p.coaleff = float(coaleff)
    p.const_kernel = float(const_kernel)
    p.nfrags_kind = int(nfrags_kind)
    p.nfrags_tv = int(nfrags_tv)
    p.nfrags = float(nfrags)
    p.flag_kind = int(flag_kind)
    p.flag_tv = int(flag_tv)
    p.flag_coaleff = float(flag_coaleff)
    p.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
    p.motion_tv = int(motion_tv)
    p.nr_seed = int(nr_seed)
    p.exec_mode = int(exec_mode)
    p.monitors = int(monitors)
    return p


def _finite_nghbrs(idx: np.ndarray, inc: int, ndim: int):
    """finitedomain_nghbrs, domainboundaries.hpp:46-63 (unsigned int arithmetic)."""
    idx = idx.astype(np.uint64)
    fwd = idx + inc
    back = (idx - inc) & 0xFFFFFFFF
    back = np.where((idx // inc) % ndim == 0, OOB, back)
    fwd = np.where((fwd // inc) % ndim == 0, OOB, fwd)
    return back.astype(np.uint32), fwd.astype(np.uint32)


def _periodic_nghbrs(idx: np.ndarray, inc: int, ndim: int):
    """periodicdomain_nghbrs, domainboundaries.hpp:71-88."""
    idx = idx.astype(np.int64)
    fwd = idx + inc
    back = idx - inc
    back = np.where((idx // inc) % ndim == 0, idx + (ndim - 1) * inc, back)
    fwd = np.where((fwd // inc) % ndim == 0, idx - (ndim - 1) * inc, fwd)
    return back.astype(np.uint32), fwd.astype(np.uint32)


def cartesian_grid(ndims, spacing_m, nspacedims: int = 3, origin_m=(0.0, 0.0, 0.0)) -> dict:
    """Maps of a regular Cartesian grid. ndims = (nz, nx, ny); spacing_m = (dz, dx, dy) metres.

    Bounds are dimensionless (metres / COORD0). Directions beyond ``nspacedims`` (order z, x, y)
    get null bounds and self neighbours (createcartesianmaps.cpp:38-45, 262-327).
    """
    nz, nx, ny = (int(n) for n in ndims)
    ngbxs = nz * nx * ny
    idx = np.arange(ngbxs, dtype=np.uint64)
    iz = idx % nz
    ix = (idx // nz) % nx
    iy = idx // (nz * nx)
    g = {"ngbxs": ngbxs, "ndims": (nz, nx, ny)}
    for name, i, d, o, used in (("coord3", iz, spacing_m[0], origin_m[0], nspacedims >= 1),
                                ("coord1", ix, spacing_m[1], origin_m[1], nspacedims >= 2),
                                ("coord2", iy, spacing_m[2], origin_m[2], nspacedims >= 3)):
        if used:
            lo = (o + i.astype(np.float64) * d) / COORD0
            hi = (o + (i.astype(np.float64) + 1.0) * d) / COORD0
        else:
            lo = np.full(ngbxs, LLIM)
            hi = np.full(ngbxs, ULIM)
        g[name + "lo"] = np.ascontiguousarray(lo, dtype=np.float64)
        g[name + "hi"] = np.ascontiguousarray(hi, dtype=np.float64)
    selfn = idx.astype(np.uint32)
    if nspacedims >= 1:
        g["back3"], g["fwd3"] = _finite_nghbrs(idx, 1, nz)
    else:
        g["back3"], g["fwd3"] = selfn.copy(), selfn.copy()
    if nspacedims >= 2:
        g["back1"], g["fwd1"] = _periodic_nghbrs(idx, nz, nx)
    else:
        g["back1"], g["fwd1"] = selfn.copy(), selfn.copy()
    if nspacedims >= 3:
        g["back2"], g["fwd2"] = _periodic_nghbrs(idx, nz * nx, ny)
    else:
        g["back2"], g["fwd2"] = selfn.copy(), selfn.copy()
    for k in ("back3", "fwd3", "back1", "fwd1", "back2", "fwd2"):
        g[k] = np.ascontiguousarray(g[k], dtype=np.uint32)
    g["volume_m3"] = float(spacing_m[0] * spacing_m[1] * spacing_m[2])
    # horizontal area from the gridbox extents, as a gridfile holds them for every model
    # dimension (GbxBoundsFromBinary::gbxarea, gbx_bounds_from_binary.cpp:206-215)
    g["gbxarea"] = np.full(ngbxs, (spacing_m[1] / COORD0) * (spacing_m[2] / COORD0))
    return g
