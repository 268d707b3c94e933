"""ctypes mirror of include/cleo_b200.h and the loader of the CUDA library.

The structures here have exactly the field order and types of the C header, so one set of
structures serves the CUDA library (``libcleo_b200.so``) and, in the tests, the CPU checkers that
share its API shape. Loading the CUDA library never falls back to anything: if the shared object
is missing, :func:`load_library` raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libcleo_b200.so"

STEP_OFF = 0xFFFFFFFF
OOB = 0xFFFFFFFF

# status codes (enum cleo_status)
STATUS = {
    0: "CLEO_OK",
    1: "CLEO_ERR_XI_ZERO",
    2: "CLEO_ERR_RADIUS_BELOW_DRY",
    3: "CLEO_ERR_NEG_CONDENSATE",
    4: "CLEO_ERR_COALESCENCE",
    5: "CLEO_ERR_BREAKUP",
    6: "CLEO_ERR_NR_NOCONVERGE",
    7: "CLEO_ERR_SUBDELT",
    8: "CLEO_ERR_CFL",
    9: "CLEO_ERR_OUT_OF_BOX",
    10: "CLEO_ERR_TEMPERATURE",
    11: "CLEO_ERR_CAPACITY",
    12: "CLEO_ERR_ARGUMENT",
    13: "CLEO_ERR_CUDA",
    14: "CLEO_ERR_TIMEOUT",
    15: "CLEO_ERR_MLP",
    16: "CLEO_ERR_XI_OUTPUT",
    17: "CLEO_ERR_IO",
}
CODE = {v: k for k, v in STATUS.items()}

TV_NULL, TV_SIMMEL, TV_ROGERSYAU, TV_ROGERSGK = 0, 1, 2, 3
PROB_GOLOVIN, PROB_LONG, PROB_CONST = 0, 1, 2
ENACT_COALESCENCE, ENACT_BREAKUP, ENACT_COALBURE = 0, 1, 2
NFRAGS_CONST, NFRAGS_CKE = 0, 1
FLAG_STRAUB, FLAG_TESTIKSTRAUB, FLAG_SZAKALLURBICH, FLAG_CONST = 0, 1, 2, 3
NRSEED_REFERENCE, NRSEED_MLP = 0, 1
EXEC_PLAIN, EXEC_BATCHED = 0, 1
MLP_TCGEN05, MLP_MMA_SYNC, MLP_FP32 = 0, 1, 2
MONITOR_MASSMOMENTS, MONITOR_RAINMASSMOMENTS, MONITOR_PRECIPITATION = 1, 2, 4
NITERS_FAILED = 0x80000000  # or-ed into a batch solve's iteration count: that droplet aborted
RESORT_AUTO, RESORT_PAGES, RESORT_FULL = 0, 1, 2
MATH_POW, MATH_EXP, MATH_VENT = 0, 1, 2  # cleo_b200_check_math's functions
MLP_NFEATURES, MLP_NHIDDEN, MLP_NPARAMS, MLP_NNORM = 7, 64, 4737, 16
# enum cleo_obs_var: superdroplet output variables, with their output types
OBS_VARS = {"sdId": (1, np.uint32), "sdgbxindex": (2, np.uint32), "xi": (4, np.uint64),
            "radius": (8, np.float32), "msol": (16, np.float32), "coord3": (32, np.float32),
            "coord1": (64, np.float32), "coord2": (128, np.float32)}
OBS_ALL = 255
# cleo_b200_obs_supers member of each output variable
OBS_MEMBER = {"sdId": "sdid", "sdgbxindex": "sdgbxindex", "xi": "xi", "radius": "radius",
              "msol": "msol", "coord3": "coord3", "coord1": "coord1", "coord2": "coord2"}

_d = C.POINTER(C.c_double)
_u32 = C.POINTER(C.c_uint32)
_u64 = C.POINTER(C.c_uint64)


class Params(C.Structure):
    """cleo_b200_params."""

    _fields_ = [
        ("condstep", C.c_uint32),
        ("collstep", C.c_uint32),
        ("motionstep", C.c_uint32),
        ("pad0", C.c_uint32),
        ("cond_delt", C.c_double),
        ("cond_minsubdelt", C.c_double),
        ("coll_delt", C.c_double),
        ("motion_delt", C.c_double),
        ("do_alter_thermo", C.c_int32),
        ("maxniters", C.c_uint32),
        ("rtol", C.c_double),
        ("atol", C.c_double),
        ("coll_prob", C.c_int32),
        ("coll_enact", C.c_int32),
        ("coaleff", C.c_double),
        ("const_kernel", C.c_double),
        ("nfrags_kind", C.c_int32),
        ("nfrags_tv", C.c_int32),
        ("nfrags", C.c_double),
        ("flag_kind", C.c_int32),
        ("flag_tv", C.c_int32),
        ("flag_coaleff", C.c_double),
        ("seed", C.c_uint64),
        ("motion_tv", C.c_int32),
        ("nr_seed", C.c_int32),
        ("exec_mode", C.c_int32),
        ("monitors", C.c_int32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Grid(C.Structure):
    """cleo_b200_grid (pointers into numpy arrays kept alive by the owner)."""

    _fields_ = [
        ("ngbxs", C.c_uint32),
        ("ndims", C.c_uint32 * 3),
        ("coord3lo", _d), ("coord3hi", _d),
        ("coord1lo", _d), ("coord1hi", _d),
        ("coord2lo", _d), ("coord2hi", _d),
        ("back3", _u32), ("fwd3", _u32),
        ("back1", _u32), ("fwd1", _u32),
        ("back2", _u32), ("fwd2", _u32),
        ("gbxarea", _d),
    ]


STATE_FIELDS = ("volume", "press", "temp", "qvap", "qcond",
                "wvel_lo", "wvel_hi", "uvel_lo", "uvel_hi", "vvel_lo", "vvel_hi")


class GbxState(C.Structure):
    """cleo_b200_gbx_state."""

    _fields_ = [(f, _d) for f in STATE_FIELDS]


SUPERS_FIELDS = (("sdgbxindex", np.uint32), ("coord3", np.float64), ("coord1", np.float64),
                 ("coord2", np.float64), ("xi", np.uint64), ("radius", np.float64),
                 ("msol", np.float64), ("sdid", np.uint64))


class Supers(C.Structure):
    """cleo_b200_supers."""

    _fields_ = [
        ("sdgbxindex", _u32),
        ("coord3", _d), ("coord1", _d), ("coord2", _d),
        ("xi", _u64),
        ("radius", _d), ("msol", _d),
        ("sdid", _u64),
    ]


class Error(C.Structure):
    """cleo_b200_error."""

    _fields_ = [("code", C.c_int32), ("gbxindex", C.c_uint32), ("index", C.c_uint64)]


def ptr(a: np.ndarray, ctype):
    """Pointer to the data of a contiguous numpy array."""
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(ctype))


_CT = {np.float64: C.c_double, np.uint32: C.c_uint32, np.uint64: C.c_uint64}


def supers_struct(arrs: dict) -> Supers:
    """Supers struct pointing at the numpy arrays of ``arrs`` (keys of SUPERS_FIELDS)."""
    s = Supers()
    for name, dt in SUPERS_FIELDS:
        a = arrs.get(name)
        if a is None:
            setattr(s, name, None)
        else:
            assert a.dtype == dt, (name, a.dtype)
            setattr(s, name, ptr(a, _CT[dt]))
    return s


def state_struct(arrs: dict) -> GbxState:
    st = GbxState()
    for f in STATE_FIELDS:
        a = arrs[f]
        assert a.dtype == np.float64
        setattr(st, f, ptr(a, C.c_double))
    return st


def grid_struct(g: dict) -> Grid:
    gr = Grid()
    gr.ngbxs = int(g["ngbxs"])
    for i in range(3):
        gr.ndims[i] = int(g["ndims"][i])
    for f in ("coord3lo", "coord3hi", "coord1lo", "coord1hi", "coord2lo", "coord2hi"):
        setattr(gr, f, ptr(g[f], C.c_double))
    for f in ("back3", "fwd3", "back1", "fwd1", "back2", "fwd2"):
        setattr(gr, f, ptr(g[f], C.c_uint32))
    if g.get("gbxarea") is not None:
        gr.gbxarea = ptr(g["gbxarea"], C.c_double)
    return gr


_f32 = C.POINTER(C.c_float)
MONITOR_FIELDS = (("mom0_micro", np.uint64), ("mom0_motion", np.uint64),
                  ("rain_mom0_micro", np.uint64), ("rain_mom0_motion", np.uint64),
                  ("mom1_micro", np.float32), ("mom2_micro", np.float32),
                  ("mom1_motion", np.float32), ("mom2_motion", np.float32),
                  ("rain_mom1_micro", np.float32), ("rain_mom2_micro", np.float32),
                  ("rain_mom1_motion", np.float32), ("rain_mom2_motion", np.float32),
                  ("precip", np.float64))


class Monitors(C.Structure):
    """cleo_b200_monitors (host pointers; owner keeps the arrays alive)."""

    _fields_ = [(name, {np.uint64: _u64, np.float32: _f32, np.float64: _d}[dt])
                for name, dt in MONITOR_FIELDS]


def monitors_struct(arrs: dict) -> Monitors:
    m = Monitors()
    ct = {np.uint64: C.c_uint64, np.float32: C.c_float, np.float64: C.c_double}
    for name, dt in MONITOR_FIELDS:
        setattr(m, name, ptr(arrs[name], ct[dt]))
    return m


class ObsSupers(C.Structure):
    """cleo_b200_obs_supers (host arrays of the output types; NULL members are skipped)."""

    _fields_ = [("sdid", _u32), ("sdgbxindex", _u32), ("xi", _u64), ("radius", _f32),
                ("msol", _f32), ("coord3", _f32), ("coord1", _f32), ("coord2", _f32)]


def obs_struct(arrs: dict) -> ObsSupers:
    """ObsSupers over arrays keyed by output variable name (absent names stay NULL)."""
    o = ObsSupers()
    ct = {np.uint32: C.c_uint32, np.uint64: C.c_uint64, np.float32: C.c_float}
    for name, (_, dt) in OBS_VARS.items():
        if name in arrs and arrs[name] is not None:
            setattr(o, OBS_MEMBER[name], ptr(arrs[name], ct[dt]))
    return o


def declare_api(lib: C.CDLL, prefix: str) -> C.CDLL:
    """Declare argtypes/restype of the context API ``<prefix>_create`` ... on ``lib``."""
    for name, args in (("monitors_begin", [C.c_void_p]),
                       ("download_monitors", [C.c_void_p, C.POINTER(Monitors), C.c_int])):
        f = getattr(lib, f"{prefix}_{name}", None)
        if f is not None:
            f.argtypes = args
            f.restype = C.c_int
    vp = C.c_void_p
    f = getattr(lib, f"{prefix}_create")
    f.argtypes = [C.POINTER(Params), C.POINTER(Grid), C.c_size_t, C.POINTER(vp)]
    f.restype = C.c_int
    f = getattr(lib, f"{prefix}_destroy")
    f.argtypes = [vp]
    f.restype = None
    f = getattr(lib, f"{prefix}_upload_supers")
    f.argtypes = [vp, C.POINTER(Supers), C.c_size_t]
    f.restype = C.c_int
    f = getattr(lib, f"{prefix}_upload_state")
    f.argtypes = [vp, C.POINTER(GbxState)]
    f.restype = C.c_int
    f = getattr(lib, f"{prefix}_step")
    f.argtypes = [vp, C.c_uint32, C.c_uint32]
    f.restype = C.c_int
    f = getattr(lib, f"{prefix}_status")
    f.argtypes = [vp, C.POINTER(Error)]
    f.restype = C.c_int
    f = getattr(lib, f"{prefix}_download_supers")
    f.argtypes = [vp, C.POINTER(Supers), C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
    f.restype = C.c_int
    f = getattr(lib, f"{prefix}_download_state")
    f.argtypes = [vp, C.POINTER(GbxState)]
    f.restype = C.c_int
    f = getattr(lib, f"{prefix}_download_budgets")
    f.argtypes = [vp, _d, _u64]
    f.restype = C.c_int
    return lib


# Every symbol include/cleo_b200.h declares (checked by the CPU tests against the built library).
EXPORTED = (
    "cleo_b200_create", "cleo_b200_destroy", "cleo_b200_upload_supers", "cleo_b200_upload_state",
    "cleo_b200_step", "cleo_b200_status", "cleo_b200_clear_status", "cleo_b200_domain_nsupers",
    "cleo_b200_download_supers",
    "cleo_b200_download_state", "cleo_b200_download_budgets", "cleo_b200_condensation_solve",
    "cleo_b200_stream", "cleo_b200_kernel_launches", "cleo_b200_resort_stats",
    "cleo_b200_set_resort_policy",
    "cleo_b200_set_profiling",
    "cleo_b200_stage_times", "cleo_b200_sort_by_gridbox_static", "cleo_b200_version",
    "cleo_b200_mlp_create", "cleo_b200_mlp_destroy", "cleo_b200_mlp_set_params",
    "cleo_b200_mlp_get_params", "cleo_b200_mlp_features", "cleo_b200_mlp_fit_normalisation",
    "cleo_b200_mlp_loss_grad", "cleo_b200_mlp_train", "cleo_b200_mlp_infer",
    "cleo_b200_set_surrogate", "cleo_b200_set_graphs", "cleo_b200_autotune",
    "cleo_b200_tuned_config", "cleo_b200_set_launch_config", "cleo_b200_monitors_begin",
    "cleo_b200_download_monitors",
    "cleo_b200_upload_state_async", "cleo_b200_download_budgets_async", "cleo_b200_synchronize",
    "cleo_b200_check_bounded_wait", "cleo_b200_check_math",
    "cleo_b200_gather_supers", "cleo_b200_zarr_open", "cleo_b200_zarr_observe",
    "cleo_b200_zarr_observe_host", "cleo_b200_zarr_close",
)

_LIB = None


def load_library(path: os.PathLike | str | None = None) -> C.CDLL:
    """Load libcleo_b200.so (built in-tree by ``__graft_entry__.build()``); raises if absent."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(
            f"{p} is missing: build the CUDA library first (python -c "
            f"'import __graft_entry__ as g; g.build()'); there is no CPU fallback")
    lib = C.CDLL(str(p), mode=C.RTLD_GLOBAL)
    declare_api(lib, "cleo_b200")
    vp = C.c_void_p
    lib.cleo_b200_domain_nsupers.argtypes = [vp, C.POINTER(C.c_size_t)]
    lib.cleo_b200_domain_nsupers.restype = C.c_int
    lib.cleo_b200_condensation_solve.argtypes = [vp, C.c_size_t] + [vp] * 6 + [vp, vp]
    lib.cleo_b200_condensation_solve.restype = C.c_int
    lib.cleo_b200_stream.argtypes = [vp]
    lib.cleo_b200_stream.restype = vp
    lib.cleo_b200_kernel_launches.argtypes = [vp, C.POINTER(C.c_uint64)]
    lib.cleo_b200_kernel_launches.restype = C.c_int
    lib.cleo_b200_resort_stats.argtypes = [vp, C.POINTER(C.c_uint64)]
    lib.cleo_b200_resort_stats.restype = C.c_int
    lib.cleo_b200_set_resort_policy.argtypes = [vp, C.c_int]
    lib.cleo_b200_set_resort_policy.restype = C.c_int
    lib.cleo_b200_set_profiling.argtypes = [vp, C.c_int]
    lib.cleo_b200_set_profiling.restype = C.c_int
    lib.cleo_b200_stage_times.argtypes = [vp, C.POINTER(C.c_double), C.POINTER(C.c_uint64)]
    lib.cleo_b200_stage_times.restype = C.c_int
    lib.cleo_b200_sort_by_gridbox_static.argtypes = [vp, C.c_uint32, C.c_uint32, vp, vp, vp]
    lib.cleo_b200_sort_by_gridbox_static.restype = C.c_int
    lib.cleo_b200_version.argtypes = []
    lib.cleo_b200_version.restype = C.c_char_p
    fp = C.POINTER(C.c_float)
    for name, args in (
            ("mlp_create", [vp, C.c_uint64, C.POINTER(vp)]),
            ("mlp_destroy", [vp]),
            ("mlp_set_params", [vp, fp, fp]),
            ("mlp_get_params", [vp, fp, fp]),
            ("mlp_features", [vp, C.c_size_t] + [vp] * 10),
            ("mlp_fit_normalisation", [vp, C.c_size_t, vp, vp]),
            ("mlp_loss_grad", [vp, C.c_size_t, vp, vp, vp, vp]),
            ("mlp_train", [vp, C.c_size_t, vp, vp, C.c_uint32, C.c_uint32, C.c_float,
                           C.c_uint64, vp]),
            ("mlp_infer", [vp, C.c_size_t, vp, vp, C.c_int]),
            ("set_surrogate", [vp, vp]),
            ("clear_status", [vp]),
            ("set_graphs", [vp, C.c_int]),
            ("autotune", [vp, C.c_int]),
            ("tuned_config", [vp, C.POINTER(C.c_int32)]),
            ("set_launch_config", [vp, C.POINTER(C.c_int32)]),
            ("upload_state_async", [vp, C.POINTER(GbxState)]),
            ("download_budgets_async", [vp, vp, vp]),
            ("synchronize", [vp]),
            ("check_bounded_wait", [C.c_uint32]),
            ("check_math", [C.c_int, vp, vp, vp, C.c_size_t]),
            ("gather_supers", [vp, C.c_uint32, C.POINTER(ObsSupers), C.c_size_t,
                               C.POINTER(C.c_size_t)]),
            ("zarr_open", [C.c_char_p, C.c_size_t, C.c_uint32, C.c_uint32, C.POINTER(vp)]),
            ("zarr_observe", [vp, vp, C.c_uint32]),
            ("zarr_observe_host", [vp, C.c_uint32, C.POINTER(ObsSupers), C.c_size_t]),
            ("zarr_close", [vp])):
        f = getattr(lib, "cleo_b200_" + name)
        f.argtypes = args
        f.restype = C.c_int
    if path is None:
        _LIB = lib
    return lib
