"""Loading the CPU checkers and comparing domain states (test infrastructure).

* the oracle: oracle/liboracle.so, the C restatement of the hot path with the host libm, pinned
  bit for bit to CLEO's own sources (built by oracle/Makefile);
* the correctly rounded oracle: oracle/liboracle_cr.so, the same restatement with correctly
  rounded pow and exp, which the CUDA path must match bit for bit;
* the reference build: oracle/_ref/libcleo_ref.so, CLEO's own sources compiled against the
  Kokkos-API shim (present only where CLEO's sources were available to build it).
"""
import ctypes as C
import os
import subprocess

import numpy as np

from cleo_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
ORACLE_CR_SO = os.path.join(ROOT, "oracle", "liboracle_cr.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libcleo_ref.so")

_oracle = {}
_ref = None


def oracle_lib(cr=False):
    """The oracle (host libm), or with cr=True its correctly rounded build."""
    if cr not in _oracle:
        path = ORACLE_CR_SO if cr else ORACLE_SO
        if not os.path.exists(path):
            subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                           capture_output=True)
        lib = C.CDLL(path)
        abi.declare_api(lib, "oc")
        lib.oc_set_num_threads.argtypes = [C.c_int]
        lib.oc_set_num_threads.restype = C.c_int
        P = C.POINTER(abi.Params)
        d = C.POINTER(C.c_double)
        lib.oc_condensation_solve.argtypes = [P, C.c_size_t] + [d] * 6 + [d, C.POINTER(C.c_uint32)]
        lib.oc_condensation_solve.restype = C.c_int
        lib.oc_condensation_solve_seeded.argtypes = ([P, C.c_size_t] + [d] * 7
                                                     + [d, C.POINTER(C.c_uint32)])
        lib.oc_condensation_solve_seeded.restype = C.c_int
        lib.oc_rng_u64.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64]
        lib.oc_rng_u64.restype = C.c_uint64
        lib.oc_rng_drand.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64]
        lib.oc_rng_drand.restype = C.c_double
        lib.oc_rng_urand.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint64,
                                     C.c_uint64, C.c_uint64]
        lib.oc_rng_urand.restype = C.c_uint64
        lib.oc_terminal_velocity.argtypes = [C.c_int, C.c_double]
        lib.oc_terminal_velocity.restype = C.c_double
        lib.oc_pair_probability.argtypes = [P, C.c_double, C.c_uint64, C.c_double, C.c_double,
                                            C.c_uint64, C.c_double, C.c_double]
        lib.oc_pair_probability.restype = C.c_double
        _oracle[cr] = lib
    return _oracle[cr]


def oracle_threads(lib, n=None):
    """Run the oracle's gridbox loops on n threads (default: every host core); results do not
    depend on the count."""
    return lib.oc_set_num_threads(int(n if n is not None else (os.cpu_count() or 1)))


ADAPTER_SO = os.path.join(ROOT, "oracle", "_ref", "libcleo_adapter.so")
_adapter = None


def ref_available():
    return os.path.exists(REF_SO)


def adapter_available():
    return os.path.exists(ADAPTER_SO)


def adapter_lib():
    """CLEO's RunCLEO with the B200 SDMMethods or CLEO's own (oracle/adapter_harness.cpp)."""
    global _adapter
    if _adapter is None:
        abi.load_library()  # the harness links libcleo_b200.so: load it from the package first
        lib = C.CDLL(ADAPTER_SO)
        vp = C.c_void_p
        lib.adp_run_cleo.argtypes = [C.POINTER(abi.Params), C.POINTER(abi.Grid),
                                     C.POINTER(abi.GbxState), C.POINTER(abi.Supers), C.c_size_t,
                                     C.c_uint, C.c_uint32, C.c_uint32, C.c_double, C.c_int,
                                     C.POINTER(vp)]
        lib.adp_run_cleo.restype = C.c_int
        lib.adp_error.argtypes = [vp]
        lib.adp_error.restype = C.c_char_p
        lib.adp_nobs.argtypes = [vp]
        lib.adp_nobs.restype = C.c_size_t
        lib.adp_obs.argtypes = [vp, C.c_size_t, C.POINTER(C.c_uint32), C.POINTER(C.c_size_t),
                                C.POINTER(abi.Supers), C.c_size_t, C.POINTER(abi.GbxState)]
        lib.adp_obs.restype = C.c_int
        lib.adp_free.argtypes = [vp]
        lib.adp_free.restype = None
        _adapter = lib
    return _adapter


def run_cleo(w, t_end, obsstep, b200, amp=0.0, nspacedims=3):
    """RunCLEO over the workload from t = 0 to t_end (model steps), coupling every motion step:
    the list of observations (t, domain superdroplets dict, gridbox states dict), one every
    obsstep."""
    lib = adapter_lib()
    g = abi.grid_struct(w["grid"])
    st = abi.state_struct(w["state"])
    sd = w["supers"]
    n = len(sd["xi"])
    arrs = {k: np.ascontiguousarray(v) for k, v in sd.items()}
    sup = abi.supers_struct(arrs)
    run = C.c_void_p()
    rc = lib.adp_run_cleo(C.byref(w["params"]), C.byref(g), C.byref(st), C.byref(sup), n,
                          int(nspacedims), int(t_end), int(obsstep),
                          float(amp), int(b200), C.byref(run))
    try:
        if rc != 0:
            raise RuntimeError(lib.adp_error(run).decode())
        out = []
        ng = int(w["grid"]["ngbxs"])
        for i in range(lib.adp_nobs(run)):
            o_sd = {k: np.zeros(n, dtype=v.dtype) for k, v in arrs.items()}
            o_st = {f: np.zeros(ng) for f in abi.STATE_FIELDS}
            t, nd = C.c_uint32(), C.c_size_t()
            so, stt = abi.supers_struct(o_sd), abi.state_struct(o_st)
            assert lib.adp_obs(run, i, C.byref(t), C.byref(nd), C.byref(so), n,
                               C.byref(stt)) == 0
            k = int(nd.value)
            out.append((int(t.value), {kk: v[:k] for kk, v in o_sd.items()} | {"n_domain": k},
                        o_st))
        return out
    finally:
        lib.adp_free(run)


def ref_lib():
    global _ref
    if _ref is None:
        lib = C.CDLL(REF_SO)
        abi.declare_api(lib, "ref")
        P = C.POINTER(abi.Params)
        d = C.POINTER(C.c_double)
        lib.ref_set_num_threads.argtypes = [C.c_int]
        lib.ref_set_num_threads.restype = None
        lib.ref_condensation_solve.argtypes = [P, C.c_size_t] + [d] * 6 + [d]
        lib.ref_condensation_solve.restype = C.c_int
        lib.ref_terminal_velocity.argtypes = [C.c_int, C.c_double]
        lib.ref_terminal_velocity.restype = C.c_double
        lib.ref_pair_probability.argtypes = [P, C.c_double, C.c_uint64, C.c_double, C.c_double,
                                             C.c_uint64, C.c_double, C.c_double]
        lib.ref_pair_probability.restype = C.c_double
        lib.ref_cartesian_neighbours.argtypes = [C.POINTER(C.c_uint32), C.c_uint32,
                                                 C.POINTER(C.c_uint32)]
        lib.ref_cartesian_neighbours.restype = None
        _ref = lib
    return _ref


def dptr(a):
    return abi.ptr(a, C.c_double)


def condsolve(lib, prefix, params, w, seed_rsqrd=None):
    n = len(w["radius"])
    out = np.zeros(n)
    arrs = [np.ascontiguousarray(w[k], dtype=np.float64)
            for k in ("radius", "msol", "temp", "press", "s_ratio", "delt")]
    if prefix == "ref":
        rc = lib.ref_condensation_solve(C.byref(params), n, *[dptr(a) for a in arrs], dptr(out))
        return rc, out, None
    it = np.zeros(n, dtype=np.uint32)
    if seed_rsqrd is None:
        rc = lib.oc_condensation_solve(C.byref(params), n, *[dptr(a) for a in arrs], dptr(out),
                                       abi.ptr(it, C.c_uint32))
    else:
        s = np.ascontiguousarray(seed_rsqrd, dtype=np.float64)
        rc = lib.oc_condensation_solve_seeded(C.byref(params), n, *[dptr(a) for a in arrs],
                                              dptr(s), dptr(out), abi.ptr(it, C.c_uint32))
    return rc, out, it


def assert_same_domain(a: dict, b: dict, rtol=1e-12, what=""):
    """In-domain superdroplets: order, gridbox index, xi and id bit-identical; radius, msol and
    coordinates within rtol (relative, FP64). Out-of-domain ones: the same set of ids."""
    assert a["n_domain"] == b["n_domain"], (what, a["n_domain"], b["n_domain"])
    assert a["n_total"] == b["n_total"], (what, a["n_total"], b["n_total"])
    nd = a["n_domain"]
    for k in ("sdid", "sdgbxindex", "xi"):
        x, y = a[k][:nd], b[k][:nd]
        bad = np.nonzero(x != y)[0]
        assert bad.size == 0, (what, k, bad[:10], x[bad[:5]], y[bad[:5]])
    for k in ("radius", "msol", "coord3", "coord1", "coord2"):
        x, y = a[k][:nd], b[k][:nd]
        scale = np.maximum(np.abs(x), np.abs(y))
        err = np.abs(x - y)
        ok = err <= rtol * scale + 1e-300
        if k.startswith("coord"):
            ok |= err <= 1e-15  # coordinates near zero
        bad = np.nonzero(~ok)[0]
        rel = err / np.maximum(scale, 1e-300)
        assert bad.size == 0, (what, k, f"{bad.size} of {nd} beyond rtol; max rel {rel.max():.3e}",
                               bad[:10], x[bad[:5]], y[bad[:5]])
    ia = np.sort(a["sdid"][nd:])
    ib = np.sort(b["sdid"][nd:])
    assert np.array_equal(ia, ib), (what, "oob ids differ")


def assert_identical_domain(a: dict, b: dict, what=""):
    """Every field of every in-domain superdroplet bit for bit (order included); the same set of
    out-of-domain ids."""
    assert a["n_domain"] == b["n_domain"], (what, a["n_domain"], b["n_domain"])
    assert a["n_total"] == b["n_total"], (what, a["n_total"], b["n_total"])
    nd = a["n_domain"]
    for k in ("sdid", "sdgbxindex", "xi", "radius", "msol", "coord3", "coord1", "coord2"):
        x, y = a[k][:nd], b[k][:nd]
        same = (x.view(np.uint64) == y.view(np.uint64)) if x.dtype == np.float64 else (x == y)
        bad = np.nonzero(~same)[0]
        rel = (float(np.max(np.abs(x[bad] - y[bad]) / np.maximum(np.abs(y[bad]), 1e-300)))
               if bad.size and x.dtype == np.float64 else None)
        assert bad.size == 0, (what, k, f"{bad.size} of {nd} differ (max rel {rel})", bad[:10],
                               x[bad[:5]], y[bad[:5]])
    assert np.array_equal(np.sort(a["sdid"][nd:]), np.sort(b["sdid"][nd:])), (what, "oob ids")


def assert_identical_run(g, o, what=""):
    """Two SDM contexts after the same steps: superdroplets, gridbox states and budgets (condensed
    mass and Newton iterations) bit for bit."""
    assert_identical_domain(g.download_supers(), o.download_supers(), what)
    sg, so = g.download_state(), o.download_state()
    for f in abi.STATE_FIELDS:
        bad = np.nonzero(sg[f].view(np.uint64) != so[f].view(np.uint64))[0]
        assert bad.size == 0, (what, f, f"{bad.size} gridboxes differ",
                               max_rel(sg[f][bad], so[f][bad]))
    cg, ig = g.download_budgets()
    co, io = o.download_budgets()
    assert np.array_equal(cg.view(np.uint64), co.view(np.uint64)), (what, "condensed mass",
                                                                    max_rel(cg, co))
    assert np.array_equal(ig, io), (what, "newton iterations")


def max_rel(x, y):
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    s = np.maximum(np.abs(x), np.abs(y))
    s[s == 0] = 1.0
    return float(np.max(np.abs(x - y) / s)) if x.size else 0.0


GOLDEN = os.path.join(ROOT, "tests", "golden")


def params_from_bytes(b) -> abi.Params:
    """Params from stored bytes; fields added after a fixture was written keep their zero
    default (exec_mode 0 = plain)."""
    p = abi.Params()
    raw = bytes(np.asarray(b, dtype=np.uint8))
    n = min(len(raw), C.sizeof(abi.Params))
    C.memmove(C.byref(p), raw, n)
    return p


def load_step_fixture(path):
    """(workload dict, expected outputs dict) of a golden step fixture."""
    z = np.load(path)
    grid = {}
    for k in z.files:
        if k.startswith("grid_"):
            v = z[k]
            grid[k[5:]] = v.item() if v.ndim == 0 else v
    grid["ndims"] = tuple(int(x) for x in grid["ndims"])
    w = {
        "grid": grid,
        "state": {k[9:]: z[k] for k in z.files if k.startswith("in_state_")},
        "supers": {k[6:]: z[k] for k in z.files if k.startswith("in_sd_")},
        "params": params_from_bytes(z["params"]),
        "tstep": int(z["tstep"]),
    }
    exp = {
        "supers": {k[7:]: (z[k].item() if z[k].ndim == 0 else z[k])
                   for k in z.files if k.startswith("out_sd_")},
        "state": {k[10:]: z[k] for k in z.files if k.startswith("out_state_")},
        "cond_mass": z["out_cond_mass"],
        "nsteps": int(z["nsteps"]),
    }
    return w, exp


def step_fixtures():
    return sorted(f for f in os.listdir(GOLDEN) if f.startswith("step_") and f.endswith(".npz"))
