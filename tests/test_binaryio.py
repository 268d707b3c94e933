"""CLEO's binary input files (gridbox boundaries, initial superdroplets, coupled dynamics from
files) read by cleo_b200/binaryio.py: against the arrays that tests/golden/make_binaries.py wrote
with the reference's own writer, against CLEO's C++ readers (GbxBoundsFromBinary,
InitAllSupersFromBinary, CartesianDynamics) compiled in the reference build, and end to end:
a domain initialised and driven from the files steps the same in the oracle and in CLEO."""
import ctypes as C
import os

import numpy as np
import pytest

import checkers as K
from cleo_b200 import abi, binaryio as B
from cleo_b200.config import make_params
from cleo_b200.sdm import SDM

G = K.GOLDEN
EXP = np.load(os.path.join(G, "binaries.npz"))
PATHS = {f: os.path.join(G, f"dimless_{f}.dat") for f in B.FromFileDynamics.FIELDS}
GRIDFILE = os.path.join(G, "dimlessGBxboundaries.dat")
SUPERSFILE = os.path.join(G, "dimlessSDsinit.dat")
needs_ref = pytest.mark.skipif(not K.ref_available(), reason="reference build absent")


def test_layout_and_metadata():
    metastr, meta, raw = B.read_binary(SUPERSFILE)
    assert "sdgbxindex, xi, radius, msol" in metastr
    assert [m.bsize for m in meta] == [4, 8, 8, 8, 8, 8, 8]
    assert [m.vtype for m in meta] == [b"I", b"Q", b"d", b"d", b"d", b"d", b"d"]
    assert meta[2].scale_factor == 1e-6 and meta[4].scale_factor == 1000.0
    assert meta[-1].b0 + meta[-1].nvar * meta[-1].bsize == len(raw)


def test_readers_match_written_arrays():
    g = B.gridfile(GRIDFILE, 3)
    b = EXP["bounds"]
    for k, name in enumerate(("coord3", "coord1", "coord2")):
        assert np.array_equal(g[name + "lo"], b[:, 2 * k])
        assert np.array_equal(g[name + "hi"], b[:, 2 * k + 1])
    assert tuple(g["ndims"]) == tuple(int(v) for v in EXP["ndims"])
    sd = B.initsupers(SUPERSFILE, 3)
    for k in ("xi", "radius", "msol", "coord3", "coord1", "coord2"):
        assert np.array_equal(sd[k], EXP[k]), k
    assert np.array_equal(sd["sdgbxindex"], EXP["gbx"])
    dyn = B.FromFileDynamics(PATHS, EXP["ndims"], 3, int(EXP["nsteps"]))
    ng = g["ngbxs"]
    for s in range(int(EXP["nsteps"])):
        st = dyn.state(g["volume"])
        assert np.array_equal(st["press"], EXP["dyn_press"][s * ng:(s + 1) * ng])
        dyn.advance()


def _ref_fns():
    lib = K.ref_lib()
    d, u32, u64 = C.POINTER(C.c_double), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64)
    lib.ref_read_gridfile.argtypes = [C.c_char_p, C.c_size_t, C.c_uint, d, d, d]
    lib.ref_read_initsupers.argtypes = [C.c_char_p, C.c_size_t, C.c_uint, u32, u64] + [d] * 5
    lib.ref_fromfile_state.argtypes = [C.POINTER(C.c_char_p), C.c_uint, u64, C.c_uint, C.c_uint,
                                       C.POINTER(d)]
    return lib


@needs_ref
def test_readers_match_cleo_readers():
    lib = _ref_fns()
    g = B.gridfile(GRIDFILE, 3)
    ng = g["ngbxs"]
    bounds, areas, vols = np.zeros(6 * ng), np.zeros(ng), np.zeros(ng)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))  # noqa: E731
    assert lib.ref_read_gridfile(GRIDFILE.encode(), ng, 3, dp(bounds), dp(areas), dp(vols)) == 0
    b = bounds.reshape(-1, 6)
    assert np.array_equal(g["coord3lo"], b[:, 0]) and np.array_equal(g["coord2hi"], b[:, 5])
    assert np.array_equal(g["gbxarea"], areas) and np.array_equal(g["volume"], vols)

    sd = B.initsupers(SUPERSFILE, 3)
    n = sd["xi"].size
    out = {k: np.zeros(n, dtype=dt) for k, dt in (("gbx", np.uint32), ("xi", np.uint64),
                                                   ("radius", np.float64), ("msol", np.float64),
                                                   ("c3", np.float64), ("c1", np.float64),
                                                   ("c2", np.float64))}
    rc = lib.ref_read_initsupers(
        SUPERSFILE.encode(), n, 3, out["gbx"].ctypes.data_as(C.POINTER(C.c_uint32)),
        out["xi"].ctypes.data_as(C.POINTER(C.c_uint64)),
        *[dp(out[k]) for k in ("radius", "msol", "c3", "c1", "c2")])
    assert rc == 0
    assert np.array_equal(sd["sdgbxindex"], out["gbx"]) and np.array_equal(sd["xi"], out["xi"])
    for a, bk in (("radius", "radius"), ("msol", "msol"), ("coord3", "c3"), ("coord1", "c1"),
                  ("coord2", "c2")):
        assert np.array_equal(sd[a], out[bk]), a

    nsteps = int(EXP["nsteps"])
    paths = (C.c_char_p * 7)(*[PATHS[f].encode() for f in B.FromFileDynamics.FIELDS])
    ndims = np.asarray(EXP["ndims"], dtype=np.uint64)
    dyn = B.FromFileDynamics(PATHS, ndims, 3, nsteps)
    names = ("press", "temp", "qvap", "qcond", "wvel_lo", "wvel_hi", "uvel_lo", "uvel_hi",
             "vvel_lo", "vvel_hi")
    for s in range(nsteps):
        outs = [np.zeros(ng) for _ in names]
        arr = (C.POINTER(C.c_double) * 10)(*[dp(o) for o in outs])
        assert lib.ref_fromfile_state(paths, 3, ndims.ctypes.data_as(C.POINTER(C.c_uint64)),
                                      nsteps, s, arr) == 0
        st = dyn.state(g["volume"])
        for name, o in zip(names, outs):
            assert np.array_equal(st[name], o), (s, name)
        dyn.advance()


def run_from_files(lib, prefix, nsteps=3):
    """A domain set up from the files and driven by them: every 1 s coupling step the gridbox
    states come from the next time step of the dynamics files."""
    g = B.gridfile(GRIDFILE, 3)
    sd = B.initsupers(SUPERSFILE, 3)
    p = make_params(condtstep=1.0, colltstep=1.0, motiontstep=1.0,
                    coll_prob=abi.PROB_LONG, coll_enact=abi.ENACT_COALBURE,
                    motion_tv=abi.TV_ROGERSGK, seed=5,
                    monitors=abi.MONITOR_MASSMOMENTS | abi.MONITOR_PRECIPITATION)
    s = SDM(p, g, sd["xi"].size, lib=lib, prefix=prefix)
    dyn = B.FromFileDynamics(PATHS, g["ndims"], 3, nsteps)
    s.upload_state(dyn.state(g["volume"]))
    s.upload_supers(sd)
    s.monitors_begin()
    for k in range(nsteps):
        s.run_step(k * 100, (k + 1) * 100)
        dyn.advance()
        if k + 1 < nsteps:
            st = dyn.state(g["volume"])
            s.upload_state(st)
    s.check()
    return s


@needs_ref
def test_domain_from_files_oracle_matches_cleo():
    o = run_from_files(K.oracle_lib(), "oc")
    r = run_from_files(K.ref_lib(), "ref")
    K.assert_same_domain(o.download_supers(), r.download_supers(), rtol=0.0, what="from files")
    mo, mr = o.download_monitors(), r.download_monitors()
    for f, dt in abi.MONITOR_FIELDS:
        assert np.array_equal(mo[f], mr[f], equal_nan=(dt != np.uint64)), f
