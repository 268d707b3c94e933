"""The oracle against golden fixtures produced by CLEO's own sources (tests/golden/make_golden.py).

These run without the reference sources, so the oracle used as checker on any machine is pinned
to the reference's outputs: integer fields and order bit-exact, floating-point fields identical
(the fixtures and the oracle both come from the same operation order and libm).
"""
import ctypes as C
import os

import numpy as np
import pytest

import checkers as K
from cleo_b200 import abi
from cleo_b200.sdm import make_sdm


@pytest.mark.parametrize("fname", K.step_fixtures())
def test_oracle_matches_golden_step(fname):
    w, exp = K.load_step_fixture(os.path.join(K.GOLDEN, fname))
    a = make_sdm(w, lib=K.oracle_lib(), prefix="oc")
    for s in range(exp["nsteps"]):
        a.run_step(s * w["tstep"], (s + 1) * w["tstep"])
    d = a.download_supers()
    K.assert_same_domain(d, exp["supers"], rtol=1e-15, what=fname)
    st = a.download_state()
    for f in abi.STATE_FIELDS:
        assert K.max_rel(st[f], exp["state"][f]) <= 1e-15, (fname, f)
    assert K.max_rel(a.download_budgets()[0], exp["cond_mass"]) <= 1e-14


@pytest.mark.parametrize("tag", ["reftol", "tight"])
def test_oracle_matches_golden_condsolve(tag):
    z = np.load(os.path.join(K.GOLDEN, "condsolve.npz"))
    p = K.params_from_bytes(z[f"params_{tag}"])
    w = {k: z[k] for k in ("radius", "msol", "temp", "press", "s_ratio", "delt")}
    rc, r, it = K.condsolve(K.oracle_lib(), "oc", p, w)
    assert rc == 0
    assert K.max_rel(r, z[f"out_{tag}"]) <= 1e-15


def test_oracle_matches_golden_terminal_velocity():
    z = np.load(os.path.join(K.GOLDEN, "terminalv.npz"))
    lib = K.oracle_lib()
    for kind in (abi.TV_SIMMEL, abi.TV_ROGERSYAU, abi.TV_ROGERSGK):
        mine = np.array([lib.oc_terminal_velocity(kind, x) for x in z["radius"]])
        assert K.max_rel(mine, z[f"tv_{kind}"]) <= 1e-15


def test_golden_fixtures_present():
    names = K.step_fixtures()
    assert len(names) >= 6 and os.path.exists(os.path.join(K.GOLDEN, "condsolve.npz"))
