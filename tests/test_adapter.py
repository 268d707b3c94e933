"""CPU check of the harness that runs CLEO's own RunCLEO (oracle/adapter_harness.cpp): with CLEO's
own SDMMethods and dynamics that keep the states, its observations are the oracle's stepping bit
for bit. The GPU tests use the same harness with the B200 SDMMethods of
include/cleo_b200_sdmmethods.hpp (tests/test_gpu_adapter.py)."""
import numpy as np
import pytest

import checkers as K
from cleo_b200 import abi, workloads as W
from cleo_b200.sdm import make_sdm

needs_adapter = pytest.mark.skipif(not K.adapter_available(),
                                   reason="adapter harness absent (needs CLEO's sources)")


def oracle_observations(lib, w, t_end, obsstep):
    s = make_sdm(w, lib=lib, prefix="oc")
    out, t, ts = [], 0, w["tstep"]
    while True:
        if t % obsstep == 0:
            out.append((t, s.download_supers(), s.download_state()))
        if t >= t_end:
            return out
        s.run_step(t, t + ts)
        t += ts


def same_observation(a, b, what, rtol=0.0):
    ta, da, sa = a
    tb, db, sb = b
    assert ta == tb, what
    if rtol == 0.0:
        K.assert_identical_domain(da, {k: v for k, v in db.items()}, what)
        for f in abi.STATE_FIELDS:
            assert np.array_equal(sa[f], sb[f]), (what, f)
    else:
        K.assert_same_domain(da, db, rtol=rtol, what=what)
        for f in abi.STATE_FIELDS:
            assert K.max_rel(sa[f], sb[f]) <= rtol, (what, f)


def domain_only(d):
    """An observation's superdroplets hold the domain ones only: compare those."""
    nd = d["n_domain"]
    return {k: (v[:nd] if isinstance(v, np.ndarray) else v) for k, v in d.items()} | \
        {"n_total": nd}


def with_cleo_volumes(w, states):
    """The workload with the gridbox volumes CLEO's maps computed from the bounds (dz dx dy;
    they differ from the workload's in the last bits)."""
    w = dict(w)
    w["state"] = dict(w["state"])
    w["state"]["volume"] = states["volume"].copy()
    return w


@needs_adapter
def test_runcleo_with_cleo_sdmmethods_is_the_oracle():
    w = W.uneven3d(ndims=(6, 8, 8), seed=41)
    obs = K.run_cleo(w, 1000, 200, b200=0)
    ref = oracle_observations(K.oracle_lib(), with_cleo_volumes(w, obs[0][2]), 1000, 200)
    assert [o[0] for o in obs] == [0, 200, 400, 600, 800, 1000]
    for a, b in zip(obs, ref):
        same_observation((a[0], domain_only(a[1]), a[2]), (b[0], domain_only(b[1]), b[2]),
                         f"t={a[0]}")
