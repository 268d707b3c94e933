"""SDMMonitor members (mass-moment changes of all droplets and of raindrops, precipitation): the
C restatement against CLEO's own monitor code (MonitorMassMomentsChange, MonitorPrecipitation,
massmoments_observer.cpp) compiled unmodified in the reference build. Bit for bit: the moments
are sums in the superdroplets' order on both sides."""
import numpy as np
import pytest

import checkers as K
from cleo_b200 import abi, workloads as W
from cleo_b200.sdm import make_sdm

pytestmark = pytest.mark.skipif(not K.ref_available(), reason="reference build absent")

ALL = abi.MONITOR_MASSMOMENTS | abi.MONITOR_RAINMASSMOMENTS | abi.MONITOR_PRECIPITATION


def _rainshaft_with_drizzle():
    w = W.rainshaft(nz=24, per_gbx=48, seed=8)
    r = w["supers"]["radius"]
    r[::37] = 300.0   # 300 um drops fall ~2.4 m/s through the 20 m boxes and out of the bottom
    return w


def _cases():
    rs = _rainshaft_with_drizzle()                        # sedimentation, rain, out of the bottom
    u3 = W.uneven3d(ndims=(6, 5, 4), seed=11)             # collisions, condensation, motion
    bb = W.bubble3d(ndims=(8, 6, 4), seed=2)              # 2-D flow, wraps
    return [("rainshaft", rs, 30), ("uneven3d", u3, 4), ("bubble3d", bb, 4)]


def run_monitored(lib, prefix, w, nsteps, mask=ALL, reset_at=None):
    w["params"].monitors = mask
    s = make_sdm(w, lib=lib, prefix=prefix)
    s.monitors_begin()
    outs = []
    for k in range(nsteps):
        s.run_step(k * w["tstep"], (k + 1) * w["tstep"])
        if reset_at is not None and k == reset_at:
            outs.append(s.download_monitors(reset=True))
    s.check()
    outs.append(s.download_monitors())
    return s, outs


@pytest.mark.parametrize("name,w,nsteps", _cases(), ids=[c[0] for c in _cases()])
def test_oracle_monitors_match_reference(name, w, nsteps):
    _, mo = run_monitored(K.oracle_lib(), "oc", w, nsteps, reset_at=1)
    _, mr = run_monitored(K.ref_lib(), "ref", w, nsteps, reset_at=1)
    for a, b in zip(mo, mr):
        for f, dt in abi.MONITOR_FIELDS:
            # float moments of heavy drops can overflow (inf, then nan) on both sides alike
            same = np.array_equal(a[f], b[f], equal_nan=(dt != np.uint64))
            assert same, (name, f, np.nonzero(a[f] != b[f])[0][:5])
    last = mo[-1]
    assert np.any(last["mom0_micro"] != 0) or np.any(last["mom1_micro"] != 0)
    if name == "rainshaft":
        assert np.any(last["precip"] > 0)


def test_monitors_off_leave_zeros():
    w = W.uneven3d(ndims=(4, 4, 4), seed=2)
    _, outs = run_monitored(K.oracle_lib(), "oc", w, 2, mask=0)
    for f, _ in abi.MONITOR_FIELDS:
        assert not np.any(outs[-1][f])
