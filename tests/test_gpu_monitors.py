"""SDMMonitor members on the GPU against the oracle (itself pinned bit for bit to CLEO's monitor
code by tests/test_monitors.py), on both schedules with graph replay. The sums run in the same
order on both sides: against the correctly rounded oracle build every monitor field is equal bit
for bit. Against the host-libm build, whose radii differ from the correctly rounded ones in the
last bits where the libm misrounds: multiplicity moments (u64) exact; precipitation within 1e-12
relative; float mass moments within 1e-5 of the field's largest magnitude (a float ulp of the
moment), with inf / nan in the same places."""
import numpy as np
import pytest

import checkers as K
from cleo_b200 import abi
from test_monitors import ALL, _cases, run_monitored

pytestmark = pytest.mark.gpu


def close_monitor(a, b, dt, what):
    if dt == np.uint64:
        assert np.array_equal(a, b), (what, np.nonzero(a != b)[0][:5])
        return
    a = a.astype(np.float64)
    b = b.astype(np.float64)
    fa, fb = np.isfinite(a), np.isfinite(b)
    assert np.array_equal(fa, fb), (what, "non-finite positions")
    assert np.array_equal(np.isnan(a), np.isnan(b)), (what, "nan positions")
    assert np.array_equal(a[~fa & ~np.isnan(a)], b[~fb & ~np.isnan(b)]), (what, "infinities")
    if not fa.any():
        return
    scale = max(np.max(np.abs(a[fa])), np.max(np.abs(b[fb])))
    rtol = 1e-12 if dt == np.float64 else 1e-5
    err = np.max(np.abs(a[fa] - b[fb]))
    assert err <= rtol * scale, (what, err / max(scale, 1e-300))


def same_bits(a, b, what):
    """Equal bit for bit, except that a NaN only has to be a NaN (its payload bits are the
    producing processor's: x86 and CUDA make different default NaNs from inf - inf)."""
    a, b = np.asarray(a), np.asarray(b)
    if a.dtype.kind == "f":
        na, nb = np.isnan(a), np.isnan(b)
        assert np.array_equal(na, nb), (what, "nan positions")
        a, b = a[~na], b[~nb]
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), (what, np.nonzero(a != b)[0][:5])


@pytest.fixture(scope="module")
def lib():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return abi.load_library()


@pytest.mark.parametrize("mode", [abi.EXEC_PLAIN, abi.EXEC_BATCHED], ids=["plain", "batched"])
@pytest.mark.parametrize("name,w,nsteps", _cases(), ids=[c[0] for c in _cases()])
def test_gpu_monitors_match_oracle(lib, name, w, nsteps, mode):
    w["params"].exec_mode = mode
    g, mg = run_monitored(lib, "cleo_b200", w, nsteps, reset_at=1)
    oc, mc = run_monitored(K.oracle_lib(cr=True), "oc", w, nsteps, reset_at=1)
    for a, b in zip(mg, mc):
        for f, dt in abi.MONITOR_FIELDS:
            same_bits(a[f], b[f], (name, f))
    K.assert_identical_domain(g.download_supers(), oc.download_supers(), name)
    _, mo = run_monitored(K.oracle_lib(), "oc", w, nsteps, reset_at=1)
    for a, b in zip(mg, mo):
        for f, dt in abi.MONITOR_FIELDS:
            close_monitor(a[f], b[f], dt, (name, f))


def test_gpu_monitors_off(lib):
    from cleo_b200 import workloads as W
    w = W.uneven3d(ndims=(4, 4, 4), seed=2)
    _, outs = run_monitored(lib, "cleo_b200", w, 2, mask=0)
    for f, _ in abi.MONITOR_FIELDS:
        assert not np.any(outs[-1][f])


@pytest.mark.parametrize("mode", [abi.EXEC_PLAIN, abi.EXEC_BATCHED], ids=["plain", "batched"])
def test_gpu_domain_from_files(lib, mode, monkeypatch):
    """The GPU path set up and driven from CLEO's binary files matches the oracle."""
    import test_binaryio as TB
    from cleo_b200 import config
    orig = config.make_params

    def with_mode(**kw):
        p = orig(**kw)
        p.exec_mode = mode
        return p

    monkeypatch.setattr(TB, "make_params", with_mode)
    g = TB.run_from_files(lib, "cleo_b200")
    o = TB.run_from_files(K.oracle_lib(), "oc")
    K.assert_same_domain(g.download_supers(), o.download_supers(), rtol=1e-12, what="files")
    mg, mo = g.download_monitors(), o.download_monitors()
    for f, dt in abi.MONITOR_FIELDS:
        close_monitor(mg[f], mo[f], dt, ("files", f))
    K.assert_identical_run(g, TB.run_from_files(K.oracle_lib(cr=True), "oc"), "files")
