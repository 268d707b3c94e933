"""CPU tests of the oracle's two builds and of its threaded gridbox loops.

* Threads: oc_step's loops over gridboxes may run on OpenMP threads (so that the oracle can check
  full-size domains); every gridbox's work is independent within a loop, so the results, the
  error codes and their attribution must be the same as on one thread, bit for bit.
* liboracle_cr.so is the oracle with correctly rounded pow and exp (the CUDA path's arithmetic);
  liboracle.so, with the host libm, is pinned bit for bit to CLEO's own sources. The two may
  differ only where the host libm misrounds, which must stay within the parity bar (1e-12).
"""
import numpy as np
import pytest

import checkers as K
from cleo_b200 import abi, workloads as W
from cleo_b200.sdm import CleoError, make_sdm
from test_oracle import ERRS, VARIANTS, _err_case


def _run(lib, w, nsteps, threads=1):
    K.oracle_threads(lib, threads)
    try:
        s = make_sdm(w, lib=lib, prefix="oc")
        ts = w["tstep"]
        for k in range(nsteps):
            s.run_step(k * ts, (k + 1) * ts)
        return s.download_supers(), s.download_state(), s.download_budgets()
    finally:
        K.oracle_threads(lib, 1)


def _same(a, b, what):
    da, sa, ba = a
    db, sb, bb = b
    K.assert_same_domain(da, db, rtol=0.0, what=what)
    for f in abi.STATE_FIELDS:
        assert np.array_equal(sa[f], sb[f]), (what, f)
    assert np.array_equal(ba[0], bb[0]) and np.array_equal(ba[1], bb[1]), what


@pytest.mark.parametrize("name,build,nsteps", VARIANTS, ids=[v[0] for v in VARIANTS])
def test_threads_give_the_same_doubles(name, build, nsteps):
    lib = K.oracle_lib()
    _same(_run(lib, build(), nsteps, 1), _run(lib, build(), nsteps, 4), name)


def test_threads_on_a_3d_domain():
    lib = K.oracle_lib(cr=True)
    w = W.uneven3d(ndims=(8, 16, 16), seed=5)
    _same(_run(lib, w, 3, 1), _run(lib, w, 3, 6), "uneven3d 8x16x16")


@pytest.mark.parametrize("name,pov,sov,dov,code", ERRS, ids=[e[0] for e in ERRS])
def test_threads_report_the_first_error(name, pov, sov, dov, code):
    lib = K.oracle_lib()
    errs = []
    for threads in (1, 3):
        K.oracle_threads(lib, threads)
        try:
            s = make_sdm(_err_case(pov, sov, dov), lib=lib, prefix="oc")
            with pytest.raises(CleoError) as ei:
                for k in range(3):
                    s.run_step(k * 100, (k + 1) * 100)
            e = s.status()
            errs.append((ei.value.name, e.gbxindex, e.index))
        finally:
            K.oracle_threads(lib, 1)
    assert errs[0] == errs[1] and errs[0][0] == code, errs


@pytest.mark.parametrize("name,build,nsteps", VARIANTS, ids=[v[0] for v in VARIANTS])
def test_correctly_rounded_build_within_bar(name, build, nsteps):
    """Host libm against correctly rounded pow/exp: integers and order identical, every double
    within 1e-12 relative (the libm's rare misroundings are all that separates them)."""
    a = _run(K.oracle_lib(), build(), nsteps)
    b = _run(K.oracle_lib(cr=True), build(), nsteps)
    K.assert_same_domain(a[0], b[0], rtol=1e-12, what=name)
    for f in abi.STATE_FIELDS:
        assert K.max_rel(a[1][f], b[1][f]) <= 1e-12, (name, f)
    scale = float(np.max(np.abs(a[2][0]))) if len(a[2][0]) else 0.0
    assert np.all(np.abs(a[2][0] - b[2][0]) <= 1e-12 * scale + 1e-300), name
