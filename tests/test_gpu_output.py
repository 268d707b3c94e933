"""Superdroplet output from the GPU: the gather of the domain superdroplets against the
downloaded domain (same order, the reference's conversions), and a dataset observed from a
GPU run against the oracle's writer fed with the oracle's run (CPU restatement of the SDM step
and of CLEO's writer).

Bars: integer variables, time and raggedcount bit-exact; float variables within one float
spacing of the oracle's (the FP64 states agree to 1e-12 relative, so a conversion to float may
round the other way only at a rounding boundary); metadata files identical.
"""
import copy
import os
import sys

import numpy as np
import pytest

import checkers as K
from cleo_b200 import abi, workloads as W
from cleo_b200.output import SuperdropsZarr, gather_supers, read_dataset
from cleo_b200.sdm import make_sdm

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", "oracle"))
import zarr_writer as ZW  # noqa: E402

pytestmark = pytest.mark.gpu

FLOATS = ("radius", "msol", "coord3", "coord1", "coord2")


@pytest.fixture(scope="module")
def lib():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return abi.load_library()


def _nulls_workload(exec_mode):
    """Gridboxes of an uneven 3-D domain with multiplicities 1-3 and large Golovin collision
    probabilities: coalescence of equal multiplicities leaves null superdroplets in many
    gridboxes between re-sorts, while droplets sediment across gridboxes."""
    w = W.uneven3d(ndims=(6, 5, 4), seed=31)
    rng = np.random.default_rng(2)
    w["supers"]["xi"][:] = rng.integers(1, 4, w["n_sd"]).astype(np.uint64)
    p = copy.copy(w["params"])
    p.coll_prob = abi.PROB_GOLOVIN
    p.coll_enact = abi.ENACT_COALESCENCE
    p.exec_mode = exec_mode
    w["params"] = p
    w["state"]["volume"][:] = 1e-24
    return w


def _domain(d):
    nd = d["n_domain"]
    return {k: v[:nd] for k, v in d.items() if isinstance(v, np.ndarray)}


@pytest.mark.parametrize("exec_mode", [abi.EXEC_PLAIN, abi.EXEC_BATCHED])
def test_gather_matches_download(lib, exec_mode):
    w = _nulls_workload(exec_mode)
    g = make_sdm(w, lib=lib)
    ts = w["tstep"]
    saw_nulls = False
    for s in range(6):
        g.run_step(s * ts, (s + 1) * ts)
        got = gather_supers(g)
        dom = _domain(g.download_supers())
        n = len(dom["xi"])
        assert all(len(v) == n for v in got.values())
        assert np.array_equal(got["sdgbxindex"], dom["sdgbxindex"].astype(np.uint32))
        assert np.array_equal(got["sdId"], dom["sdid"].astype(np.uint32))
        assert np.array_equal(got["xi"], dom["xi"])
        for f in FLOATS:
            assert np.array_equal(got[f], dom[f].astype(np.float32)), f
        d = g.download_supers()
        saw_nulls |= bool(np.any(d["xi"][d["n_domain"]:] == 0))
    assert saw_nulls
    g.check()
    g.close()


@pytest.mark.parametrize("maxchunk", [7, 1000])
def test_dataset_matches_oracle(lib, tmp_path, maxchunk):
    w = _nulls_workload(abi.EXEC_BATCHED)
    g = make_sdm(w, lib=lib)
    o = make_sdm(w, lib=K.oracle_lib(), prefix="oc")
    ts = w["tstep"]
    interval = 2 * ts
    orc = ZW.SuperdropsDataset(os.fspath(tmp_path / "orc"), maxchunk, interval)
    with SuperdropsZarr(tmp_path / "gpu", maxchunk, interval) as z:
        for s in range(9):  # RunCLEO: observe at the start of each step, then step
            t = s * ts
            z.observe(g, t)
            orc.observe(t, _domain(o.download_supers()))
            g.run_step(t, t + ts)
            o.run_step(t, t + ts)
    orc.close()
    a, b = ZW.tree(tmp_path / "gpu"), ZW.tree(tmp_path / "orc")
    assert sorted(a) == sorted(b)
    for k in a:
        if k.endswith((".zarray", ".zattrs", ".zgroup")):
            assert a[k] == b[k], k
    dg, do = read_dataset(tmp_path / "gpu"), read_dataset(tmp_path / "orc")
    for k in ("time", "raggedcount", "sdId", "sdgbxindex", "xi"):
        assert np.array_equal(dg[k], do[k]), k
    for f in FLOATS:
        d = np.abs(dg[f].astype(np.float64) - do[f].astype(np.float64))
        assert np.all(d <= np.spacing(np.abs(do[f]))), f
    assert dg["raggedcount"].size == 5 and dg["raggedcount"].min() > 0
    g.close()
