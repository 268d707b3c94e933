"""CUDA-graph replay of batched SDM steps gives the same results as eager launches and as the
oracle, for uniform and mixed sub-step patterns (each distinct pattern is its own graph)."""
import numpy as np
import pytest

import checkers as K
from cleo_b200 import abi, workloads as W
from cleo_b200.config import realtime2step
from cleo_b200.sdm import make_sdm

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def lib():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    return abi.load_library()


def _workload(pattern):
    w = W.uneven3d(ndims=(8, 12, 10), seed=21)
    w["params"].exec_mode = abi.EXEC_BATCHED
    if pattern == "mixed":  # collisions every 2 s, condensation and motion every 1 s
        w["params"].collstep = realtime2step(2.0)
        w["params"].coll_delt = 2.0
    return w


@pytest.mark.parametrize("pattern", ["uniform", "mixed"])
def test_graphs_match_eager_and_oracle(lib, pattern):
    w = _workload(pattern)
    runs = {}
    for name, graphs in (("graph", 1), ("eager", 0)):
        s = make_sdm(w, lib=lib)
        assert lib.cleo_b200_set_graphs(s.ctx, graphs) == 0
        ts = w["tstep"]
        for k in range(6):
            s.run_step(k * ts, (k + 1) * ts)
        s.check()
        runs[name] = s
    o = make_sdm(w, lib=K.oracle_lib(cr=True), prefix="oc")
    for k in range(6):
        o.run_step(k * w["tstep"], (k + 1) * w["tstep"])
    K.assert_identical_run(runs["graph"], runs["eager"], "graph vs eager")
    K.assert_identical_run(runs["graph"], o, "graph vs oracle")


def test_graph_step_after_irregular_call(lib):
    # a call over several SDM steps, then single steps: the device step time stays in sync
    w = _workload("uniform")
    ts = w["tstep"]
    g = make_sdm(w, lib=lib)
    e = make_sdm(w, lib=lib)
    lib.cleo_b200_set_graphs(e.ctx, 0)
    g.run_step(0, 3 * ts)
    g.run_step(3 * ts, 4 * ts)
    g.run_step(4 * ts, 5 * ts)
    for k in range(5):
        e.run_step(k * ts, (k + 1) * ts)
    g.check()
    e.check()
    K.assert_same_domain(g.download_supers(), e.download_supers(), rtol=0.0, what="irregular")


def test_autotune_keeps_results_and_picks_a_candidate(lib):
    import ctypes as C
    w = _workload("uniform")
    ts = w["tstep"]
    tuned = make_sdm(w, lib=lib)
    plain = make_sdm(w, lib=lib)
    assert lib.cleo_b200_autotune(tuned.ctx, 2) == 0
    cfg = (C.c_int32 * 4)()
    for k in range(10):
        tuned.run_step(k * ts, (k + 1) * ts)
        plain.run_step(k * ts, (k + 1) * ts)
        rc = lib.cleo_b200_tuned_config(tuned.ctx, cfg)
        assert rc == (1 if k < 7 else 0)
    tuned.check()
    K.assert_same_domain(tuned.download_supers(), plain.download_supers(), rtol=0.0, what="tuned")
    assert cfg[0] in (128, 256) and cfg[1] in (4, 5)
    assert cfg[2] in (64, 128) and cfg[3] in (2, 3)
    # plain schedule: nothing to tune
    w["params"].exec_mode = abi.EXEC_PLAIN
    p = make_sdm(w, lib=lib)
    assert lib.cleo_b200_autotune(p.ctx, 1) == abi.CODE["CLEO_ERR_ARGUMENT"]


@pytest.mark.parametrize("cfg", [(256, 3, 64, 2), (128, 4, 128, 2), (256, 4, 128, 3),
                                 (128, 5, 20, 3), (256, 5, 64, 2)])
def test_launch_configs_match_oracle(lib, cfg):
    """Every launch configuration the autotuner can choose (and an arbitrary warp-kernel limit)
    gives the oracle's results; the workload has gridboxes on both sides of 64 and 128."""
    import ctypes as C
    w = W.uneven3d(ndims=(6, 8, 8), seed=23, median=60.0, sigma=0.5)
    w["params"].exec_mode = abi.EXEC_BATCHED
    counts = np.bincount(w["supers"]["sdgbxindex"], minlength=w["grid"]["ngbxs"])
    assert counts.max() > 128 and ((counts > 64) & (counts <= 128)).sum() > 20
    g = make_sdm(w, lib=lib)
    arr = (C.c_int32 * 4)(*cfg)
    assert lib.cleo_b200_set_launch_config(g.ctx, arr) == 0
    got = (C.c_int32 * 4)()
    assert lib.cleo_b200_tuned_config(g.ctx, got) == 0 and tuple(got) == cfg
    o = make_sdm(w, lib=K.oracle_lib(cr=True), prefix="oc")
    for k in range(4):
        g.run_step(k * w["tstep"], (k + 1) * w["tstep"])
        o.run_step(k * w["tstep"], (k + 1) * w["tstep"])
    g.check()
    K.assert_identical_run(g, o, str(cfg))
    for bad_cfg in ((256, 3, 129, 2), (256, 3, 64, 4)):
        bad = (C.c_int32 * 4)(*bad_cfg)
        assert lib.cleo_b200_set_launch_config(g.ctx, bad) == abi.CODE["CLEO_ERR_ARGUMENT"]


def test_async_state_upload_matches_sync(lib):
    """States uploaded asynchronously (copy stream, taken at the next step's start) and budgets
    copied back asynchronously give the synchronous calls' results, with states that change
    every step."""
    w = _workload("uniform")
    ts = w["tstep"]
    rng = np.random.default_rng(3)
    states = []
    for _ in range(5):
        st = {f: w["state"][f].copy() for f in abi.STATE_FIELDS}
        st["temp"] = st["temp"] * (1.0 + 2e-3 * rng.standard_normal(st["temp"].size))
        st["qvap"] = st["qvap"] * (1.0 + 5e-3 * rng.standard_normal(st["qvap"].size))
        states.append(st)
    a, b = make_sdm(w, lib=lib), make_sdm(w, lib=lib)
    ng = w["grid"]["ngbxs"]
    bud_a, bud_b = [], []
    for k in range(5):
        a.upload_state(states[k])
        a.run_step(k * ts, (k + 1) * ts)
        bud_a.append(a.download_budgets())
    for k in range(5):
        b.upload_state_async(states[k])
        b.run_step(k * ts, (k + 1) * ts)
        cm, it = np.zeros(ng), np.zeros(ng, dtype=np.uint64)
        b.download_budgets_async(cm, it)
        bud_b.append((cm, it))
    b.synchronize()
    for (ca, ia), (cb, ib) in zip(bud_a, bud_b):
        assert np.array_equal(ca, cb) and np.array_equal(ia, ib)
    K.assert_same_domain(a.download_supers(), b.download_supers(), rtol=0.0, what="async")
    sa, sb = a.download_state(), b.download_state()
    for f in abi.STATE_FIELDS:
        assert np.array_equal(sa[f], sb[f]), f
    # a synchronous upload replaces states staged but not yet taken
    b.upload_state_async(states[0])
    b.upload_state(states[4])
    a.upload_state(states[4])
    a.run_step(5 * ts, 6 * ts)
    b.run_step(5 * ts, 6 * ts)
    K.assert_same_domain(a.download_supers(), b.download_supers(), rtol=0.0, what="replaced")
    a.check()
    b.check()
