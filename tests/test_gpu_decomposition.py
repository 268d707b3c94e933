"""The domain decomposition (cleo_b200/decomposition.py) through the GPU kernels.

Two ranks' domains (whole rows of constant coord2 index each) run in one process on one GPU, each
with its own contexts; after every motion step the emigrants go to their destination through the
host (decomposition.split / merge, the exchange's order rules), qcond of the rank's gridboxes is
recomputed from the superdroplets now in them, and the microphysics runs. The union of the ranks'
superdroplets (order included) and their gridboxes' states must equal the single-domain run bit
for bit, and that run — a step split at the exchange — must equal the library's whole step. The
exchange's collectives (counts all-gathered, records by point-to-point send/receive) are covered
by test_decomposition.py's two gloo ranks; no kernel here waits on another context.
"""
import copy

import numpy as np
import pytest

import checkers as K
from cleo_b200 import abi, decomposition as D
from cleo_b200.sdm import SDM, make_sdm
from test_decomposition import NDIMS, NSTEPS, _step, _workload

pytestmark = pytest.mark.gpu


def _gpu_halves(w):
    """GPU contexts (batched schedule) for the motion-only and the microphysics-only halves of a
    step."""
    pm, pu = copy.copy(w["params"]), copy.copy(w["params"])
    pm.condstep = pm.collstep = abi.STEP_OFF
    pu.motionstep = abi.STEP_OFF
    pm.exec_mode = pu.exec_mode = abi.EXEC_BATCHED
    cap = 2 * len(w["supers"]["xi"])
    return SDM(pm, w["grid"], cap), SDM(pu, w["grid"], cap)


def _copy_state(st):
    return {k: np.array(v, copy=True) for k, v in st.items()}


def test_gpu_two_slabs_reproduce_the_single_domain_run():
    import torch
    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    w = _workload()
    ts, ng = w["tstep"], w["grid"]["ngbxs"]

    # the library's whole step, and the same step split at the exchange, on one domain
    full_w = dict(w)
    full_w["params"] = copy.copy(w["params"])
    full_w["params"].exec_mode = abi.EXEC_BATCHED
    full = make_sdm(full_w)
    for t in range(NSTEPS):
        full.run_step(t * ts, (t + 1) * ts)
    full.check()
    st_full, sd_full = full.download_state(), full.download_supers()
    full.close()

    cm, cu = _gpu_halves(w)
    st, sd = _copy_state(w["state"]), w["supers"]
    for t in range(NSTEPS):
        st, sd = _step(cm, st, sd, t, ts)
        q = D.qcond_of_gridboxes(sd, st, 0, ng)
        assert np.array_equal(q, st["qcond"]), t  # the device's qcond after motion, bit for bit
        st, sd = _step(cu, st, sd, t, ts)
    cm.close()
    cu.close()
    K.assert_same_domain(sd, sd_full, rtol=0.0, what="split step")
    for f in abi.STATE_FIELDS:
        assert np.array_equal(st[f], st_full[f]), f

    # two ranks
    ranges = D.slab_ranges(NDIMS, 2)
    sd0 = w["supers"]
    ranks = []
    for r, (lo, hi) in enumerate(ranges):
        mine = (sd0["sdgbxindex"] >= lo) & (sd0["sdgbxindex"] < hi)
        ranks.append({"sd": D.take(sd0, np.nonzero(mine)[0]), "st": _copy_state(w["state"]),
                      "ctx": _gpu_halves(w)})
    moved = 0
    for t in range(NSTEPS):
        parts = []
        for r, rk in enumerate(ranks):
            rk["st"], after = _step(rk["ctx"][0], rk["st"], rk["sd"], t, ts)
            parts.append(D.split(after, after["n_domain"], r, ranges))
        for r, rk in enumerate(ranks):
            kept, _, grave = parts[r]
            imm = {s: parts[s][1][r] for s in range(len(ranks))
                   if s != r and len(parts[s][1][r]["xi"])}
            moved += sum(len(e["xi"]) for e in imm.values())
            rk["sd"] = D.merge(kept, imm, grave, r)
            lo, hi = ranges[r]
            rk["st"]["qcond"][lo:hi] = D.qcond_of_gridboxes(rk["sd"], rk["st"], lo, hi)
        for rk in ranks:
            rk["st"], rk["sd"] = _step(rk["ctx"][1], rk["st"], rk["sd"], t, ts)
    for rk in ranks:
        for c in rk["ctx"]:
            c.close()
    assert moved > 50, moved  # superdroplets crossed between the slabs, both ways

    doms, graves = [], []
    for rk in ranks:
        nd = rk["sd"]["n_domain"]
        doms.append({f: rk["sd"][f][:nd] for f in D.FIELDS})
        graves.append({f: rk["sd"][f][nd:] for f in D.FIELDS})
    dom, grave = D.concat(doms), D.concat(graves)
    got = {f: np.concatenate([dom[f], grave[f]]) for f in D.FIELDS}
    got["n_domain"] = len(dom["xi"])
    got["n_total"] = len(got["xi"])
    K.assert_same_domain(got, sd_full, rtol=0.0, what="decomposed")
    for f in abi.STATE_FIELDS:
        s = np.concatenate([ranks[r]["st"][f][lo:hi] for r, (lo, hi) in enumerate(ranges)])
        assert np.array_equal(s, st_full[f]), f
