"""The slab decomposition's host logic (cleo_b200/decomposition.py) on CPU: two gloo ranks, each
owning half the rows of a domain with winds in every direction, stepping its superdroplets through
the oracle and exchanging the emigrants after every motion step, end with exactly the
single-domain run's superdroplets (same order, same values) and states.

Both runs take each SDM step as a motion-only step, the exchange (decomposed run only), qcond
from the superdroplets now in each gridbox (CLEO applies it after the transport across ranks), and
a microphysics-only step, with the superdroplets and states moved between the two contexts through
the C ABI: so the only difference between the runs is the decomposition itself.
"""
import copy
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from cleo_b200 import abi, decomposition as D

NDIMS = (4, 5, 6)
NSTEPS = 12


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _workload():
    from cleo_b200 import workloads as W
    w = W.uneven3d(ndims=NDIMS, seed=31)
    st = w["state"]
    st["vvel_lo"][:] = -0.9
    st["vvel_hi"][:] = 1.6
    st["uvel_lo"][:] = 0.4
    st["uvel_hi"][:] = -0.3
    st["wvel_lo"][:] = 0.5
    st["wvel_hi"][:] = -0.2
    return w


def _halves(w):
    """Contexts for the motion-only and the microphysics-only halves of a step."""
    import checkers as K
    from cleo_b200.sdm import SDM
    pm, pu = copy.copy(w["params"]), copy.copy(w["params"])
    pm.condstep = pm.collstep = abi.STEP_OFF
    pu.motionstep = abi.STEP_OFF
    cap = 2 * len(w["supers"]["xi"])
    lib = K.oracle_lib()
    return (SDM(pm, w["grid"], cap, lib=lib, prefix="oc"),
            SDM(pu, w["grid"], cap, lib=lib, prefix="oc"))


def _step(ctx, state, supers, t, ts):
    ctx.upload_state(state)
    ctx.upload_supers(supers)
    ctx.run_step(t * ts, (t + 1) * ts)
    ctx.check()
    return ctx.download_state(), ctx.download_supers()


def _single_domain():
    w = _workload()
    cm, cu = _halves(w)
    st, sd = w["state"], w["supers"]
    ts = w["tstep"]
    ng = w["grid"]["ngbxs"]
    for t in range(NSTEPS):
        st, sd = _step(cm, st, sd, t, ts)
        q = D.qcond_of_gridboxes(sd, st, 0, ng)
        # the host restatement gives the oracle's own qcond after motion, bit for bit
        assert np.array_equal(q, st["qcond"]), t
        st["qcond"] = q
        st, sd = _step(cu, st, sd, t, ts)
    return st, sd


def _rank_main(rank, world, port, out):
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        w = _workload()
        ranges = D.slab_ranges(NDIMS, world)
        lo, hi = ranges[rank]
        sd0 = w["supers"]
        mine = (sd0["sdgbxindex"] >= lo) & (sd0["sdgbxindex"] < hi)
        sd = D.take(sd0, np.nonzero(mine)[0])
        st = w["state"]
        cm, cu = _halves(w)
        ts = w["tstep"]
        moved = 0
        for t in range(NSTEPS):
            st, after = _step(cm, st, sd, t, ts)
            kept, emig, grave = D.split(after, after["n_domain"], rank, ranges)
            moved += sum(len(e["xi"]) for e in emig.values())
            imm = D.exchange(emig, rank, world, dist)
            sd = D.merge(kept, imm, grave, rank)
            st["qcond"][lo:hi] = D.qcond_of_gridboxes(sd, st, lo, hi)
            st, sd = _step(cu, st, sd, t, ts)
        nd = sd["n_domain"]
        out[rank] = ({f: sd[f][:nd] for f in D.FIELDS}, {f: sd[f][nd:] for f in D.FIELDS},
                     {f: st[f][lo:hi] for f in abi.STATE_FIELDS}, moved)
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_slab_ranges_and_owner():
    r = D.slab_ranges((4, 5, 6), 2)
    assert r == [(0, 60), (60, 120)]
    assert D.slab_ranges((4, 5, 7), 3) == [(0, 40), (40, 80), (80, 140)]
    g = np.array([0, 59, 60, 119, 120, 4000000000], dtype=np.uint32)
    assert list(D.owner(g, r)) == [0, 0, 1, 1, -1, -1]


def test_pack_round_trip():
    w = _workload()
    sd = w["supers"]
    back = D.unpack(D.pack(sd))
    for f, dt in abi.SUPERS_FIELDS:
        assert back[f].dtype == dt and np.array_equal(back[f], sd[f]), f


def test_two_ranks_reproduce_the_single_domain_run():
    import checkers as K
    st_ref, sd_ref = _single_domain()
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    moved = res[0][3] + res[1][3]
    assert moved > 50, moved  # superdroplets crossed between the slabs, both ways
    dom = D.concat([res[0][0], res[1][0]])
    grave = D.concat([res[0][1], res[1][1]])
    got = {f: np.concatenate([dom[f], grave[f]]) for f in D.FIELDS}
    got["n_domain"] = len(dom["xi"])
    got["n_total"] = len(got["xi"])
    K.assert_same_domain(got, sd_ref, rtol=0.0, what="decomposed")
    for f in abi.STATE_FIELDS:
        s = np.concatenate([res[0][2][f], res[1][2][f]])
        assert np.array_equal(s, st_ref[f]), f
