"""The multi-rank host logic on CPU: world_size-2 gloo process groups, each rank stepping its own
domain through the oracle (the CPU checker) exactly as bench.py steps one per GPU, then the
max-over-ranks / sum-over-ranks combination of timings and counts."""
import os
import socket

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from cleo_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import sys
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import checkers as K
    from cleo_b200 import workloads as W
    from cleo_b200.sdm import make_sdm
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        w = W.uneven3d(ndims=(4, 4, 4), seed=replicas.domain_seed(3, rank))
        s = make_sdm(w, lib=K.oracle_lib(), prefix="oc")
        dist.barrier()
        for k in range(2):
            s.run_step(k * w["tstep"], (k + 1) * w["tstep"])
        d = s.download_supers()
        nd = d["n_domain"]
        times, counts = replicas.combine([10.0 * (rank + 1), 5.0 - rank], [nd, 1], dist)
        out[rank] = (times, counts, nd, float(np.sum(d["radius"][:nd])))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_ranks_step_independent_domains_and_combine():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    (t0, c0, n0, s0), (t1, c1, n1, s1) = res[0], res[1]
    assert t0 == t1 == [20.0, 5.0]            # max over ranks
    assert c0 == c1 == [float(n0 + n1), 2.0]  # sum over ranks
    assert s0 != s1                           # each rank its own domain


def test_domain_seed_and_single_rank_combine():
    assert replicas.domain_seed(3, 0) == 3 and replicas.domain_seed(3, 5) == 8
    assert replicas.combine([1.5, 2.0], [3, 4]) == ([1.5, 2.0], [3.0, 4.0])
